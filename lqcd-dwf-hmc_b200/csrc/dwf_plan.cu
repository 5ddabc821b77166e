// Operator plan, mode dispatch, solvers and the extern "C" boundary of the
// B200 domain-wall library (declared in include/b200dwf.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/b200dwf.h"
#include "dwf_hop.cuh"
#include "dwf_kernels.h"

using namespace b200;

// ------------------------------------------------------------ errors
namespace {
thread_local std::string g_err = "no error";

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define B200_CHECK_CUDA(call)                                                      \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(B200_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,           \
                  cudaGetErrorString(e_));                                         \
  } while (0)

bool ls_supported(int ls) { return ls == 4 || ls == 6 || ls == 8 || ls == 12 || ls == 16; }
}  // namespace

// ------------------------------------------------------------ chiral maps
// Every fifth-dimension operator of the even/odd DWF matrix is block-diagonal
// in chirality x+- = v_p +- v_(p+2) (Dirac basis, gamma5 swaps spins p, p+2)
// and acts identically on every site, color, re/im and spin pair.  A map is
// stored as two dense Ls x Ls real matrices: m[chi*Ls*Ls + s*Ls + t].
namespace {

struct Chiral {
  int ls = 0;
  std::vector<double> m;
  Chiral() {}
  explicit Chiral(int n) : ls(n), m(2 * n * n, 0.0) {}
  double& at(int chi, int s, int t) { return m[(size_t)chi * ls * ls + s * ls + t]; }
  double at(int chi, int s, int t) const { return m[(size_t)chi * ls * ls + s * ls + t]; }
  static Chiral identity(int n, double sp = 1.0, double sm = 1.0) {
    Chiral r(n);
    for (int s = 0; s < n; ++s) { r.at(0, s, s) = sp; r.at(1, s, s) = sm; }
    return r;
  }
};

// C = A * B  (B applied first)
Chiral mul(const Chiral& A, const Chiral& B) {
  Chiral C(A.ls);
  for (int chi = 0; chi < 2; ++chi)
    for (int s = 0; s < A.ls; ++s)
      for (int t = 0; t < A.ls; ++t) {
        double v = 0;
        for (int k = 0; k < A.ls; ++k) v += A.at(chi, s, k) * B.at(chi, k, t);
        C.at(chi, s, t) = v;
      }
  return C;
}

Chiral transpose(const Chiral& A) {
  Chiral C(A.ls);
  for (int chi = 0; chi < 2; ++chi)
    for (int s = 0; s < A.ls; ++s)
      for (int t = 0; t < A.ls; ++t) C.at(chi, s, t) = A.at(chi, t, s);
  return C;
}

Chiral scaled(const Chiral& A, double a) {
  Chiral C = A;
  for (auto& v : C.m) v *= a;
  return C;
}

// Build a chiral map from a function that applies it to one chirality column.
template <typename Fn>
Chiral from_fn(int ls, Fn fn) {
  Chiral C(ls);
  std::vector<double> x(ls), y(ls);
  for (int chi = 0; chi < 2; ++chi)
    for (int t = 0; t < ls; ++t) {
      std::fill(x.begin(), x.end(), 0.0);
      x[t] = 1.0;
      fn(chi, x.data(), y.data());
      for (int s = 0; s < ls; ++s) C.at(chi, s, t) = y[s];
    }
  return C;
}

struct DwfCoef {
  int ls;
  double mq, M0, alpha;
  std::vector<double> b, c, dp, dm, e, f;
  double g;
};

// LU coefficients of D_ee (reference src/lib_alt_Accel/Fopr/
// afopr_Domainwall_5din_eo-tmpl.h:410-441, identical in the corelib
// src/lib/Fopr/afopr_Domainwall_eo-tmpl.h:239-273).
void set_precond(DwfCoef& k) {
  const int n = k.ls;
  k.dp.assign(n, 0); k.dm.assign(n, 0); k.e.assign(n, 0); k.f.assign(n, 0);
  for (int s = 0; s < n; ++s) {
    k.dp[s] = k.alpha * (1.0 + k.b[s] * (4.0 - k.M0));
    k.dm[s] = k.alpha * (1.0 - k.c[s] * (4.0 - k.M0));
  }
  k.e[0] = k.mq * k.dm[n - 1] / k.dp[0];
  k.f[0] = k.mq * k.dm[0] / k.alpha;
  for (int s = 1; s < n - 1; ++s) {
    k.e[s] = k.e[s - 1] * k.dm[s - 1] / k.dp[s];
    k.f[s] = k.f[s - 1] * k.dm[s] / k.dp[s - 1];
  }
  k.g = k.e[n - 2] * k.dm[n - 2];
}

// M5-type map y = cw*Wf(x) + cv*(Fup (1-g5) x(s+1) + Fdn (1+g5) x(s-1)) in the
// chiral basis.  Wf = (alpha P+ + P-) at s=0, (P+ + alpha P-) at s=Ls-1, alpha
// in the bulk; Fup = alpha/2 except -mq/2 at s=Ls-1, Fdn = alpha/2 except
// -mq/2 at s=0 (walls wrap in s).  Reference: D_eo pre-factor
// mult_Domainwall_5din_eo_openacc-inc.h:122-227, D_ee :14-119.
Chiral m5_map(const DwfCoef& k, const std::vector<double>& cw, const std::vector<double>& cv) {
  const int n = k.ls;
  return from_fn(n, [&](int chi, const double* x, double* y) {
    for (int s = 0; s < n; ++s) {
      double wf;
      if (chi == 0) wf = (s == n - 1) ? 1.0 : k.alpha;
      else wf = (s == 0) ? 1.0 : k.alpha;
      const double fup = (s == n - 1) ? -0.5 * k.mq : 0.5 * k.alpha;
      const double fdn = (s == 0) ? -0.5 * k.mq : 0.5 * k.alpha;
      double v = cw[s] * wf * x[s];
      if (chi == 0) v += 2.0 * cv[s] * fdn * x[(s - 1 + n) % n];
      else v += 2.0 * cv[s] * fup * x[(s + 1) % n];
      y[s] = v;
    }
  });
}

// M_ee^-1 = U^-1 L^-1 (corelib afopr_Domainwall_eo-tmpl.h:1022-1119; Accel
// mult_Domainwall_5din_LUinv_openacc-inc.h:14-200), chiral form.
Chiral lu_inv_map(const DwfCoef& k) {
  const int n = k.ls;
  return from_fn(n, [&](int chi, const double* w, double* out) {
    std::vector<double> v(n);
    // L^-1
    if (chi == 0) {
      v[0] = w[0];
      for (int s = 1; s < n; ++s) v[s] = w[s] + k.dm[s] / k.dp[s - 1] * v[s - 1];
    } else {
      double y = 0;
      for (int s = 0; s < n - 1; ++s) { v[s] = w[s]; y += k.e[s] * w[s]; }
      v[n - 1] = w[n - 1] - y;
    }
    // U^-1
    if (chi == 0) {
      out[n - 1] = k.alpha * v[n - 1] / (k.dp[n - 1] + k.g);
      const double Y = out[n - 1];
      for (int s = n - 2; s >= 0; --s) out[s] = (v[s] - k.f[s] * Y) / k.dp[s];
    } else {
      out[n - 1] = v[n - 1] / (k.dp[n - 1] + k.g);
      for (int s = n - 2; s >= 0; --s) out[s] = (v[s] + k.dm[s] * out[s + 1]) / k.dp[s];
      out[0] *= k.alpha;
    }
  });
}

// (M_ee^-1)^+ = L^-+ U^-+ (corelib afopr_Domainwall_eo-tmpl.h:1124-1240; Accel
// mult_Domainwall_5din_LUinv_openacc-inc.h:204-398), chiral form.
Chiral lu_dag_inv_map(const DwfCoef& k) {
  const int n = k.ls;
  return from_fn(n, [&](int chi, const double* w, double* out) {
    std::vector<double> v(n);
    // U^-+
    if (chi == 0) {
      double Y = 0;
      for (int s = 0; s < n - 1; ++s) { v[s] = w[s] / k.dp[s]; Y += k.f[s] * v[s]; }
      v[n - 1] = k.alpha * (w[n - 1] - Y) / (k.dp[n - 1] + k.g);
    } else {
      v[0] = k.alpha * w[0] / k.dp[0];
      for (int s = 1; s < n - 1; ++s) v[s] = (w[s] + k.dm[s - 1] * v[s - 1]) / k.dp[s];
      v[n - 1] = (w[n - 1] + k.dm[n - 2] * v[n - 2]) / (k.dp[n - 1] + k.g);
    }
    // L^-+
    if (chi == 0) {
      out[n - 1] = v[n - 1];
      for (int s = n - 2; s >= 0; --s) out[s] = v[s] + k.dm[s + 1] / k.dp[s] * out[s + 1];
    } else {
      const double Y = v[n - 1];
      out[n - 1] = v[n - 1];
      for (int s = n - 2; s >= 0; --s) out[s] = v[s] - k.e[s] * Y;
    }
  });
}

Chiral reflect_map(int n, double sm) {
  Chiral C(n);
  for (int s = 0; s < n; ++s) { C.at(0, n - 1 - s, s) = 1.0; C.at(1, n - 1 - s, s) = sm; }
  return C;
}

enum MatId {
  MAT_M5PRE = 0,   // D_eo pre-factor (alone, before a hop)
  MAT_HALF,        // -1/2 (hop of D_eo)
  MAT_DDAGEO,      // M5^+ (-1/2 g5)            : Ddag_eo epilogue
  MAT_DEE,
  MAT_DEE_T,
  MAT_LU,
  MAT_LUDAG,
  MAT_G5R,
  MAT_R,
  MAT_K1,          // M5pre LU (-1/2)           : D chain, first hop
  MAT_K2N,         // -LU (-1/2)                : D chain, second hop (o = w - ...)
  MAT_K3,          // LUdag M5^+ (-1/2 g5)      : Ddag chain, first hop
  MAT_K4N,         // -M5^+ (-1/2 g5)           : Ddag chain, second hop
  MAT_ID,
  MAT_COUNT
};

}  // namespace

// ------------------------------------------------------------ plan
struct b200_dwf {
  int L[4];
  DwfCoef k;
  int bc[4];
  Geom g;
  double* mats = nullptr;       // device [MAT_COUNT][2][Ls][Ls]
  void* links[4] = {nullptr, nullptr, nullptr, nullptr};
  double* u_lex = nullptr;      // device copy of the lexical links
  bool have_links = false;
  double* red = nullptr;        // reduction partials
  int red_n = 0;
  double* sc = nullptr;         // solver scalars (device)
  double* sc_host = nullptr;    // pinned mirror
  double* stage = nullptr;      // device f64 staging for convert/reverse
  void* work[8][4] = {};        // work fields per precision
  const double* mat(int id) const { return mats + (size_t)id * 2 * k.ls * k.ls; }
};

namespace {

int ensure_work(b200_dwf* op, int prec, int i) {
  if (!op->work[i][prec]) {
    const size_t bytes = field_bytes(prec, op->g.vh, op->g.ls);
    if (cudaMalloc(&op->work[i][prec], bytes) != cudaSuccess)
      return fail(B200_ENOMEM, "cudaMalloc of %zu bytes for a work field failed", bytes);
  }
  return 0;
}

int link_format_for(int prec) {
  return prec == PREC_F64 ? LINK_F64_18 : (prec == PREC_F32 ? LINK_F32_12 : LINK_F16_12);
}

int ensure_links(b200_dwf* op, int prec, cudaStream_t st) {
  if (!op->have_links) return fail(B200_EINVAL, "set_config has not been called on this operator");
  const int lf = link_format_for(prec);
  if (!op->links[lf]) {
    if (cudaMalloc(&op->links[lf], link_bytes(lf, op->g.vh)) != cudaSuccess)
      return fail(B200_ENOMEM, "cudaMalloc for links failed");
    B200_CHECK_CUDA(launch_links_from_lex(lf, op->links[lf], op->u_lex, op->g, st));
  }
  return 0;
}

HopParams hop_base(const b200_dwf* op, int prec, int ieo) {
  HopParams p;
  memset(&p, 0, sizeof(p));
  p.links = op->links[link_format_for(prec)];
  p.vh = op->g.vh; p.nx2 = op->g.nx2; p.ny = op->g.ny; p.nz = op->g.nz; p.nt = op->g.nt;
  p.ls = op->g.ls;
  p.ieo = ieo;
  p.ce = 1.0;
  for (int mu = 0; mu < 4; ++mu) p.bc[mu] = op->bc[mu];
  return p;
}

SopParams sop_base(const b200_dwf* op) {
  SopParams p;
  memset(&p, 0, sizeof(p));
  p.g = op->g;
  p.ce = 1.0;
  return p;
}

int run_hop(b200_dwf* op, int prec, bool dag, HopParams& p, cudaStream_t st) {
  B200_CHECK_CUDA(launch_hop(prec, dag, p, st));
  return 0;
}

int run_sop(int prec, SopParams& p, cudaStream_t st) {
  B200_CHECK_CUDA(launch_sop(prec, p, st));
  return 0;
}

// v = E(w) with a site-local map
int apply_sop(b200_dwf* op, int prec, void* v, const void* w, int mat, cudaStream_t st) {
  SopParams p = sop_base(op);
  p.in = w; p.out1 = v; p.E = op->mat(mat);
  return run_sop(prec, p, st);
}

// D = 1 - M_ee^-1 D_eo M_oo^-1 D_oe on w; v = w - ...;  optional F(v) -> v2,
// optional |v|^2 partials.  With F the first output may be skipped (v = null).
int apply_D(b200_dwf* op, int prec, void* v, const void* w, int fmat, void* v2, double* red,
            cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 0)) || (rc = ensure_work(op, prec, 1))) return rc;
  void* t0 = op->work[0][prec];
  void* y1 = op->work[1][prec];
  if ((rc = apply_sop(op, prec, t0, w, MAT_M5PRE, st))) return rc;
  HopParams p1 = hop_base(op, prec, 1);
  p1.in = t0; p1.out1 = y1; p1.E = op->mat(MAT_K1);
  if ((rc = run_hop(op, prec, false, p1, st))) return rc;
  HopParams p2 = hop_base(op, prec, 0);
  p2.in = y1; p2.out1 = v; p2.E = op->mat(MAT_K2N);
  p2.x1 = w; p2.c_x1 = 1.0;
  if (fmat >= 0) { p2.F = op->mat(fmat); p2.out2 = v2; }
  p2.red = red;
  return run_hop(op, prec, false, p2, st);
}

// Ddag = 1 - D_eo^+ M_oo^-+ D_oe^+ M_ee^-+ on u = LUdag(x);  v = xw - ...
int apply_Ddag_from_u(b200_dwf* op, int prec, void* v, const void* xw, const void* u,
                      cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 3))) return rc;
  void* t3 = op->work[3][prec];
  HopParams p3 = hop_base(op, prec, 1);
  p3.in = u; p3.out1 = t3; p3.E = op->mat(MAT_K3);
  if ((rc = run_hop(op, prec, true, p3, st))) return rc;
  HopParams p4 = hop_base(op, prec, 0);
  p4.in = t3; p4.out1 = v; p4.E = op->mat(MAT_K4N);
  p4.x1 = xw; p4.c_x1 = 1.0;
  return run_hop(op, prec, true, p4, st);
}

int apply_Ddag(b200_dwf* op, int prec, void* v, const void* w, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 2))) return rc;
  void* u = op->work[2][prec];
  if ((rc = apply_sop(op, prec, u, w, MAT_LUDAG, st))) return rc;
  return apply_Ddag_from_u(op, prec, v, w, u, st);
}

int apply_DdagD(b200_dwf* op, int prec, void* v, const void* w, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 2)) || (rc = ensure_work(op, prec, 4))) return rc;
  void* t2 = op->work[4][prec];
  void* u = op->work[2][prec];
  if ((rc = apply_D(op, prec, t2, w, MAT_LUDAG, u, nullptr, st))) return rc;
  return apply_Ddag_from_u(op, prec, v, t2, u, st);
}

int apply_Hdag(b200_dwf* op, int prec, void* v, const void* w, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 2)) || (rc = ensure_work(op, prec, 4))) return rc;
  void* gw = op->work[4][prec];
  void* u = op->work[2][prec];
  SopParams p = sop_base(op);
  p.in = w; p.out1 = gw; p.E = op->mat(MAT_G5R); p.F = op->mat(MAT_LUDAG); p.out2 = u;
  if ((rc = run_sop(prec, p, st))) return rc;
  return apply_Ddag_from_u(op, prec, v, gw, u, st);
}

int apply_mode(b200_dwf* op, int prec, void* v, const void* w, const std::string& mode_in,
               int dag, cudaStream_t st) {
  int rc;
  if ((rc = ensure_links(op, prec, st))) return rc;
  std::string mode = mode_in;
  // mult_dag of the composite modes is the mult of the adjoint mode
  if (dag) {
    if (mode == "D") { mode = "Ddag"; dag = 0; }
    else if (mode == "Ddag") { mode = "D"; dag = 0; }
    else if (mode == "H") { mode = "Hdag"; dag = 0; }
    else if (mode == "Hdag") { mode = "H"; dag = 0; }
    else if (mode == "DdagD") { dag = 0; }
  }
  if (mode == "Deo" || mode == "Doe") {
    const int out_par = (mode == "Deo") ? (dag ? 1 : 0) : (dag ? 0 : 1);
    if (dag) {
      HopParams p = hop_base(op, prec, out_par);
      p.in = w; p.out1 = v; p.E = op->mat(MAT_DDAGEO);
      return run_hop(op, prec, true, p, st);
    }
    if ((rc = ensure_work(op, prec, 0))) return rc;
    void* t0 = op->work[0][prec];
    if ((rc = apply_sop(op, prec, t0, w, MAT_M5PRE, st))) return rc;
    HopParams p = hop_base(op, prec, out_par);
    p.in = t0; p.out1 = v; p.E = op->mat(MAT_HALF);
    return run_hop(op, prec, false, p, st);
  }
  if (mode == "Dee" || mode == "Doo") return apply_sop(op, prec, v, w, dag ? MAT_DEE_T : MAT_DEE, st);
  if (mode == "Dee_inv" || mode == "Doo_inv") return apply_sop(op, prec, v, w, dag ? MAT_LUDAG : MAT_LU, st);
  if (mode == "gm5R") return apply_sop(op, prec, v, w, MAT_G5R, st);
  if (mode == "R") return apply_sop(op, prec, v, w, MAT_R, st);
  if (mode == "D") return apply_D(op, prec, v, w, -1, nullptr, nullptr, st);
  if (mode == "H") return apply_D(op, prec, nullptr, w, MAT_G5R, v, nullptr, st);
  if (mode == "Ddag") return apply_Ddag(op, prec, v, w, st);
  if (mode == "Hdag") return apply_Hdag(op, prec, v, w, st);
  if (mode == "DdagD") return apply_DdagD(op, prec, v, w, st);
  return fail(B200_EINVAL, "mode undefined in AFopr_Domainwall_5din_eo (B200): %s", mode_in.c_str());
}

int reduce_to(b200_dwf* op, int nblocks, double* out_dev, int fin_op, cudaStream_t st) {
  B200_CHECK_CUDA(launch_finalize(op->red, nblocks, out_dev, fin_op, st));
  return 0;
}

int host_scalar(b200_dwf* op, int idx, double* out, cudaStream_t st) {
  B200_CHECK_CUDA(cudaMemcpyAsync(op->sc_host + idx, op->sc + idx, sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  *out = op->sc_host[idx];
  return 0;
}

int field_norm2_dev(b200_dwf* op, int prec, const void* x, double* out_dev, cudaStream_t st) {
  const int nb = site_s_grid(op->g.ls, op->g.vh);
  B200_CHECK_CUDA(launch_dot(prec, op->g, x, x, op->red, st));
  return reduce_to(op, nb, out_dev, FIN_SUM, st);
}

}  // namespace

// ------------------------------------------------------------ extern "C"
extern "C" {

const char* b200_last_error(void) { return g_err.c_str(); }

int b200_init(int rank, int device_offset) {
  int ndev = 0;
  B200_CHECK_CUDA(cudaGetDeviceCount(&ndev));
  if (ndev <= 0) return fail(B200_ECUDA, "no CUDA device visible");
  const int dev = (rank % ndev + device_offset) % ndev;
  B200_CHECK_CUDA(cudaSetDevice(dev));
  return 0;
}

int b200_dwf_create(b200_dwf_t** out, const int lattice[4], int Ls, double mq, double M0,
                    const double* b, const double* c, double alpha, const int bc[4]) {
  if (!out || !lattice || !bc) return fail(B200_EINVAL, "null argument");
  *out = nullptr;
  if (lattice[0] % 2 != 0 || lattice[0] < 2)
    return fail(B200_EINVAL, "Nx must be even (got %d)", lattice[0]);
  for (int mu = 1; mu < 4; ++mu)
    if (lattice[mu] < 1) return fail(B200_EINVAL, "lattice extent %d invalid", lattice[mu]);
  if (!ls_supported(Ls))
    return fail(B200_EINVAL, "extent_of_5th_dimension %d unsupported (4, 6, 8, 12, 16)", Ls);
  if (alpha == 0.0) return fail(B200_EINVAL, "parameter_alpha must be non-zero");
  b200_dwf* op = new b200_dwf();
  memcpy(op->L, lattice, sizeof(op->L));
  memcpy(op->bc, bc, sizeof(op->bc));
  op->k.ls = Ls; op->k.mq = mq; op->k.M0 = M0; op->k.alpha = alpha;
  op->k.b.assign(Ls, 1.0); op->k.c.assign(Ls, 0.0);
  if (b) op->k.b.assign(b, b + Ls);
  if (c) op->k.c.assign(c, c + Ls);
  set_precond(op->k);
  const long vol = (long)lattice[0] * lattice[1] * lattice[2] * lattice[3];
  op->g.nx2 = lattice[0] / 2; op->g.ny = lattice[1]; op->g.nz = lattice[2]; op->g.nt = lattice[3];
  op->g.ls = Ls; op->g.vh = (int)(vol / 2);

  // fifth-dimension maps
  const DwfCoef& k = op->k;
  std::vector<double> F1(Ls), F2(Ls);
  for (int s = 0; s < Ls; ++s) {
    F1[s] = k.b[s] * (4.0 - k.M0) + 1.0;
    F2[s] = k.c[s] * (4.0 - k.M0) - 1.0;
  }
  std::vector<Chiral> M(MAT_COUNT);
  const Chiral m5pre = m5_map(k, k.b, k.c);
  const Chiral half = Chiral::identity(Ls, -0.5, -0.5);
  const Chiral halfg5 = Chiral::identity(Ls, -0.5, 0.5);
  const Chiral lu = lu_inv_map(k);
  const Chiral ludag = lu_dag_inv_map(k);
  const Chiral m5dag = transpose(m5pre);
  M[MAT_M5PRE] = m5pre;
  M[MAT_HALF] = half;
  M[MAT_DDAGEO] = mul(m5dag, halfg5);
  M[MAT_DEE] = m5_map(k, F1, F2);
  M[MAT_DEE_T] = transpose(M[MAT_DEE]);
  M[MAT_LU] = lu;
  M[MAT_LUDAG] = ludag;
  M[MAT_G5R] = reflect_map(Ls, -1.0);
  M[MAT_R] = reflect_map(Ls, 1.0);
  M[MAT_K1] = mul(m5pre, mul(lu, half));
  M[MAT_K2N] = scaled(mul(lu, half), -1.0);
  M[MAT_K3] = mul(ludag, M[MAT_DDAGEO]);
  M[MAT_K4N] = scaled(M[MAT_DDAGEO], -1.0);
  M[MAT_ID] = Chiral::identity(Ls);
  std::vector<double> flat;
  for (int i = 0; i < MAT_COUNT; ++i) flat.insert(flat.end(), M[i].m.begin(), M[i].m.end());

  const int red_n = site_s_grid(Ls, op->g.vh) + hop_grid(Ls, op->g.vh);
  op->red_n = red_n;
  if (cudaMalloc(&op->mats, flat.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&op->red, (size_t)red_n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&op->sc, SC_N * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&op->sc_host, SC_N * sizeof(double)) != cudaSuccess) {
    b200_dwf_destroy(op);
    return fail(B200_ENOMEM, "device allocation for the operator plan failed");
  }
  cudaError_t e = cudaMemcpy(op->mats, flat.data(), flat.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    b200_dwf_destroy(op);
    return fail(B200_ECUDA, "upload of fifth-dimension maps failed: %s", cudaGetErrorString(e));
  }
  *out = op;
  return 0;
}

int b200_dwf_destroy(b200_dwf_t* op) {
  if (!op) return 0;
  cudaFree(op->mats);
  for (int i = 0; i < 4; ++i) cudaFree(op->links[i]);
  cudaFree(op->u_lex);
  cudaFree(op->red);
  cudaFree(op->sc);
  if (op->sc_host) cudaFreeHost(op->sc_host);
  cudaFree(op->stage);
  for (int i = 0; i < 8; ++i)
    for (int p = 0; p < 4; ++p) cudaFree(op->work[i][p]);
  delete op;
  return 0;
}

size_t b200_dwf_field_bytes(const b200_dwf_t* op, int prec) {
  if (!op || prec < 0 || prec > 3) return 0;
  return field_bytes(prec, op->g.vh, op->g.ls);
}

size_t b200_dwf_field_nreal(const b200_dwf_t* op) {
  return op ? (size_t)24 * op->g.vh * op->g.ls : 0;
}

static int set_config_common(b200_dwf_t* op, const double* u, cudaMemcpyKind kind, cudaStream_t st) {
  const size_t n = (size_t)18 * 8 * op->g.vh;   // 18 * Nvol * 4
  if (!op->u_lex && cudaMalloc(&op->u_lex, n * sizeof(double)) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for lexical links failed");
  B200_CHECK_CUDA(cudaMemcpyAsync(op->u_lex, u, n * sizeof(double), kind, st));
  op->have_links = true;
  for (int lf = 0; lf < 4; ++lf)
    if (op->links[lf]) B200_CHECK_CUDA(launch_links_from_lex(lf, op->links[lf], op->u_lex, op->g, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  return 0;
}

int b200_dwf_set_config(b200_dwf_t* op, const double* u_lex_host, void* stream) {
  if (!op || !u_lex_host) return fail(B200_EINVAL, "null argument");
  return set_config_common(op, u_lex_host, cudaMemcpyHostToDevice, (cudaStream_t)stream);
}

int b200_dwf_set_config_device(b200_dwf_t* op, const double* u_lex_dev, void* stream) {
  if (!op || !u_lex_dev) return fail(B200_EINVAL, "null argument");
  return set_config_common(op, u_lex_dev, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
}

int b200_field_convert(b200_dwf_t* op, int prec, void* v, const double* w_host, void* stream) {
  if (!op || !v || !w_host || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = b200_dwf_field_nreal(op);
  if (!op->stage && cudaMalloc(&op->stage, n * sizeof(double)) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for the staging field failed");
  B200_CHECK_CUDA(cudaMemcpyAsync(op->stage, w_host, n * sizeof(double), cudaMemcpyHostToDevice, st));
  B200_CHECK_CUDA(launch_from_corelib(prec, v, op->stage, op->g, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  return 0;
}

int b200_field_reverse(b200_dwf_t* op, int prec, double* v_host, const void* w, void* stream) {
  if (!op || !v_host || !w || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = b200_dwf_field_nreal(op);
  if (!op->stage && cudaMalloc(&op->stage, n * sizeof(double)) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for the staging field failed");
  B200_CHECK_CUDA(launch_to_corelib(prec, op->stage, w, op->g, st));
  B200_CHECK_CUDA(cudaMemcpyAsync(v_host, op->stage, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  return 0;
}

int b200_dwf_mult(b200_dwf_t* op, int prec, void* v, const void* w, const char* mode, int dag,
                  void* stream) {
  if (!op || !v || !w || !mode || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  if (v == w) return fail(B200_EINVAL, "mult: input and output fields must differ");
  return apply_mode(op, prec, v, w, mode, dag, (cudaStream_t)stream);
}

int b200_field_axpby(b200_dwf_t* op, int prec, void* y, double a, const void* x, double b,
                     void* stream) {
  if (!op || !y || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  B200_CHECK_CUDA(launch_axpby(prec, op->g, y, x, a, nullptr, b, nullptr, (cudaStream_t)stream));
  return 0;
}

int b200_field_dot(b200_dwf_t* op, int prec, const void* x, const void* y, double* result,
                   void* stream) {
  if (!op || !x || !y || !result || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = site_s_grid(op->g.ls, op->g.vh);
  B200_CHECK_CUDA(launch_dot(prec, op->g, x, y, op->red, st));
  int rc = reduce_to(op, nb, op->sc + SC_RR_NEW, FIN_SUM, st);
  if (rc) return rc;
  return host_scalar(op, SC_RR_NEW, result, st);
}

int b200_field_norm2(b200_dwf_t* op, int prec, const void* x, double* result, void* stream) {
  return b200_field_dot(op, prec, x, x, result, stream);
}

int b200_field_copy_convert(b200_dwf_t* op, int prec_out, void* out, int prec_in, const void* in,
                            void* stream) {
  if (!op || !out || !in || prec_out < 0 || prec_out > 3 || prec_in < 0 || prec_in > 3)
    return fail(B200_EINVAL, "invalid argument");
  B200_CHECK_CUDA(launch_convert(prec_out, out, prec_in, in, op->g, (cudaStream_t)stream));
  return 0;
}

// ASolver_CG on DdagD (src/lib_alt/Solver/asolver_CG-tmpl.h:118-234) with the
// iteration split into five fused kernels:
//   K1 y1 = M5pre LU (-1/2) hop(yp)                       [yp = M5pre p]
//   K2 t2 = p - LU(-1/2) hop(y1) = D p ; u = LUdag t2 ; pq = |t2|^2 = <p, DdagD p>
//   K3 t3 = LUdag M5^+ (-1/2 g5) hop^+(u)
//   K4 r  = r - alpha*(t2 - M5^+(-1/2 g5) hop^+(t3)) = r - alpha DdagD p ; rr
//   K5 x += alpha p ; p = r + beta p ; yp = M5pre p
int b200_cg_solve(b200_dwf_t* op, int prec, void* x, const void* b, int maxiter, double tol2,
                  int* nconv, double* diff, void* stream) {
  if (!op || !x || !b || prec < 0 || prec > 3 || maxiter < 0) return fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if ((rc = ensure_links(op, prec, st))) return rc;
  for (int i = 0; i < 8; ++i)
    if ((rc = ensure_work(op, prec, i))) return rc;
  void* yp = op->work[0][prec];
  void* y1 = op->work[1][prec];
  void* u = op->work[2][prec];
  void* t3 = op->work[3][prec];
  void* t2 = op->work[4][prec];
  void* r = op->work[5][prec];
  void* p = op->work[6][prec];
  void* s = op->work[7][prec];
  const Geom& g = op->g;
  const int nb_hop = hop_grid(g.ls, g.vh);

  // r = b, p = b, x = 0, rr = |r|^2, yp = M5pre p
  B200_CHECK_CUDA(launch_axpby(prec, g, r, b, 1.0, nullptr, 0.0, nullptr, st));
  B200_CHECK_CUDA(launch_axpby(prec, g, p, b, 1.0, nullptr, 0.0, nullptr, st));
  B200_CHECK_CUDA(launch_axpby(prec, g, x, nullptr, 0.0, nullptr, 0.0, nullptr, st));
  if ((rc = field_norm2_dev(op, prec, r, op->sc + SC_RR, st))) return rc;
  double bnorm2 = 0.0;
  if ((rc = host_scalar(op, SC_RR, &bnorm2, st))) return rc;
  if (!(bnorm2 > 0.0)) {
    if (nconv) *nconv = 0;
    if (diff) *diff = 0.0;
    return 0;
  }
  if ((rc = apply_sop(op, prec, yp, p, MAT_M5PRE, st))) return rc;

  int it_conv = -1;
  double rr = bnorm2;
  for (int it = 0; it < maxiter; ++it) {
    HopParams p1 = hop_base(op, prec, 1);
    p1.in = yp; p1.out1 = y1; p1.E = op->mat(MAT_K1);
    if ((rc = run_hop(op, prec, false, p1, st))) return rc;

    HopParams p2 = hop_base(op, prec, 0);
    p2.in = y1; p2.out1 = t2; p2.E = op->mat(MAT_K2N);
    p2.x1 = p; p2.c_x1 = 1.0;
    p2.F = op->mat(MAT_LUDAG); p2.out2 = u;
    p2.red = op->red;
    if ((rc = run_hop(op, prec, false, p2, st))) return rc;
    if ((rc = reduce_to(op, nb_hop, op->sc, FIN_CG_ALPHA, st))) return rc;

    HopParams p3 = hop_base(op, prec, 1);
    p3.in = u; p3.out1 = t3; p3.E = op->mat(MAT_K3);
    if ((rc = run_hop(op, prec, true, p3, st))) return rc;

    HopParams p4 = hop_base(op, prec, 0);
    p4.in = t3; p4.out1 = r; p4.E = op->mat(MAT_K4N);
    p4.ce = -1.0; p4.ce_dev = op->sc + SC_ALPHA;
    p4.x1 = r; p4.c_x1 = 1.0;
    p4.x2 = t2; p4.c_x2 = -1.0; p4.c_x2_dev = op->sc + SC_ALPHA;
    p4.red = op->red;
    if ((rc = run_hop(op, prec, true, p4, st))) return rc;
    if ((rc = reduce_to(op, nb_hop, op->sc, FIN_CG_BETA, st))) return rc;

    CgUpdParams pu;
    pu.x = x; pu.p = p; pu.r = r; pu.y = yp; pu.E = op->mat(MAT_M5PRE);
    pu.alpha = op->sc + SC_ALPHA; pu.beta = op->sc + SC_BETA; pu.g = g;
    B200_CHECK_CUDA(launch_cg_update(prec, pu, st));

    if ((rc = host_scalar(op, SC_RR, &rr, st))) return rc;
    if (!(rr == rr)) return fail(B200_ENOCONV, "CG breakdown: residual is NaN at iteration %d", it + 1);
    if (rr / bnorm2 < tol2) { it_conv = it + 1; break; }
  }

  // true residual |DdagD x - b|^2 / |b|^2
  if ((rc = apply_DdagD(op, prec, s, x, st))) return rc;
  B200_CHECK_CUDA(launch_axpby(prec, g, s, b, -1.0, nullptr, 1.0, nullptr, st));
  if ((rc = field_norm2_dev(op, prec, s, op->sc + SC_RR_NEW, st))) return rc;
  double d2 = 0.0;
  if ((rc = host_scalar(op, SC_RR_NEW, &d2, st))) return rc;
  if (diff) *diff = std::sqrt(d2 / bnorm2);
  if (nconv) *nconv = it_conv < 0 ? maxiter : it_conv;
  if (it_conv < 0) return fail(B200_ENOCONV, "CG not converged in %d iterations: |r|^2/|b|^2 = %.3e",
                               maxiter, rr / bnorm2);
  return 0;
}

}  // extern "C"
