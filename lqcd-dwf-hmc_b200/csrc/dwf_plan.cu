// Operator plan, mode dispatch, solvers and the extern "C" boundary of the
// B200 domain-wall library (declared in include/b200dwf.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/b200dwf.h"
#include "dwf_hop.cuh"
#include "dwf_kernels.h"
#include "learned.h"

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

// Field buffers are read by 16-byte vector loads and bulk (TMA) copies.
bool misaligned(const void* p) { return p && (reinterpret_cast<uintptr_t>(p) & 15u) != 0; }
}  // namespace

namespace b200 {
// Error reporting for the library's other translation units.
void set_last_error(int code, const char* fmt, ...) {
  (void)code;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}
}  // namespace b200

// ------------------------------------------------------------ coefficients
namespace {

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

}  // namespace

// ------------------------------------------------------------ plan
// Per-call device workspace shared by every plan of one device and geometry
// (vh, Ls): the work fields of the operator modes, solvers and forces, and the
// multishift solver's shifted directions and residual window.  At 24^3x48
// Ls=16 a field is 1 GB and a plan touches up to ~40 of them, so the several
// operators of an action set (light, Hasenbusch, strange, Pauli-Villars)
// share one copy instead of holding one each.  Every entry point uses these
// fields only for the duration of one call, so the one rule is: plans of one
// geometry must not run calls concurrently on different streams.
struct Workspace {
  void* work[12][4] = {};       // work fields per slot and storage precision
  void* tune_out[2][4] = {};    // autotuner scratch outputs per precision (trials run inside one call)
  std::vector<void*> p;         // multishift directions p_1..p_(n-1)
  std::vector<void*> win;       // multishift residual window slots
  int users = 0;
};
static std::mutex g_ws_mu;
static std::map<std::tuple<int, int, int>, Workspace*> g_workspaces;

static Workspace* workspace_acquire(int vh, int ls) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_ws_mu);
  Workspace*& ws = g_workspaces[std::make_tuple(dev, vh, ls)];
  if (!ws) ws = new Workspace();
  ++ws->users;
  return ws;
}

static void workspace_release(Workspace* ws) {
  if (!ws) return;
  std::lock_guard<std::mutex> lock(g_ws_mu);
  if (--ws->users > 0) return;
  for (int i = 0; i < 12; ++i)
    for (int p = 0; p < 4; ++p) cudaFree(ws->work[i][p]);
  for (int i = 0; i < 2; ++i)
    for (int p = 0; p < 4; ++p) cudaFree(ws->tune_out[i][p]);
  for (void* q : ws->p) cudaFree(q);
  for (void* q : ws->win) cudaFree(q);
  for (auto it = g_workspaces.begin(); it != g_workspaces.end(); ++it)
    if (it->second == ws) { g_workspaces.erase(it); break; }
  delete ws;
}

// slot i of a workspace vector, allocated on first use
static int ms_pool_slot(std::vector<void*>& v, size_t i, size_t bytes, void** out) {
  std::lock_guard<std::mutex> lock(g_ws_mu);
  if (v.size() <= i) v.resize(i + 1, nullptr);
  if (!v[i] && cudaMalloc(&v[i], bytes) != cudaSuccess) { v[i] = nullptr; return 1; }
  *out = v[i];
  return 0;
}

struct b200_dwf {
  int L[4];
  DwfCoef k;
  int bc[4];
  Geom g;
  void* links[LINK_NFMT] = {};
  double* u_lex = nullptr;      // device copy of the lexical links
  bool have_links = false;
  double* red = nullptr;        // reduction partials
  int* err = nullptr;           // device error word of the bounded waits
  int red_n = 0;
  double* sc = nullptr;         // solver scalars (device)
  double* sc_host = nullptr;    // pinned mirror (also of the multishift scalars)
  int* err_host = nullptr;      // pinned mirror of err
  bool async_calls = false;     // mult / force return without synchronising (b200_dwf_set_async)
  b200_halo_fn halo_fn = nullptr;   // fills (or starts filling) a field's ghost t-slices
  b200_halo_fn halo_finish = nullptr;  // with the split hooks: waits for that filling
  void* halo_ctx = nullptr;
  int inject_dir = -1;          // hop direction whose bulk-copy wait reports failure (-1: none)
  double* stage = nullptr;      // device f64 staging for convert/reverse
  // staging rings of the asynchronous host transfers (upload, download): a
  // slot is reused only after the event of its previous use has fired
  double* ring_buf[2][2] = {};
  cudaEvent_t ring_done[2][2] = {};
  int ring_next[2] = {0, 0};
  Workspace* ws = nullptr;      // shared per-call workspace of this geometry
  void* (*work)[4] = nullptr;   // = ws->work: work fields per slot and precision
  ChainCoefs coefs;             // fifth-dimension chain coefficients
  bool m5pre_id = false;        // D_eo pre-factor is the identity (b = 1, c = 0, alpha = 1)
  double* ms_state = nullptr;   // multishift scalar state (device)
  double* ms_red = nullptr;     // multishift per-shift partials
  void** ms_ptrs = nullptr;     // device arrays of x_i and p_i pointers
  int ms_window = 16;           // multishift residual window (0: per-iteration shift updates)
  bool init_guess = false;      // CG / Richardson start from the x passed in
  void** ms_win_ptrs = nullptr; // device array of the window slots
  std::vector<void*> fcg_buf;   // flexible-CG fields (FP64 ring of directions)
  void* fcg_part = nullptr;     // complex reduction partials
  void* fcg_sc = nullptr;       // complex device scalars
  cudaStream_t gst = nullptr;   // private stream for captured solver iterations
};

namespace {

int ensure_work(b200_dwf* op, int prec, int i) {
  std::lock_guard<std::mutex> lock(g_ws_mu);
  if (!op->work[i][prec]) {
    const size_t bytes = field_bytes(prec, op->g.vh, op->g.ls);
    if (cudaMalloc(&op->work[i][prec], bytes) != cudaSuccess) {
      op->work[i][prec] = nullptr;
      return fail(B200_ENOMEM, "cudaMalloc of %zu bytes for a work field failed", bytes);
    }
  }
  return 0;
}

// link format read by the hop kernels of each storage precision: full 3x3
// records with the boundary phase folded in
int link_format_for(int prec) {
  return prec == PREC_F64 ? LINK_F64_18 : (prec == PREC_F32 ? LINK_F32_18 : LINK_F16_18);
}

int ensure_link_format(b200_dwf* op, int lf, cudaStream_t st) {
  if (!op->have_links) return fail(B200_EINVAL, "set_config has not been called on this operator");
  if (!op->links[lf]) {
    if (cudaMalloc(&op->links[lf], link_bytes(lf, op->g.vh)) != cudaSuccess)
      return fail(B200_ENOMEM, "cudaMalloc for links failed");
    B200_CHECK_CUDA(launch_links_from_lex(lf, op->links[lf], op->u_lex, op->g, op->bc, st));
  }
  return 0;
}

int ensure_links(b200_dwf* op, int prec, cudaStream_t st) {
  return ensure_link_format(op, link_format_for(prec), st);
}

// Suspend-time hint of the TMA hop kernels' barrier waits (B200_WAIT_NS,
// default 0: plain tries).
unsigned int wait_hint_ns() {
  static const unsigned int v = [] {
    const char* e = getenv("B200_WAIT_NS");
    return (e && e[0]) ? (unsigned int)strtoul(e, nullptr, 10) : 0u;
  }();
  return v;
}

HopParams hop_base(const b200_dwf* op, int prec, int ieo, int epi, int fk = F_NONE) {
  HopParams p;
  memset(&p, 0, sizeof(p));
  p.epi = epi;
  p.fk = fk;
  p.links = op->links[link_format_for(prec)];
  p.vh = op->g.vh; p.nx2 = op->g.nx2; p.ny = op->g.ny; p.nz = op->g.nz; p.nt = op->g.nt;
  p.ls = op->g.ls;
  p.site0 = 0;
  p.site_end = op->g.vh;
  p.ieo = ieo;
  p.ce = 1.0;
  p.err = op->err;
  p.fail_dir = op->inject_dir;
  p.wait_ns = wait_hint_ns();
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

// ------------------------------------------------------------ autotuner
// The hop kernel comes in occupancy variants (register budget per thread).
// On the first launch of a (geometry, precision, epilogue) combination the
// variants are timed with CUDA events on the caller's stream, writing to
// scratch outputs, and the fastest is kept for the rest of the process.
// B200_AUTOTUNE=0 disables tuning (variant 0).  The first call of a
// combination must not be inside a CUDA graph capture.
typedef std::tuple<int, int, int, int, int> TuneKey;   // vh, ls, prec, epi, fk
constexpr int kHopVariants = 10;   // direct, TMA 2-stage, TMA 3-stage, TMA 2-stage + direct at
                                  // higher occupancy, packed two-slice FP32x2 (direct, TMA),
                                  // 4-deep TMA, packed with all directions in flight, packed
                                  // half-storage with register prefetch

bool variant_supported(int prec, int ls, int v) {
  if (v < 5) return true;
  if (v == 7 && prec == PREC_F64) return true;
  if (v == 9 && (prec == PREC_F64 || prec == PREC_F32)) return false;
  // 8 stages of 16 sites x (f32 column + 80-byte link record) per warp would
  // need 232 KB of shared memory per block, above the 227 KB limit
  if (v == 8 && ls == 4 && prec == PREC_F32) return false;
  // packed two-slice kernels: every supported Ls (all even); Ls/2 lanes per
  // site, 32/(Ls/2) sites per warp, the remaining lanes idle (Ls 6, 12)
  return prec != PREC_F64;
}
std::map<TuneKey, std::pair<int, float> > g_tune;
std::mutex g_tune_mu;

bool tuning_enabled() {
  const char* e = getenv("B200_AUTOTUNE");
  return !(e && e[0] == '0');
}

int tune_hop(b200_dwf* op, int prec, const HopParams& p0, cudaStream_t st, int* best) {
  {
    // scratch outputs shared by the plans of this geometry
    std::lock_guard<std::mutex> lock(g_ws_mu);
    for (int i = 0; i < 2; ++i)
      if (!op->ws->tune_out[i][prec]) {
        const size_t bytes = field_bytes(prec, op->g.vh, op->g.ls);
        if (cudaMalloc(&op->ws->tune_out[i][prec], bytes) != cudaSuccess) {
          op->ws->tune_out[i][prec] = nullptr;
          return fail(B200_ENOMEM, "cudaMalloc for autotuner scratch failed");
        }
      }
  }
  HopParams p = p0;
  p.fail_dir = -1;   // the trials time real launches
  if (p.out1) p.out1 = op->ws->tune_out[0][prec];
  if (p.out2) p.out2 = op->ws->tune_out[1][prec];
  // The SM clock moves with the power cap while the trials run, so the
  // variants are timed in turn, round after round, and each keeps its
  // fastest round: a clock change then touches every variant alike instead
  // of whichever was timed during it.
  constexpr int kRounds = 3, kReps = 2;
  int vs[kHopVariants];
  float t[kHopVariants];
  int nv = 0;
  for (int v = 0; v < kHopVariants; ++v)
    if (variant_supported(prec, op->g.ls, v)) { vs[nv] = v; t[nv] = 1e30f; ++nv; }
  for (int i = 0; i < nv; ++i) {     // first launches: module loads, first touches
    p.variant = vs[i];
    B200_CHECK_CUDA(launch_hop(prec, p, op->coefs, st));
  }
  cudaEvent_t a, b;
  B200_CHECK_CUDA(cudaEventCreate(&a));
  B200_CHECK_CUDA(cudaEventCreate(&b));
  for (int r = 0; r < kRounds; ++r) {
    for (int i = 0; i < nv; ++i) {
      p.variant = vs[i];
      B200_CHECK_CUDA(cudaEventRecord(a, st));
      for (int k = 0; k < kReps; ++k) B200_CHECK_CUDA(launch_hop(prec, p, op->coefs, st));
      B200_CHECK_CUDA(cudaEventRecord(b, st));
      B200_CHECK_CUDA(cudaEventSynchronize(b));
      float ms = 0.f;
      B200_CHECK_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (ms < t[i]) t[i] = ms;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  float best_ms = 1e30f;
  *best = 0;
  for (int i = 0; i < nv; ++i)
    if (t[i] < best_ms) { best_ms = t[i]; *best = vs[i]; }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[TuneKey(op->g.vh, op->g.ls, prec, p0.epi, p0.fk)] = std::make_pair(*best, best_ms / kReps);
  return 0;
}

// B200_HOP_VARIANT=<n> pins the hop variant (no tuning), e.g. to test each.
int forced_variant() {
  const char* e = getenv("B200_HOP_VARIANT");
  if (!e || !e[0]) return -1;
  const int v = atoi(e);
  return (v >= 0 && v < kHopVariants) ? v : -1;
}

// A rank's share of a lattice split along t is run as its own periodic
// lattice with two ghost t-slices after its interior (the next rank's first
// slice, then the previous rank's last); a stencil reads the previous rank's
// slice through the t wrap.  Before a kernel reads a field at neighbouring
// sites, the host's exchange hook fills that field's ghost slices.
static int halo_call(b200_dwf* op, b200_halo_fn fn, const void* f, int prec, cudaStream_t st) {
  if (!fn || !f) return 0;
  const int rc = fn(op->halo_ctx, const_cast<void*>(f), prec, (void*)st);
  if (rc) return fail(B200_EINVAL, "the halo exchange hook failed (%d)", rc);
  return 0;
}

// the whole exchange: start, and finish where the hooks are split
static int halo(b200_dwf* op, const void* f, int prec, cudaStream_t st) {
  const int rc = halo_call(op, op->halo_fn, f, prec, st);
  return rc ? rc : halo_call(op, op->halo_finish, f, prec, st);
}

static int no_halo(const b200_dwf* op, const char* what) {
  if (!op->halo_fn) return 0;
  return fail(B200_EINVAL,
              "%s: not available on a plan with a halo exchange hook (its reductions would "
              "cover only this rank's extended lattice)",
              what);
}

// The hop variant for p (pinned, tuned earlier, or tuned now on p's sites).
static int select_variant(b200_dwf* op, int prec, HopParams& p, cudaStream_t st) {
  int variant = 0;
  const int fv = forced_variant();
  if (fv >= 0 && variant_supported(prec, op->g.ls, fv)) {
    variant = fv;
  } else if (tuning_enabled()) {
    const TuneKey key(op->g.vh, op->g.ls, prec, p.epi, p.fk);
    bool found = false;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) { variant = it->second.first; found = true; }
    }
    if (!found) {
      int rc = tune_hop(op, prec, p, st, &variant);
      if (rc) return rc;
    }
  }
  p.variant = variant;
  return 0;
}

int run_hop(b200_dwf* op, int prec, HopParams& p, cudaStream_t st) {
  int rc;
  if (op->halo_fn && !p.red) {
    // The two ghost t-slices come last and their outputs are not meaningful:
    // a launch that writes no block partials skips them.  With split hooks
    // the sites whose t neighbours are this rank's own (t = 1 .. nt-2) run
    // while the edge slices travel, the two edge slices after.
    const int slice = op->g.nx2 * op->g.ny * op->g.nz;
    const int nt = op->g.nt - 2;
    if (op->halo_finish) {
      if ((rc = halo_call(op, op->halo_fn, p.in, prec, st))) return rc;
      HopParams pi = p;
      pi.site0 = slice;
      pi.site_end = (nt - 1) * slice;
      const bool interior = pi.site_end > pi.site0;
      if (interior) {
        if ((rc = select_variant(op, prec, pi, st))) return rc;
        B200_CHECK_CUDA(launch_hop(prec, pi, op->coefs, st));
      }
      if ((rc = halo_call(op, op->halo_finish, p.in, prec, st))) return rc;
      HopParams pb = p;
      pb.site0 = 0;
      pb.site_end = slice;
      if (interior) pb.variant = pi.variant;
      else if ((rc = select_variant(op, prec, pb, st))) return rc;
      B200_CHECK_CUDA(launch_hop(prec, pb, op->coefs, st));
      pb.site0 = (nt - 1) * slice;
      pb.site_end = nt * slice;
      B200_CHECK_CUDA(launch_hop(prec, pb, op->coefs, st));
      p.variant = pb.variant;
      return 0;
    }
    if ((rc = halo(op, p.in, prec, st))) return rc;
    p.site_end = nt * slice;
  } else if (op->halo_fn) {
    if ((rc = halo(op, p.in, prec, st))) return rc;
  }
  if ((rc = select_variant(op, prec, p, st))) return rc;
  B200_CHECK_CUDA(launch_hop(prec, p, op->coefs, st));
  return 0;
}

int run_sop(b200_dwf* op, int prec, SopParams& p, cudaStream_t st) {
  B200_CHECK_CUDA(launch_sop(prec, p, op->coefs, st));
  return 0;
}

// v = A(w) with a site-local fifth-dimension map A (SopKind)
int apply_sop(b200_dwf* op, int prec, void* v, const void* w, int opa, cudaStream_t st) {
  SopParams p = sop_base(op);
  p.in = w; p.out1 = v; p.opa = opa;
  return run_sop(op, prec, p, st);
}

// D = 1 - M_ee^-1 D_eo M_oo^-1 D_oe on w; v = w - ...;  optional F(v) -> v2,
// optional |v|^2 partials.  With F the first output may be skipped (v = null).
int apply_D(b200_dwf* op, int prec, void* v, const void* w, int fk, void* v2, double* red,
            cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 0)) || (rc = ensure_work(op, prec, 1))) return rc;
  void* t0 = op->work[0][prec];
  void* y1 = op->work[1][prec];
  if (!op->m5pre_id && (rc = apply_sop(op, prec, t0, w, SOP_M5PRE, st))) return rc;
  HopParams p1 = hop_base(op, prec, 1, EPI_K1);
  p1.in = op->m5pre_id ? w : t0; p1.out1 = y1;
  if ((rc = run_hop(op, prec, p1, st))) return rc;
  HopParams p2 = hop_base(op, prec, 0, EPI_K2N, fk);
  p2.in = y1; p2.out1 = v;
  p2.x1 = w; p2.c_x1 = 1.0;
  p2.out2 = v2;
  p2.red = red;
  return run_hop(op, prec, p2, st);
}

// Ddag = 1 - D_eo^+ M_oo^-+ D_oe^+ M_ee^-+ on u = LUdag(x);  v = xw - ...
int apply_Ddag_from_u(b200_dwf* op, int prec, void* v, const void* xw, const void* u,
                      cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 3))) return rc;
  void* t3 = op->work[3][prec];
  HopParams p3 = hop_base(op, prec, 1, EPI_K3);
  p3.in = u; p3.out1 = t3;
  if ((rc = run_hop(op, prec, p3, st))) return rc;
  HopParams p4 = hop_base(op, prec, 0, EPI_K4N);
  p4.in = t3; p4.out1 = v;
  p4.x1 = xw; p4.c_x1 = 1.0;
  return run_hop(op, prec, p4, st);
}

int apply_Ddag(b200_dwf* op, int prec, void* v, const void* w, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 2))) return rc;
  void* u = op->work[2][prec];
  if ((rc = apply_sop(op, prec, u, w, SOP_LUDAG, st))) return rc;
  return apply_Ddag_from_u(op, prec, v, w, u, st);
}

int apply_DdagD(b200_dwf* op, int prec, void* v, const void* w, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 2)) || (rc = ensure_work(op, prec, 4))) return rc;
  void* t2 = op->work[4][prec];
  void* u = op->work[2][prec];
  if ((rc = apply_D(op, prec, t2, w, F_LUDAG, u, nullptr, st))) return rc;
  return apply_Ddag_from_u(op, prec, v, t2, u, st);
}

int apply_Hdag(b200_dwf* op, int prec, void* v, const void* w, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 2)) || (rc = ensure_work(op, prec, 4))) return rc;
  void* gw = op->work[4][prec];
  void* u = op->work[2][prec];
  SopParams p = sop_base(op);
  p.in = w; p.out1 = gw; p.opa = SOP_G5R; p.opb = SOP_LUDAG; p.out2 = u;
  if ((rc = run_sop(op, prec, p, st))) return rc;
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
      HopParams p = hop_base(op, prec, out_par, EPI_DDAGEO);
      p.in = w; p.out1 = v;
      return run_hop(op, prec, p, st);
    }
    HopParams p = hop_base(op, prec, out_par, EPI_HALF);
    p.in = w; p.out1 = v;
    if (!op->m5pre_id || v == w) {
      if ((rc = ensure_work(op, prec, 0))) return rc;
      void* t0 = op->work[0][prec];
      if ((rc = apply_sop(op, prec, t0, w, SOP_M5PRE, st))) return rc;
      p.in = t0;
    }
    return run_hop(op, prec, p, st);
  }
  if (mode == "Dee" || mode == "Doo") return apply_sop(op, prec, v, w, dag ? SOP_DEE_T : SOP_DEE, st);
  if (mode == "Dee_inv" || mode == "Doo_inv") return apply_sop(op, prec, v, w, dag ? SOP_LUDAG : SOP_LU, st);
  if (mode == "gm5R") return apply_sop(op, prec, v, w, SOP_G5R, st);
  if (mode == "R") return apply_sop(op, prec, v, w, SOP_R, st);
  if (mode == "D") return apply_D(op, prec, v, w, F_NONE, nullptr, nullptr, st);
  if (mode == "H") return apply_D(op, prec, nullptr, w, F_G5R, v, nullptr, st);
  if (mode == "Ddag") return apply_Ddag(op, prec, v, w, st);
  if (mode == "Hdag") return apply_Hdag(op, prec, v, w, st);
  if (mode == "DdagD") return apply_DdagD(op, prec, v, w, st);
  return fail(B200_EINVAL, "mode undefined in AFopr_Domainwall_5din_eo (B200): %s", mode_in.c_str());
}

int reduce_to(b200_dwf* op, int nblocks, double* out_dev, int fin_op, cudaStream_t st) {
  B200_CHECK_CUDA(launch_finalize(op->red, nblocks, out_dev, fin_op, st));
  return 0;
}

// The device error word of the bounded bulk-copy waits, after the stream has
// been synchronised with err_host's copy in it: report a set word as
// B200_ECUDA and clear it, so that the next call starts clean.  The hop that
// gave up returned without writing its outputs.
int report_err(b200_dwf* op, cudaStream_t st) {
  const int code = *op->err_host;
  if (code == 0) return 0;
  *op->err_host = 0;
  B200_CHECK_CUDA(cudaMemsetAsync(op->err, 0, sizeof(int), st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  return fail(B200_ECUDA,
              "a kernel gave up waiting for its bulk copies or tensor-core work "
              "(device error word %d); its outputs were not written",
              code);
}

// Synchronises the stream, then reads, reports and clears the error word.
int check_err(b200_dwf* op, cudaStream_t st) {
  B200_CHECK_CUDA(cudaMemcpyAsync(op->err_host, op->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  return report_err(op, st);
}

// The end of a call that launched hops: synchronous plans (the reference's
// behaviour, the default) wait for the work and report the error word; plans
// switched to asynchronous calls leave that to the next synchronising call.
int finish_call(b200_dwf* op, int rc, cudaStream_t st) {
  if (rc || op->async_calls) return rc;
  return check_err(op, st);
}

// Reads one solver scalar (and the device error word) back to the host.
int host_scalar(b200_dwf* op, int idx, double* out, cudaStream_t st) {
  B200_CHECK_CUDA(cudaMemcpyAsync(op->sc_host + idx, op->sc + idx, sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaMemcpyAsync(op->err_host, op->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  int rc = report_err(op, st);
  if (rc) return rc;
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
  // Shamir kernel at alpha = 1: M5pre = b_s Wf + c_s(...) is the identity, so
  // the pre-factor pass before each D_eo hop (and the M5pre p field of the
  // solvers) is skipped and the hop reads its input directly.
  op->m5pre_id = (alpha == 1.0);
  for (int s = 0; s < Ls; ++s)
    if (op->k.b[s] != 1.0 || op->k.c[s] != 0.0) op->m5pre_id = false;
  const long vol = (long)lattice[0] * lattice[1] * lattice[2] * lattice[3];
  op->g.nx2 = lattice[0] / 2; op->g.ny = lattice[1]; op->g.nz = lattice[2]; op->g.nt = lattice[3];
  op->g.ls = Ls; op->g.vh = (int)(vol / 2);
  op->ws = workspace_acquire(op->g.vh, Ls);
  op->work = op->ws->work;

  // fifth-dimension chain coefficients (both arithmetic types)
  {
    const DwfCoef& kk = op->k;
    ChainCoef<double>& cd = op->coefs.d;
    memset(&cd, 0, sizeof(cd));
    for (int s = 0; s < Ls; ++s) {
      cd.wb[s] = kk.b[s];
      cd.wc2[s] = 2.0 * kk.c[s];
      cd.dm[s] = kk.dm[s];
      cd.dpinv[s] = 1.0 / kk.dp[s];
      cd.e[s] = kk.e[s];
      cd.f[s] = kk.f[s];
      cd.rl[s] = (s >= 1) ? kk.dm[s] / kk.dp[s - 1] : 0.0;
      cd.rld[s] = (s <= Ls - 2) ? kk.dm[s + 1] / kk.dp[s] : 0.0;
    }
    cd.alpha = kk.alpha;
    cd.half_alpha = 0.5 * kk.alpha;
    cd.mhalf_mq = -0.5 * kk.mq;
    cd.dpg_inv = 1.0 / (kk.dp[Ls - 1] + kk.g);
    ChainCoef<float>& cf = op->coefs.f;
    for (int s = 0; s < kMaxLs; ++s) {
      cf.wb[s] = (float)cd.wb[s]; cf.wc2[s] = (float)cd.wc2[s]; cf.rl[s] = (float)cd.rl[s];
      cf.rld[s] = (float)cd.rld[s]; cf.dm[s] = (float)cd.dm[s]; cf.dpinv[s] = (float)cd.dpinv[s];
      cf.e[s] = (float)cd.e[s]; cf.f[s] = (float)cd.f[s];
    }
    cf.alpha = (float)cd.alpha; cf.half_alpha = (float)cd.half_alpha;
    cf.mhalf_mq = (float)cd.mhalf_mq; cf.dpg_inv = (float)cd.dpg_inv;
    // D_ee is the M5-type map with b -> b(4-M0)+1, c -> c(4-M0)-1
    // (reference src/lib_alt_Accel/BridgeOpenACC/src/mult_Domainwall_5din_eo_openacc-inc.h:14-119)
    op->coefs.dee_d = cd;
    for (int s = 0; s < Ls; ++s) {
      op->coefs.dee_d.wb[s] = kk.b[s] * (4.0 - kk.M0) + 1.0;
      op->coefs.dee_d.wc2[s] = 2.0 * (kk.c[s] * (4.0 - kk.M0) - 1.0);
    }
    op->coefs.dee_f = cf;
    for (int s = 0; s < kMaxLs; ++s) {
      op->coefs.dee_f.wb[s] = (float)op->coefs.dee_d.wb[s];
      op->coefs.dee_f.wc2[s] = (float)op->coefs.dee_d.wc2[s];
    }
  }
  const int red_n = site_s_grid(Ls, op->g.vh) + hop_grid(Ls, op->g.vh);
  op->red_n = red_n;
  if (cudaMalloc(&op->red, (size_t)red_n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&op->sc, SC_N * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&op->err, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&op->err_host, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&op->sc_host, (SC_N > MS_N ? SC_N : MS_N) * sizeof(double)) != cudaSuccess) {
    b200_dwf_destroy(op);
    return fail(B200_ENOMEM, "device allocation for the operator plan failed");
  }
  if (cudaMemset(op->err, 0, sizeof(int)) != cudaSuccess) {
    b200_dwf_destroy(op);
    return fail(B200_ECUDA, "clearing the device error word failed");
  }
  *out = op;
  return 0;
}

int b200_dwf_destroy(b200_dwf_t* op) {
  if (!op) return 0;
  for (int i = 0; i < LINK_NFMT; ++i) cudaFree(op->links[i]);
  cudaFree(op->u_lex);
  cudaFree(op->red);
  cudaFree(op->sc);
  cudaFree(op->err);
  if (op->sc_host) cudaFreeHost(op->sc_host);
  if (op->err_host) cudaFreeHost(op->err_host);
  cudaFree(op->stage);
  for (int d = 0; d < 2; ++d)
    for (int k = 0; k < 2; ++k) {
      cudaFree(op->ring_buf[d][k]);
      if (op->ring_done[d][k]) cudaEventDestroy(op->ring_done[d][k]);
    }
  cudaFree(op->ms_state);
  cudaFree(op->ms_red);
  cudaFree(op->ms_ptrs);
  workspace_release(op->ws);
  cudaFree(op->ms_win_ptrs);
  for (void* q : op->fcg_buf) cudaFree(q);
  cudaFree(op->fcg_part);
  cudaFree(op->fcg_sc);
  if (op->gst) cudaStreamDestroy(op->gst);
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
  for (int lf = 0; lf < LINK_NFMT; ++lf)
    if (op->links[lf]) B200_CHECK_CUDA(launch_links_from_lex(lf, op->links[lf], op->u_lex, op->g, op->bc, st));
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

// A staging slot of ring dir (0 upload, 1 download) for `st`: allocated on
// first use; later uses wait on the device for the slot's previous use.
static int ring_slot(b200_dwf_t* op, int dir, cudaStream_t st, int* slot) {
  const int k = op->ring_next[dir];
  op->ring_next[dir] = (k + 1) % 2;
  if (!op->ring_buf[dir][k]) {
    const size_t bytes = b200_dwf_field_nreal(op) * sizeof(double);
    if (cudaMalloc(&op->ring_buf[dir][k], bytes) != cudaSuccess) {
      op->ring_buf[dir][k] = nullptr;
      return fail(B200_ENOMEM, "cudaMalloc of %zu bytes for a transfer staging field failed", bytes);
    }
    B200_CHECK_CUDA(cudaEventCreateWithFlags(&op->ring_done[dir][k], cudaEventDisableTiming));
  } else {
    B200_CHECK_CUDA(cudaStreamWaitEvent(st, op->ring_done[dir][k], 0));
  }
  *slot = k;
  return 0;
}

static bool page_locked(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int b200_field_convert_async(b200_dwf_t* op, int prec, void* v, const double* w_host, void* stream) {
  if (!op || !v || !w_host || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  if (!page_locked(w_host))
    return fail(B200_EINVAL, "convert_async: the host field must be page-locked (cudaHostAlloc / cudaHostRegister)");
  cudaStream_t st = (cudaStream_t)stream;
  int k = 0, rc = ring_slot(op, 0, st, &k);
  if (rc) return rc;
  const size_t bytes = b200_dwf_field_nreal(op) * sizeof(double);
  B200_CHECK_CUDA(cudaMemcpyAsync(op->ring_buf[0][k], w_host, bytes, cudaMemcpyHostToDevice, st));
  B200_CHECK_CUDA(launch_from_corelib(prec, v, op->ring_buf[0][k], op->g, st));
  B200_CHECK_CUDA(cudaEventRecord(op->ring_done[0][k], st));
  return 0;
}

int b200_field_reverse_async(b200_dwf_t* op, int prec, double* v_host, const void* w, void* stream) {
  if (!op || !v_host || !w || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  if (!page_locked(v_host))
    return fail(B200_EINVAL, "reverse_async: the host field must be page-locked (cudaHostAlloc / cudaHostRegister)");
  cudaStream_t st = (cudaStream_t)stream;
  int k = 0, rc = ring_slot(op, 1, st, &k);
  if (rc) return rc;
  const size_t bytes = b200_dwf_field_nreal(op) * sizeof(double);
  B200_CHECK_CUDA(launch_to_corelib(prec, op->ring_buf[1][k], w, op->g, st));
  B200_CHECK_CUDA(cudaMemcpyAsync(v_host, op->ring_buf[1][k], bytes, cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaEventRecord(op->ring_done[1][k], st));
  return 0;
}

int b200_field_convert_lex_device(b200_dwf_t* op, int prec, void* v, const double* w_lex_dev, int ieo,
                                  void* stream) {
  if (!op || !v || !w_lex_dev || prec < 0 || prec > 3 || (ieo != 0 && ieo != 1))
    return fail(B200_EINVAL, "invalid argument");
  B200_CHECK_CUDA(launch_from_lex_parity(prec, v, w_lex_dev, ieo, op->g, (cudaStream_t)stream));
  return 0;
}

int b200_field_convert_device(b200_dwf_t* op, int prec, void* v, const double* w_dev, void* stream) {
  if (!op || !v || !w_dev || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  B200_CHECK_CUDA(launch_from_corelib(prec, v, w_dev, op->g, (cudaStream_t)stream));
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
  // the field read back may come from asynchronous hop calls on this plan:
  // their error word is reported here
  B200_CHECK_CUDA(cudaMemcpyAsync(op->err_host, op->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  B200_CHECK_CUDA(cudaStreamSynchronize(st));
  return report_err(op, st);
}

int b200_dwf_mult(b200_dwf_t* op, int prec, void* v, const void* w, const char* mode, int dag,
                  void* stream) {
  if (!op || !v || !w || !mode || prec < 0 || prec > 3) return fail(B200_EINVAL, "invalid argument");
  if (v == w) return fail(B200_EINVAL, "mult: input and output fields must differ");
  if (misaligned(v) || misaligned(w)) return fail(B200_EINVAL, "mult: field pointers must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  return finish_call(op, apply_mode(op, prec, v, w, mode, dag, st), st);
}

int b200_dwf_set_halo_exchange(b200_dwf_t* op, b200_halo_fn fn, void* ctx) {
  if (!op) return fail(B200_EINVAL, "null argument");
  op->halo_fn = fn;
  op->halo_finish = nullptr;
  op->halo_ctx = fn ? ctx : nullptr;
  return 0;
}

int b200_dwf_set_halo_exchange_split(b200_dwf_t* op, b200_halo_fn start, b200_halo_fn finish,
                                     void* ctx) {
  if (!op || (!start) != (!finish)) return fail(B200_EINVAL, "start and finish go together");
  if (start && op->g.nt < 4) return fail(B200_EINVAL, "a rank needs at least 2 t slices of its own");
  op->halo_fn = start;
  op->halo_finish = finish;
  op->halo_ctx = start ? ctx : nullptr;
  return 0;
}

int b200_dwf_set_async(b200_dwf_t* op, int async_calls) {
  if (!op) return fail(B200_EINVAL, "null operator");
  op->async_calls = async_calls != 0;
  return 0;
}

int b200_dwf_check_error(b200_dwf_t* op, void* stream) {
  if (!op) return fail(B200_EINVAL, "null operator");
  return check_err(op, (cudaStream_t)stream);
}

int b200_dwf_inject_wait_failure(b200_dwf_t* op, int direction) {
  if (!op) return fail(B200_EINVAL, "null operator");
  if (direction < -1 || direction > 7) return fail(B200_EINVAL, "hop direction %d not in -1..7", direction);
  op->inject_dir = direction;
  return 0;
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
// Scalars stay on the device; the host reads |r|^2 once per iteration for the
// stopping test.  Returns the iteration count in *nconv and |r|^2/|b|^2 of the
// recursive residual in *rel2.
struct CgSnap {
  int n;                 // number of snapshots
  const int* iters;      // iteration after which x is copied
  void* const* dst;      // destination fields (precision of the solve)
};

static int cg_core(b200_dwf_t* op, int prec, void* x, const void* b, int maxiter, double tol2,
                   int* nconv, double* rel2, cudaStream_t st, const CgSnap* snap = nullptr) {
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
  const Geom& g = op->g;
  const int nb_hop = hop_grid(g.ls, g.vh);

  B200_CHECK_CUDA(launch_axpby(prec, g, r, b, 1.0, nullptr, 0.0, nullptr, st));
  B200_CHECK_CUDA(launch_axpby(prec, g, p, b, 1.0, nullptr, 0.0, nullptr, st));
  B200_CHECK_CUDA(launch_axpby(prec, g, x, nullptr, 0.0, nullptr, 0.0, nullptr, st));
  if ((rc = field_norm2_dev(op, prec, r, op->sc + SC_RR, st))) return rc;
  double bnorm2 = 0.0;
  if ((rc = host_scalar(op, SC_RR, &bnorm2, st))) return rc;
  *nconv = 0;
  *rel2 = 0.0;
  if (!(bnorm2 > 0.0)) return 0;
  if (op->m5pre_id) yp = p;
  else if ((rc = apply_sop(op, prec, yp, p, SOP_M5PRE, st))) return rc;

  double rr = bnorm2;
  for (int it = 0; it < maxiter; ++it) {
    HopParams p1 = hop_base(op, prec, 1, EPI_K1);
    p1.in = yp; p1.out1 = y1;
    if ((rc = run_hop(op, prec, p1, st))) return rc;

    HopParams p2 = hop_base(op, prec, 0, EPI_K2N, F_LUDAG);
    p2.in = y1; p2.out1 = t2;
    p2.x1 = p; p2.c_x1 = 1.0;
    p2.out2 = u;
    p2.red = op->red;
    if ((rc = run_hop(op, prec, p2, st))) return rc;
    if ((rc = reduce_to(op, nb_hop, op->sc, FIN_CG_ALPHA, st))) return rc;

    HopParams p3 = hop_base(op, prec, 1, EPI_K3);
    p3.in = u; p3.out1 = t3;
    if ((rc = run_hop(op, prec, p3, st))) return rc;

    HopParams p4 = hop_base(op, prec, 0, EPI_K4N);
    p4.in = t3; p4.out1 = r;
    p4.ce = -1.0; p4.ce_dev = op->sc + SC_ALPHA;
    p4.x1 = r; p4.c_x1 = 1.0;
    p4.x2 = t2; p4.c_x2 = -1.0; p4.c_x2_dev = op->sc + SC_ALPHA;
    p4.red = op->red;
    if ((rc = run_hop(op, prec, p4, st))) return rc;
    if ((rc = reduce_to(op, nb_hop, op->sc, FIN_CG_BETA, st))) return rc;

    CgUpdParams pu;
    pu.x = x; pu.p = p; pu.r = r; pu.y = op->m5pre_id ? nullptr : yp;
    pu.alpha = op->sc + SC_ALPHA; pu.beta = op->sc + SC_BETA; pu.g = g;
    B200_CHECK_CUDA(launch_cg_update(prec, pu, op->coefs, st));
    if (snap)
      for (int j = 0; j < snap->n; ++j)
        if (snap->iters[j] == it + 1)
          B200_CHECK_CUDA(cudaMemcpyAsync(snap->dst[j], x, field_bytes(prec, g.vh, g.ls),
                                          cudaMemcpyDeviceToDevice, st));

    if ((rc = host_scalar(op, SC_RR, &rr, st))) return rc;
    *nconv = it + 1;
    if (!(rr == rr)) return fail(B200_ENOCONV, "CG breakdown: residual is NaN at iteration %d", it + 1);
    if (rr / bnorm2 < tol2) break;
  }
  *rel2 = rr / bnorm2;
  if (!(rr / bnorm2 < tol2))
    return fail(B200_ENOCONV, "CG not converged in %d iterations: |r|^2/|b|^2 = %.3e", maxiter,
                rr / bnorm2);
  return 0;
}

// sqrt(|DdagD x + sigma x - b|^2 / |b|^2) in precision prec
static int true_residual(b200_dwf_t* op, int prec, const void* x, const void* b, double sigma,
                         double* out, cudaStream_t st) {
  int rc;
  if ((rc = ensure_work(op, prec, 7))) return rc;
  void* s = op->work[7][prec];
  if ((rc = apply_DdagD(op, prec, s, x, st))) return rc;
  if (sigma != 0.0) B200_CHECK_CUDA(launch_axpby(prec, op->g, s, x, sigma, nullptr, 1.0, nullptr, st));
  B200_CHECK_CUDA(launch_axpby(prec, op->g, s, b, -1.0, nullptr, 1.0, nullptr, st));
  if ((rc = field_norm2_dev(op, prec, s, op->sc + SC_RR_NEW, st))) return rc;
  double d2 = 0.0, b2 = 0.0;
  if ((rc = host_scalar(op, SC_RR_NEW, &d2, st))) return rc;
  if ((rc = field_norm2_dev(op, prec, b, op->sc + SC_RR_NEW, st))) return rc;
  if ((rc = host_scalar(op, SC_RR_NEW, &b2, st))) return rc;
  *out = b2 > 0.0 ? std::sqrt(d2 / b2) : 0.0;
  return 0;
}

int b200_cg_solve(b200_dwf_t* op, int prec, void* x, const void* b, int maxiter, double tol2,
                  int* nconv, double* diff, void* stream) {
  if (!op || !x || !b || prec < 0 || prec > 3 || maxiter < 0) return fail(B200_EINVAL, "invalid argument");
  if (misaligned(x) || misaligned(b)) return fail(B200_EINVAL, "field pointers must be 16-byte aligned");
  if (no_halo(op, "CG")) return B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  int n = 0;
  double rel2 = 0.0;
  int rc;
  if (op->init_guess) {
    // use_initial_guess: CG on the residual equation DdagD e = b - DdagD x
    // from e = 0, stopped at the same |b - DdagD x|^2 / |b|^2, then x += e
    if ((rc = ensure_work(op, prec, 8)) || (rc = ensure_work(op, prec, 9))) return rc;
    void* r0 = op->work[8][prec];
    void* e = op->work[9][prec];
    double bn2 = 0.0, rn2 = 0.0;
    if ((rc = field_norm2_dev(op, prec, b, op->sc + SC_RR_NEW, st)) ||
        (rc = host_scalar(op, SC_RR_NEW, &bn2, st)))
      return rc;
    if ((rc = apply_DdagD(op, prec, r0, x, st))) return rc;
    B200_CHECK_CUDA(launch_axpby(prec, op->g, r0, b, 1.0, nullptr, -1.0, nullptr, st));
    if ((rc = field_norm2_dev(op, prec, r0, op->sc + SC_RR_NEW, st)) ||
        (rc = host_scalar(op, SC_RR_NEW, &rn2, st)))
      return rc;
    rc = 0;
    if (rn2 > tol2 * bn2) {
      rc = cg_core(op, prec, e, r0, maxiter, tol2 * bn2 / rn2, &n, &rel2, st);
      if (rc && rc != B200_ENOCONV) return rc;
      B200_CHECK_CUDA(launch_axpby(prec, op->g, x, e, 1.0, nullptr, 1.0, nullptr, st));
    }
  } else {
    rc = cg_core(op, prec, x, b, maxiter, tol2, &n, &rel2, st);
  }
  if (rc && rc != B200_ENOCONV) return rc;
  const std::string msg = g_err;
  double d = 0.0;
  const int rc2 = true_residual(op, prec, x, b, 0.0, &d, st);
  if (rc2) return rc2;
  if (nconv) *nconv = n;
  if (diff) *diff = d;
  if (rc) g_err = msg;
  return rc;
}

// AShiftsolver_CG (src/lib/Solver/ashiftsolver_CG-tmpl.h:89-329) on
// DdagD + sigma_i, FP64.  One iteration = the four fused DdagD hops, the base
// system's update and three single-block scalar steps.  The shifted systems
// are updated either every iteration (window 0: one fused pass over every
// active x_i, p_i) or, by default, once per window of m iterations from the
// stored residuals and device-side coefficient recurrences (the same
// recurrences regrouped; |p_i|^2 for the pruning test follows from
// |p_i|^2 = zeta_i^2 |r|^2 + alpha_i^2 |p_i|^2 since r is orthogonal to the
// earlier directions).  The iterations replay as captured CUDA graphs and the
// device decides when the solve is over.
int b200_shiftcg_solve(b200_dwf_t* op, void* const* x, const double* sigma, int nshift,
                       const void* b, int maxiter, double tol2, int* nconv, double* diff,
                       void* stream) {
  const int prec = PREC_F64;
  if (!op || !x || !sigma || !b || nshift < 1 || maxiter < 0)
    return fail(B200_EINVAL, "invalid argument");
  if (nshift > kMaxShift) return fail(B200_EINVAL, "at most %d shifts (got %d)", kMaxShift, nshift);
  if (no_halo(op, "multishift CG")) return B200_EINVAL;
  for (int i = 0; i < nshift; ++i)
    if (!x[i] || misaligned(x[i])) return fail(B200_EINVAL, "solution field %d null or not 16-byte aligned", i);
  if (misaligned(b)) return fail(B200_EINVAL, "field pointers must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if ((rc = ensure_links(op, prec, st))) return rc;
  for (int i = 0; i < 8; ++i)
    if ((rc = ensure_work(op, prec, i))) return rc;
  const Geom& g = op->g;
  const int nb_hop = hop_grid(g.ls, g.vh);
  if (!op->ms_state && cudaMalloc(&op->ms_state, kMsStateSize * sizeof(double)) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for multishift state failed");
  if (!op->ms_red && cudaMalloc(&op->ms_red, (size_t)kMaxShift * nb_hop * sizeof(double)) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for multishift partials failed");
  if (!op->ms_ptrs && cudaMalloc(&op->ms_ptrs, 2 * kMaxShift * sizeof(void*)) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for multishift pointers failed");
  // search directions p_i: p_0 is a work slot, the others come from the
  // multishift pool shared by every plan of this field size
  const size_t fbytes = field_bytes(prec, g.vh, g.ls);
  std::vector<void*> ps(nshift);
  for (int i = 0; i < nshift; ++i) {
    if (i == 0) { ps[0] = op->work[6][prec]; continue; }
    if (ms_pool_slot(op->ws->p, i - 1, fbytes, &ps[i]))
      return fail(B200_ENOMEM, "cudaMalloc for multishift direction %d failed", i);
  }
  // windowed mode: m residual slots (allocated on first use); from m = 8 on,
  // x_0 is deferred to the flush as well (one more field, p_0 at the window's
  // start: 2 field passes less per iteration against 5 more per window)
  const int window = op->ms_window;
  void* p0s = nullptr;
  if (window > 0) {
    if (!op->ms_win_ptrs && cudaMalloc(&op->ms_win_ptrs, kMaxWin * sizeof(void*)) != cudaSuccess)
      return fail(B200_ENOMEM, "cudaMalloc for multishift window pointers failed");
    std::vector<void*> wp(kMaxWin, nullptr);
    for (int l = 0; l < window; ++l)
      if (ms_pool_slot(op->ws->win, l, fbytes, &wp[l]))
        return fail(B200_ENOMEM, "cudaMalloc for multishift window slot %d failed", l);
    B200_CHECK_CUDA(cudaMemcpyAsync(op->ms_win_ptrs, wp.data(), kMaxWin * sizeof(void*),
                                    cudaMemcpyHostToDevice, st));
    if (window >= 8 && ms_pool_slot(op->ws->win, kMaxWin, fbytes, &p0s))
      return fail(B200_ENOMEM, "cudaMalloc for the multishift p_0 copy failed");
  }
  void* y0 = op->work[0][prec];
  void* y1 = op->work[1][prec];
  void* u = op->work[2][prec];
  void* t3 = op->work[3][prec];
  void* t2 = op->work[4][prec];
  void* r = op->work[5][prec];
  void* p0 = ps[0];

  // init: p_i = b, x_i = 0, r = b, rr = |b|^2 (ashiftsolver_CG-tmpl.h:188-211)
  for (int i = 0; i < nshift; ++i) {
    B200_CHECK_CUDA(launch_axpby(prec, g, ps[i], b, 1.0, nullptr, 0.0, nullptr, st));
    B200_CHECK_CUDA(launch_axpby(prec, g, x[i], nullptr, 0.0, nullptr, 0.0, nullptr, st));
  }
  B200_CHECK_CUDA(launch_axpby(prec, g, r, b, 1.0, nullptr, 0.0, nullptr, st));
  if (p0s) B200_CHECK_CUDA(launch_axpby(prec, g, p0s, b, 1.0, nullptr, 0.0, nullptr, st));
  if ((rc = field_norm2_dev(op, prec, r, op->sc + SC_RR, st))) return rc;
  double bnorm2 = 0.0;
  if ((rc = host_scalar(op, SC_RR, &bnorm2, st))) return rc;
  if (!(bnorm2 > 0.0)) {
    if (nconv) *nconv = 0;
    if (diff) *diff = 0.0;
    return 0;
  }
  std::vector<double> h(kMsStateSize, 0.0);
  h[MS_RR] = bnorm2;
  h[MS_ALPHA_P] = 0.0;
  h[MS_BETA_P] = 1.0;
  h[MS_PP0] = bnorm2;
  h[MS_SNORM] = 1.0 / bnorm2;
  h[MS_SIGMA0] = sigma[0];
  h[MS_TOL2] = tol2;
  h[MS_NACT] = nshift;
  h[MS_DONE] = 0.0;
  h[MS_ITER] = 0.0;
  h[MS_MAXITER] = (double)maxiter;
  h[MS_WIN] = 0.0;
  h[MS_NACTW] = nshift;
  h[MS_WSIZE] = window;
  for (int i = 0; i < kMaxShift; ++i) {
    h[kMsCoef + i * (kMaxWin + 1)] = 1.0;
    h[MS_N + MSA_PP * kMaxShift + i] = 1.0;     // |p_i|^2 / |b|^2 with p_i = b
  }
  for (int i = 0; i < nshift; ++i) {
    h[MS_N + MSA_ZETA1 * kMaxShift + i] = 1.0;
    h[MS_N + MSA_ZETA2 * kMaxShift + i] = 1.0;
    h[MS_N + MSA_CSH2 * kMaxShift + i] = sigma[i] - sigma[0];
  }
  std::vector<void*> hp(2 * kMaxShift, nullptr);
  for (int i = 0; i < nshift; ++i) { hp[i] = x[i]; hp[kMaxShift + i] = ps[i]; }
  B200_CHECK_CUDA(cudaMemcpyAsync(op->ms_state, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  B200_CHECK_CUDA(cudaMemcpyAsync(op->ms_ptrs, hp.data(), hp.size() * sizeof(void*), cudaMemcpyHostToDevice, st));
  if (op->m5pre_id) y0 = p0;
  else if ((rc = apply_sop(op, prec, y0, p0, SOP_M5PRE, st))) return rc;
  double* S = op->ms_state;

  // One iteration: the four fused DdagD hops, the scalar steps and the fused
  // update of every active shift.  Every kernel skips itself once S[MS_DONE]
  // is set, so iterations can be replayed past convergence as no-ops.
  auto iteration = [&](cudaStream_t s) -> int {
    int rc2;
    HopParams p1 = hop_base(op, prec, 1, EPI_K1);
    p1.in = y0; p1.out1 = y1; p1.skip = S + MS_DONE;
    if ((rc2 = run_hop(op, prec, p1, s))) return rc2;
    HopParams p2 = hop_base(op, prec, 0, EPI_K2N, F_LUDAG);
    p2.in = y1; p2.out1 = t2; p2.x1 = p0; p2.c_x1 = 1.0; p2.out2 = u; p2.red = op->red;
    p2.skip = S + MS_DONE;
    if ((rc2 = run_hop(op, prec, p2, s))) return rc2;
    B200_CHECK_CUDA(launch_ms_scalar(MSS_BETA, op->red, nb_hop, S, nshift, s));
    HopParams p3 = hop_base(op, prec, 1, EPI_K3);
    p3.in = u; p3.out1 = t3; p3.skip = S + MS_DONE;
    if ((rc2 = run_hop(op, prec, p3, s))) return rc2;
    // r += beta (DdagD p0 + sigma0 p0) = r + beta t2 + beta sigma0 p0 + beta K4N(hop)
    HopParams p4 = hop_base(op, prec, 0, EPI_K4N);
    p4.in = t3; p4.out1 = r;
    p4.ce = 1.0; p4.ce_dev = S + MS_BETA;
    p4.x1 = r; p4.c_x1 = 1.0;
    p4.x2 = t2; p4.c_x2 = 1.0; p4.c_x2_dev = S + MS_BETA;
    p4.x3 = p0; p4.c_x3 = sigma[0]; p4.c_x3_dev = S + MS_BETA;
    p4.red = op->red; p4.skip = S + MS_DONE;
    if ((rc2 = run_hop(op, prec, p4, s))) return rc2;
    B200_CHECK_CUDA(launch_ms_scalar(MSS_ALPHA, op->red, nb_hop, S, nshift, s));
    MsUpdParams mu;
    mu.xs = op->ms_ptrs; mu.ps = op->ms_ptrs + kMaxShift; mu.r = r; mu.y0 = op->m5pre_id ? nullptr : y0;
    mu.st = S; mu.red = op->ms_red; mu.nblocks = nb_hop; mu.g = g;
    mu.win = window > 0 ? op->ms_win_ptrs : nullptr;
    mu.p0s = p0s;
    B200_CHECK_CUDA(launch_ms_update(prec, mu, op->coefs, s));
    B200_CHECK_CUDA(launch_ms_scalar(MSS_PRUNE, op->ms_red, nb_hop, S, nshift, s));
    if (window > 0) {
      B200_CHECK_CUDA(launch_ms_flush(mu, s));
      B200_CHECK_CUDA(launch_ms_window_reset(S, s));
    }
    return 0;
  };
  // host view of S[MS_RR .. MS_MAXITER]
  auto read_state = [&](cudaStream_t s, double* done, double* iters, double* rr_out) -> int {
    B200_CHECK_CUDA(cudaMemcpyAsync(op->sc_host, S, (MS_MAXITER + 1) * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
    B200_CHECK_CUDA(cudaMemcpyAsync(op->err_host, op->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    B200_CHECK_CUDA(cudaStreamSynchronize(s));
    int rc_err = report_err(op, s);
    if (rc_err) return rc_err;
    *done = op->sc_host[MS_DONE];
    *iters = op->sc_host[MS_ITER];
    *rr_out = op->sc_host[MS_RR];
    return 0;
  };

  double done = 0.0, iters = 0.0, rr = bnorm2;
  if (maxiter > 0) {
    // the first iteration runs on the caller's stream (it may autotune the
    // four hop epilogues); the rest replay a captured CUDA graph of kBatch
    // iterations on a private stream, checking the device's stop flag after
    // each replay
    if ((rc = iteration(st))) return rc;
    if ((rc = read_state(st, &done, &iters, &rr))) return rc;
    if (done == 0.0) {
      constexpr int kBatch = 16;
      if (!op->gst && cudaStreamCreateWithFlags(&op->gst, cudaStreamNonBlocking) != cudaSuccess)
        return fail(B200_ECUDA, "cudaStreamCreate failed");
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      B200_CHECK_CUDA(cudaStreamBeginCapture(op->gst, cudaStreamCaptureModeThreadLocal));
      int rc_cap = 0;
      for (int b2 = 0; b2 < kBatch && !rc_cap; ++b2) rc_cap = iteration(op->gst);
      const cudaError_t ec = cudaStreamEndCapture(op->gst, &graph);
      if (rc_cap) { if (graph) cudaGraphDestroy(graph); return rc_cap; }
      B200_CHECK_CUDA(ec);
      const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      B200_CHECK_CUDA(ei);
      while (done == 0.0) {
        const cudaError_t el = cudaGraphLaunch(exec, op->gst);
        if (el != cudaSuccess) { cudaGraphExecDestroy(exec); B200_CHECK_CUDA(el); }
        if ((rc = read_state(op->gst, &done, &iters, &rr))) { cudaGraphExecDestroy(exec); return rc; }
      }
      cudaGraphExecDestroy(exec);
    }
    if (done == 2.0)
      return fail(B200_ENOCONV, "multishift CG breakdown: NaN at iteration %d", (int)iters);
  }
  const int it_conv = (done == 1.0) ? (int)iters : -1;
  double dmax = 0.0;
  for (int i = 0; i < nshift; ++i) {
    double d = 0.0;
    if ((rc = true_residual(op, prec, x[i], b, sigma[i], &d, st))) return rc;
    if (d > dmax) dmax = d;
  }
  if (diff) *diff = dmax;
  if (nconv) *nconv = it_conv < 0 ? maxiter : it_conv;
  if (it_conv < 0) return fail(B200_ENOCONV, "multishift CG not converged in %d iterations", maxiter);
  return 0;
}

int b200_solver_set_initial_guess(b200_dwf_t* op, int use) {
  if (!op) return fail(B200_EINVAL, "invalid argument");
  op->init_guess = use != 0;
  return 0;
}

int b200_shiftcg_set_window(b200_dwf_t* op, int window) {
  if (!op || window < 0 || window > kMaxWin)
    return fail(B200_EINVAL, "window must be in [0, %d]", kMaxWin);
  op->ms_window = window;
  return 0;
}

// ASolver_Richardson (src/lib_alt/Solver/asolver_Richardson-tmpl.h:131-213)
// with APrecond_Mixedprec (aprecond_Mixedprec-tmpl.h:55-108): FP64 residual
// and update, inner CG on DdagD in precision inner_prec (fp32 arithmetic over
// f32/f16/bf16 storage) started from zero on the normalised residual.
int b200_richardson_solve(b200_dwf_t* op, int inner_prec, void* x, const void* b, int maxiter,
                          double tol2, int maxiter_inner, double tol2_inner, int* nconv,
                          int* nconv_inner, double* diff, void* stream) {
  if (!op || !x || !b || inner_prec < 0 || inner_prec > 3 || maxiter < 0 || maxiter_inner < 1)
    return fail(B200_EINVAL, "invalid argument");
  if (no_halo(op, "Richardson")) return B200_EINVAL;
  if (misaligned(x) || misaligned(b)) return fail(B200_EINVAL, "field pointers must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const int P64 = PREC_F64;
  int rc;
  if ((rc = ensure_links(op, P64, st)) || (rc = ensure_links(op, inner_prec, st))) return rc;
  for (int i = 8; i < 12; ++i)
    if ((rc = ensure_work(op, P64, i)) || (rc = ensure_work(op, inner_prec, i))) return rc;
  const Geom& g = op->g;
  void* r = op->work[8][P64];
  void* s = op->work[9][P64];
  void* r_in = op->work[10][inner_prec];
  void* s_in = op->work[11][inner_prec];

  if ((rc = field_norm2_dev(op, P64, b, op->sc + SC_RR_NEW, st))) return rc;
  double bnorm2 = 0.0;
  if ((rc = host_scalar(op, SC_RR_NEW, &bnorm2, st))) return rc;
  if (!op->init_guess) B200_CHECK_CUDA(launch_axpby(P64, g, x, nullptr, 0.0, nullptr, 0.0, nullptr, st));
  int total_inner = 0;
  if (!(bnorm2 > 0.0)) {
    B200_CHECK_CUDA(launch_axpby(P64, g, x, nullptr, 0.0, nullptr, 0.0, nullptr, st));
    if (nconv) *nconv = 0;
    if (nconv_inner) *nconv_inner = 0;
    if (diff) *diff = 0.0;
    return 0;
  }
  double r2 = bnorm2;
  if (op->init_guess) {
    // use_initial_guess: start from the residual of the x passed in
    if ((rc = apply_DdagD(op, P64, r, x, st))) return rc;
    B200_CHECK_CUDA(launch_axpby(P64, g, r, b, -1.0, nullptr, 1.0, nullptr, st));
    if ((rc = field_norm2_dev(op, P64, r, op->sc + SC_RR_NEW, st))) return rc;
    if ((rc = host_scalar(op, SC_RR_NEW, &r2, st))) return rc;
  } else {
    B200_CHECK_CUDA(launch_axpby(P64, g, r, b, -1.0, nullptr, 0.0, nullptr, st));
  }
  int conv = -1;
  for (int it = 0; it < maxiter; ++it) {
    if (r2 < bnorm2 * tol2) { conv = it; break; }
    const double nrm = std::sqrt(r2);
    B200_CHECK_CUDA(launch_convert(inner_prec, r_in, P64, r, g, st));
    B200_CHECK_CUDA(launch_axpby(inner_prec, g, r_in, nullptr, 0.0, nullptr, 1.0 / nrm, nullptr, st));
    int n_in = 0;
    double rel_in = 0.0;
    rc = cg_core(op, inner_prec, s_in, r_in, maxiter_inner, tol2_inner, &n_in, &rel_in, st);
    if (rc && rc != B200_ENOCONV) return rc;
    total_inner += n_in;
    B200_CHECK_CUDA(launch_convert(P64, s, inner_prec, s_in, g, st));
    B200_CHECK_CUDA(launch_axpby(P64, g, x, s, -nrm, nullptr, 1.0, nullptr, st));
    if ((rc = apply_DdagD(op, P64, r, x, st))) return rc;
    B200_CHECK_CUDA(launch_axpby(P64, g, r, b, -1.0, nullptr, 1.0, nullptr, st));
    if ((rc = field_norm2_dev(op, P64, r, op->sc + SC_RR_NEW, st))) return rc;
    if ((rc = host_scalar(op, SC_RR_NEW, &r2, st))) return rc;
    if (!(r2 == r2)) return fail(B200_ENOCONV, "Richardson breakdown: NaN residual at iteration %d", it + 1);
  }
  if (conv < 0 && r2 < bnorm2 * tol2) conv = maxiter;
  if (nconv) *nconv = conv < 0 ? maxiter : conv;
  if (nconv_inner) *nconv_inner = total_inner;
  if (diff) *diff = std::sqrt(r2 / bnorm2);
  if (conv < 0) return fail(B200_ENOCONV, "Richardson not converged in %d iterations: |r|^2/|b|^2 = %.3e",
                            maxiter, r2 / bnorm2);
  return 0;
}

// Plain CG (as b200_cg_solve) that copies x after the listed iterations into
// snapshot fields; the (residual, error) training pairs of the learned
// preconditioner come from these snapshots and the converged solution.
int b200_cg_snapshots(b200_dwf_t* op, int prec, void* x, const void* b, int maxiter, double tol2,
                      int nsnap, const int* iters, void* const* snaps, int* nconv, void* stream) {
  if (!op || !x || !b || prec < 0 || prec > 3 || maxiter < 0 || nsnap < 0 || (nsnap > 0 && (!iters || !snaps)))
    return fail(B200_EINVAL, "invalid argument");
  if (misaligned(x) || misaligned(b)) return fail(B200_EINVAL, "field pointers must be 16-byte aligned");
  for (int j = 0; j < nsnap; ++j)
    if (!snaps[j] || misaligned(snaps[j])) return fail(B200_EINVAL, "snapshot %d is not a valid field", j);
  if (no_halo(op, "CG")) return B200_EINVAL;
  const CgSnap sn = {nsnap, iters, snaps};
  int n = 0;
  double rel2 = 0.0;
  const int rc = cg_core(op, prec, x, b, maxiter, tol2, &n, &rel2, (cudaStream_t)stream, &sn);
  if (nconv) *nconv = n;
  return rc;
}

// Flexible CG on DdagD (Notay's FCG; the pattern of the reference's flexible
// solvers, src/lib_alt/Solver/asolver_FBiCGStab-tmpl.h, with the
// preconditioner slot of APrecond<AFIELD>::mult, src/lib_alt/Solver/
// aprecond.h:28-47) preconditioned by the learned network: FP64 iterate and
// residual, z = N(r) in FP32 with BF16 weights, the new direction
// A-orthogonalised against the last mtrunc directions with complex
// coefficients (N is not Hermitian).  The FP64 true residual judges the
// result; if it misses tol2, plain CG on the residual equation finishes the
// solve from x (its iterations are returned in *nconv_fallback).
int b200_fcg_solve(b200_dwf_t* op, b200_lp_t* lp, void* x, const void* b, int maxiter, double tol2,
                   int mtrunc, int* nconv, int* nconv_fallback, double* diff, void* stream) {
  constexpr int kFallbackMaxiter = 100000;
  if (!op || !lp || !x || !b || maxiter < 0 || mtrunc < 1 || mtrunc > 8)
    return fail(B200_EINVAL, "invalid argument");
  if (no_halo(op, "flexible CG")) return B200_EINVAL;
  if (misaligned(x) || misaligned(b)) return fail(B200_EINVAL, "field pointers must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const int P64 = PREC_F64, P32 = PREC_F32;
  int rc;
  if ((rc = ensure_links(op, P64, st)) || (rc = ensure_links(op, P32, st))) return rc;
  if ((rc = ensure_work(op, P32, 10)) || (rc = ensure_work(op, P32, 11))) return rc;
  const Geom& g = op->g;
  const size_t ncplx = (size_t)g.vh * g.ls * 12;
  const size_t fb = field_bytes(P64, g.vh, g.ls);
  const int M = mtrunc;
  const size_t nbuf = 2 * (size_t)(M + 1) + 3;
  while (op->fcg_buf.size() < nbuf) {
    void* q = nullptr;
    if (cudaMalloc(&q, fb) != cudaSuccess) return fail(B200_ENOMEM, "cudaMalloc for a flexible-CG field failed");
    op->fcg_buf.push_back(q);
  }
  if (!op->fcg_part && cudaMalloc(&op->fcg_part, sizeof(double2) * zblas_blocks() * kZMaxMulti) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for flexible-CG partials failed");
  if (!op->fcg_sc && cudaMalloc(&op->fcg_sc, sizeof(double2) * 32) != cudaSuccess)
    return fail(B200_ENOMEM, "cudaMalloc for flexible-CG scalars failed");
  void** P = op->fcg_buf.data();
  void** Q = op->fcg_buf.data() + (M + 1);
  void* r = op->fcg_buf[2 * (M + 1)];
  void* z = op->fcg_buf[2 * (M + 1) + 1];
  void* dx = op->fcg_buf[2 * (M + 1) + 2];
  void* rf = op->work[10][P32];
  void* zf = op->work[11][P32];
  double2* sc = reinterpret_cast<double2*>(op->fcg_sc);   // [1] alpha, [2+i] <p_i,q_i>, [16+j] betas
  double2* pqw = sc + 24;                                  // <p_j,q_j> of the current window
  double* part = reinterpret_cast<double*>(op->fcg_part);

  auto precondition = [&]() -> int {
    B200_CHECK_CUDA(launch_convert(P32, rf, P64, r, g, st));
    int rc2 = lp_apply_internal(lp, zf, rf, st);
    if (rc2) return rc2;
    B200_CHECK_CUDA(launch_convert(P64, z, P32, zf, g, st));
    return 0;
  };

  if (nconv) *nconv = 0;
  if (nconv_fallback) *nconv_fallback = 0;
  if (diff) *diff = 0.0;
  B200_CHECK_CUDA(launch_axpby(P64, g, x, nullptr, 0.0, nullptr, 0.0, nullptr, st));
  B200_CHECK_CUDA(cudaMemcpyAsync(r, b, fb, cudaMemcpyDeviceToDevice, st));
  if ((rc = field_norm2_dev(op, P64, r, op->sc + SC_RR_NEW, st))) return rc;
  double bb = 0.0;
  if ((rc = host_scalar(op, SC_RR_NEW, &bb, st))) return rc;
  if (!(bb > 0.0)) return 0;
  if ((rc = precondition())) return rc;
  B200_CHECK_CUDA(cudaMemcpyAsync(P[0], z, fb, cudaMemcpyDeviceToDevice, st));
  double rr = bb;
  int iters = 0;
  for (int it = 0; it < maxiter; ++it) {
    const int k = it % (M + 1);
    if ((rc = apply_DdagD(op, P64, Q[k], P[k], st))) return rc;
    B200_CHECK_CUDA(launch_zdot(P[k], Q[k], ncplx, op->fcg_part, sc + 2 + k, nullptr, 1.0, st));
    B200_CHECK_CUDA(launch_zdot(P[k], r, ncplx, op->fcg_part, sc + 1, sc + 2 + k, 1.0, st));
    B200_CHECK_CUDA(launch_zcg_update(x, r, P[k], Q[k], ncplx, sc + 1, part, st));
    B200_CHECK_CUDA(launch_finalize(part, zblas_blocks(), op->sc + SC_RR_NEW, FIN_SUM, st));
    if ((rc = host_scalar(op, SC_RR_NEW, &rr, st))) return rc;
    iters = it + 1;
    if (!(rr == rr)) return fail(B200_ENOCONV, "flexible CG breakdown: NaN residual at iteration %d", iters);
    if (rr / bb < tol2) break;
    if ((rc = precondition())) return rc;
    // p_new = z - sum_j (<q_j, z> / <p_j, q_j>) p_j over the window, as two
    // passes: all dot products at once, then one combined update
    const int kn = (it + 1) % (M + 1);
    const int j0 = (it - M + 1 > 0 ? it - M + 1 : 0);
    ZMulti qv, pv;
    qv.m = pv.m = it - j0 + 1;
    for (int j = j0; j <= it; ++j) {
      const int sj = j % (M + 1);
      qv.v[j - j0] = reinterpret_cast<const double2*>(Q[sj]);
      pv.v[j - j0] = reinterpret_cast<const double2*>(P[sj]);
      B200_CHECK_CUDA(cudaMemcpyAsync(pqw + (j - j0), sc + 2 + sj, sizeof(double2),
                                      cudaMemcpyDeviceToDevice, st));
    }
    B200_CHECK_CUDA(launch_zmdot(qv, z, ncplx, op->fcg_part, sc + 16, pqw, -1.0, st));
    B200_CHECK_CUDA(launch_zmaxpy(P[kn], z, pv, sc + 16, ncplx, st));
  }
  if (nconv) *nconv = iters;
  double d = 0.0;
  if ((rc = true_residual(op, P64, x, b, 0.0, &d, st))) return rc;
  if (!(d * d < tol2)) {
    // r = b - DdagD x, then plain CG on DdagD dx = r to the remaining tolerance
    if ((rc = apply_DdagD(op, P64, r, x, st))) return rc;
    B200_CHECK_CUDA(launch_axpby(P64, g, r, b, 1.0, nullptr, -1.0, nullptr, st));
    const double r2 = d * d * bb;
    int nfb = 0;
    double rel = 0.0;
    rc = cg_core(op, P64, dx, r, kFallbackMaxiter, tol2 * bb / r2, &nfb, &rel, st);
    if (rc && rc != B200_ENOCONV) return rc;
    B200_CHECK_CUDA(launch_axpby(P64, g, x, dx, 1.0, nullptr, 1.0, nullptr, st));
    if (nconv_fallback) *nconv_fallback = nfb;
    if ((rc = true_residual(op, P64, x, b, 0.0, &d, st))) return rc;
  }
  if (diff) *diff = d;
  if (!(d * d < tol2))
    return fail(B200_ENOCONV, "flexible CG and its CG fallback missed the tolerance: |r|/|b| = %.3e", d);
  return 0;
}

// Force_F_Domainwall_eo (src/lib/Force/Fermion/force_F_Domainwall_eo.cpp:
// 150-327) on the device.  With y_e = M5pre(eta), y_o = M5pre M_oo^-1 D_oe eta,
// A_e = M_ee^-+ gm5R zeta and A_o = M_oo^-+ D_oe^+ A_e (both fifth-dimension
// chains fused into the hops), the reference's terms become
//   H    : even  +1/2 sum [(1-g) y_o(x+mu)] conj(A_e) ; odd  [(1-g) y_e(x+mu)] conj(A_o)
//   Hdag : even  +1/2 sum [(1+g) A_o(x+mu)] conj(y_e) ; odd  [(1+g) A_e(x+mu)] conj(y_o)
// (U^+ U = 1 and the dagger's M5^+ moved onto the conjugated field as M5pre).
static int force_fields(b200_dwf_t* op, const void* eta, const void* zeta, bool zeta_is_h_eta,
                        cudaStream_t st) {
  const int prec = PREC_F64;
  int rc;
  if ((rc = ensure_links(op, prec, st))) return rc;
  for (int i = 0; i < 5; ++i)
    if ((rc = ensure_work(op, prec, i))) return rc;
  const void* ye = op->m5pre_id ? eta : op->work[0][prec];
  void* yo = op->work[1][prec];
  void* ae = op->work[2][prec];
  void* ao = op->work[3][prec];
  if (!op->m5pre_id && (rc = apply_sop(op, prec, op->work[0][prec], eta, SOP_M5PRE, st))) return rc;
  HopParams p1 = hop_base(op, prec, 1, EPI_K1);
  p1.in = ye; p1.out1 = yo;
  if ((rc = run_hop(op, prec, p1, st))) return rc;
  if (zeta_is_h_eta) {
    // gm5R (H eta) = D eta, so A_e = LUdag(D eta) comes out of D's second hop
    HopParams p2 = hop_base(op, prec, 0, EPI_K2N, F_LUDAG);
    p2.in = yo; p2.out1 = nullptr; p2.x1 = eta; p2.c_x1 = 1.0; p2.out2 = ae;
    if ((rc = run_hop(op, prec, p2, st))) return rc;
  } else {
    SopParams q = sop_base(op);
    q.in = zeta; q.out1 = op->work[4][prec]; q.opa = SOP_G5R; q.opb = SOP_LUDAG; q.out2 = ae;
    if ((rc = run_sop(op, prec, q, st))) return rc;
  }
  HopParams p3 = hop_base(op, prec, 1, EPI_K3);
  p3.in = ae; p3.out1 = ao;
  return run_hop(op, prec, p3, st);
}

static ForceParams force_base(const b200_dwf_t* op, double* force, int ieo) {
  ForceParams f;
  memset(&f, 0, sizeof(f));
  f.force = force;
  f.coef = 0.5;
  f.beta = 0.0;
  f.ieo = ieo;
  f.vh = op->g.vh; f.nx2 = op->g.nx2; f.ny = op->g.ny; f.nz = op->g.nz; f.nt = op->g.nt;
  f.ls = op->g.ls;
  for (int mu = 0; mu < 4; ++mu) f.bc[mu] = op->bc[mu];
  return f;
}

// force = beta * force + scale * force_udiv1 (mode "H"/"Hdag", reference
// argument order) or force_udiv (mode "DdagD", a = eta, b unused).
static int force_impl(b200_dwf_t* op, const char* mode, double* force, const void* a,
                      const void* b, double scale, double beta, cudaStream_t st) {
  if (!op || !mode || !force || !a) return fail(B200_EINVAL, "invalid argument");
  if (op->k.alpha != 1.0)
    return fail(B200_EINVAL, "force with parameter_alpha != 1 is not available (as in the reference)");
  const std::string m = mode;
  const bool udiv = (m == "DdagD");
  if (!udiv && m != "H" && m != "Hdag")
    return fail(B200_EINVAL, "%s: unknown mode %s", "Force_F_Domainwall_eo", mode);
  if (!udiv && !b) return fail(B200_EINVAL, "invalid argument");
  if (misaligned(a) || (b && misaligned(b)))
    return fail(B200_EINVAL, "field pointers must be 16-byte aligned");
  const bool hdag = (m == "Hdag");
  const void* eta = udiv ? a : (hdag ? a : b);
  const void* zeta = udiv ? nullptr : (hdag ? b : a);
  int rc;
  if ((rc = force_fields(op, eta, zeta, udiv, st))) return rc;
  const void* ye = op->m5pre_id ? eta : op->work[0][PREC_F64];
  void* yo = op->work[1][PREC_F64];
  void* ae = op->work[2][PREC_F64];
  void* ao = op->work[3][PREC_F64];
  ForceParams fe = force_base(op, force, 0), fo = force_base(op, force, 1);
  fe.coef *= scale; fo.coef *= scale;
  fe.beta = beta; fo.beta = beta;
  if (udiv || !hdag) { fe.y1 = yo; fe.z1 = ae; fo.y1 = ye; fo.z1 = ao; }
  if (udiv || hdag) { fe.y2 = ao; fe.z2 = ye; fo.y2 = ae; fo.z2 = yo; }
  const void* read[4] = {ye, yo, ae, ao};
  for (const void* f : read)
    if ((rc = halo(op, f, PREC_F64, st))) return rc;
  B200_CHECK_CUDA(launch_force(fe, st));
  B200_CHECK_CUDA(launch_force(fo, st));
  return 0;
}

int b200_dwf_force_udiv1(b200_dwf_t* op, const char* mode, double* force, const void* a,
                         const void* b, void* stream) {
  if (mode && std::string(mode) == "DdagD")
    return fail(B200_EINVAL, "%s: unknown mode %s", "Force_F_Domainwall_eo", mode);
  if (!b) return fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  return finish_call(op, force_impl(op, mode, force, a, b, 1.0, 0.0, st), st);
}

int b200_dwf_force_udiv(b200_dwf_t* op, double* force, const void* eta, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  return finish_call(op, force_impl(op, "DdagD", force, eta, nullptr, 1.0, 0.0, st), st);
}

int b200_dwf_force_acc(b200_dwf_t* op, const char* mode, double* force, const void* a,
                       const void* b, double scale, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  return finish_call(op, force_impl(op, mode, force, a, b, scale, 1.0, st), st);
}

int b200_tuning_table(char* buf, size_t n) {
  if (!buf || n == 0) return fail(B200_EINVAL, "invalid buffer");
  std::string out;
  static const char* pn[4] = {"f64", "f32", "f16", "bf16"};
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (const auto& kv : g_tune) {
    char line[160];
    snprintf(line, sizeof(line), "vh=%d ls=%d prec=%s epi=%d fk=%d variant=%d us=%.2f\n",
             std::get<0>(kv.first), std::get<1>(kv.first), pn[std::get<2>(kv.first) & 3],
             std::get<3>(kv.first), std::get<4>(kv.first), kv.second.first, kv.second.second * 1e3f);
    out += line;
  }
  snprintf(buf, n, "%s", out.c_str());
  return 0;
}

}  // extern "C"

// Accessors used by the learned preconditioner (learned.cu).
namespace b200 {
int plan_geometry(b200_dwf* op, Geom* g, float bc[4]) {
  *g = op->g;
  for (int mu = 0; mu < 4; ++mu) bc[mu] = (float)op->bc[mu];
  return 0;
}
int plan_apply_ddagd(b200_dwf* op, void* v, const void* w, cudaStream_t st) {
  return apply_mode(op, PREC_F32, v, w, "DdagD", 0, st);
}
int* plan_error_word(b200_dwf* op) { return op->err; }
int plan_check_error(b200_dwf* op, cudaStream_t st) { return check_err(op, st); }
bool plan_has_halo(const b200_dwf* op) { return op->halo_fn != nullptr; }
int plan_links_f32(b200_dwf* op, const void** links, cudaStream_t st) {
  const int rc = ensure_link_format(op, LINK_F32_12, st);
  if (rc) return rc;
  *links = op->links[LINK_F32_12];
  return 0;
}
int plan_links_f32_folded(b200_dwf* op, const void** links, cudaStream_t st) {
  const int rc = ensure_link_format(op, LINK_F32_18, st);
  if (rc) return rc;
  *links = op->links[LINK_F32_18];
  return 0;
}
}  // namespace b200
