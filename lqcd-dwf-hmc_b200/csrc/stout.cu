// Stout link smearing and its force Jacobian on the device (FP64).
//
// Reference: Smear_APE::smear (src/lib/Smear/smear_APE.cpp:108-140),
// Projection_Stout_SU3::project / force_recursive / set_uw / set_fj
// (src/lib/Smear/projection_Stout_SU3.cpp:60-500), ForceSmear_APE::force_udiv /
// force_each / staple (src/lib/Smear/forceSmear_APE.cpp:95-260), driven by
// Director_Smear (src/lib/Smear/director_Smear.cpp) and
// AForce_F_Smeared_alt::mult_jacobian (src/lib_alt/Force/Fermion/
// aforce_F_Smeared_alt-tmpl.h:170-191).  In the reference these run on the
// host (the Accel build copies the links back for force_recursive); here each
// is one kernel over the 4*Nvol links, one thread per (site, mu).
//
// Links and forces use the lexical Field_G(Nvol, 4) layout
// ri + 2*(col + 3*row) + 18*(site + Nvol*mu).
#include <cuda_runtime.h>

#include "../../include/b200dwf.h"
#include "dwf_kernels.h"
#include "su3_lex.cuh"

namespace b200 {


// rho * sum_{nu != mu} (upper + lower) staples of U_mu(x)
__device__ M3 staple_sum(const double* u, const LexGeom& g, size_t site, int mu, double rho) {
  M3 c = zero3();
  const size_t xmu = g.shift(site, mu, 1);
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    const size_t xnu = g.shift(site, nu, 1);
    const size_t xmnu = g.shift(site, nu, -1);
    const size_t xmnu_mu = g.shift(xmnu, mu, 1);
    // U_nu(x) U_mu(x+nu) U_nu(x+mu)^+
    const M3 up = mul_nd(mul_nn(load3(u, site + g.vol * nu), load3(u, xnu + g.vol * mu)),
                         load3(u, xmu + g.vol * nu));
    // U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu)
    const M3 dn = mul_nn(mul_dn(load3(u, xmnu + g.vol * nu), load3(u, xmnu + g.vol * mu)),
                         load3(u, xmnu_mu + g.vol * nu));
    add_to(c, up, rho);
    add_to(c, dn, rho);
  }
  return c;
}

// ---------------------------------------------------------------------------
// exp(iQ) of a traceless Hermitian 3x3 matrix Q by the Cayley-Hamilton
// theorem, after C. Morningstar and M. Peardon, "Analytic smearing of SU(3)
// link variables in lattice QCD", Phys. Rev. D 69, 054501 (2004), sec. III:
//   exp(iQ) = f0 + f1 Q + f2 Q^2,
// the f_j being functions of the two invariants c0 = det Q = tr(Q^3)/3 and
// c1 = tr(Q^2)/2 only (through the eigenvalue parameters u and w).  The stout
// force needs their derivatives, B1 = sum_j (df_j/dc1) Q^j and
// B2 = sum_j (df_j/dc0) Q^j.  The closed forms are evaluated at |c0| (where
// they are best conditioned) and carried to c0 < 0 by the paper's symmetry
// f_j(-c0) = (-1)^j conj f_j(c0), whose derivative gives
// d f_j/dc1 (-c0) = (-1)^j conj(...) and d f_j/dc0 (-c0) = (-1)^(j+1) conj(...).
// ---------------------------------------------------------------------------

// sin(w)/w
__device__ __forceinline__ double sinc_w(double w) { return (w == 0.0) ? 1.0 : sin(w) / w; }

// (cos w - sin(w)/w) / w^2 = d/dw (sin(w)/w) / w.  For small w, where the
// closed form cancels, its Taylor series
//   sum_m (-1)^(m+1) (2m+2) w^(2m) / (2m+3)!
// is summed term by term (each term from the previous one).
__device__ double dsinc_w(double w) {
  if (w >= 0.5) return (cos(w) - sin(w) / w) / (w * w);
  const double w2 = w * w;
  double term = -1.0 / 3.0, sum = 0.0;
  for (int m = 1; m < 12; ++m) {
    sum += term;
    term *= -w2 * (2 * m + 2) / ((double)(2 * m) * (2 * m + 2) * (2 * m + 3));
  }
  return sum + term;
}

struct ExpCoef {
  Cx f[3];     // exp(iQ) = f0 + f1 Q + f2 Q^2
  Cx d1[3];    // d f_j / d c1
  Cx d0[3];    // d f_j / d c0
};

__device__ __forceinline__ Cx expi(double a) { return cx(cos(a), sin(a)); }
__device__ __forceinline__ Cx imul(double s, Cx a) { return cx(-s * a.i, s * a.r); }   // i s a

// kDeriv: also the derivatives (the force's B1, B2)
template <bool kDeriv>
__device__ ExpCoef expi_coef(double c0, double c1) {
  const bool flip = c0 < 0.0;
  const double a0 = fabs(c0);
  const double s3 = sqrt(c1 / 3.0);
  const double theta = acos(fmin(1.0, a0 / (2.0 * s3 * s3 * s3)));
  const double u = s3 * cos(theta / 3.0);
  const double w = sqrt(c1) * sin(theta / 3.0);
  const double uu = u * u, ww = w * w;
  const double sw = sinc_w(w), cw = cos(w);
  const Cx p2 = expi(2.0 * u);      // e^{2iu}
  const Cx m1 = expi(-u);           // e^{-iu}
  const double den = 9.0 * uu - ww;
  ExpCoef r;
  // h_j / (9u^2 - w^2), paper eqs. (30)-(33)
  r.f[0] = (1.0 / den) * ((uu - ww) * p2 + m1 * cx(8.0 * uu * cw, 2.0 * u * (3.0 * uu + ww) * sw));
  r.f[1] = (1.0 / den) * ((2.0 * u) * p2 - m1 * cx(2.0 * u * cw, -(3.0 * uu - ww) * sw));
  r.f[2] = (1.0 / den) * (p2 - m1 * cx(cw, 3.0 * u * sw));
  if (kDeriv) {
    const double ds = dsinc_w(w);
    // the paper's r_j^(1), r_j^(2) (eqs. 58-60), written out per component
    Cx ra[3], rb[3];
    ra[0] = 2.0 * (cx(u, uu - ww) * p2) +
            2.0 * (m1 * cx(8.0 * u * cw + u * (3.0 * uu + ww) * sw,
                           -4.0 * uu * cw + (9.0 * uu + ww) * sw));
    ra[1] = 2.0 * (cx(1.0, 2.0 * u) * p2) +
            m1 * cx(-2.0 * cw + (3.0 * uu - ww) * sw, 2.0 * u * cw + 6.0 * u * sw);
    ra[2] = imul(2.0, p2) + m1 * cx(-3.0 * u * sw, cw - 3.0 * sw);
    rb[0] = -2.0 * p2 + m1 * cx(-8.0 * uu * sw, 2.0 * u * (cw + sw + 3.0 * uu * ds));
    rb[1] = m1 * cx(2.0 * u * sw, -(cw + sw - 3.0 * uu * ds));
    rb[2] = m1 * cx(sw, -3.0 * u * ds);
    const double inv = 1.0 / (2.0 * den * den);
    for (int j = 0; j < 3; ++j) {
      r.d1[j] = inv * ((2.0 * u) * ra[j] + (3.0 * uu - ww) * rb[j] - (30.0 * uu + 2.0 * ww) * r.f[j]);
      r.d0[j] = inv * (ra[j] - (3.0 * u) * rb[j] - (24.0 * u) * r.f[j]);
    }
  }
  if (flip) {
    for (int j = 0; j < 3; ++j) {
      const double sj = (j & 1) ? -1.0 : 1.0;
      r.f[j] = sj * conj(r.f[j]);
      if (kDeriv) {
        r.d1[j] = sj * conj(r.d1[j]);
        r.d0[j] = -sj * conj(r.d0[j]);
      }
    }
  }
  return r;
}

// a0 + a1 Q + a2 Q^2
__device__ __forceinline__ M3 qpoly(const Cx* a, const M3& Q, const M3& Q2) {
  M3 e;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const Cx id = (k % 4 == 0) ? a[0] : cx(0.0, 0.0);
    e.m[k] = id + a[1] * Q.m[k] + a[2] * Q2.m[k];
  }
  return e;
}

// tr(A B)
__device__ __forceinline__ Cx tr_mul(const M3& a, const M3& b) {
  Cx t = cx(0.0, 0.0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) t = t + a.m[3 * i + j] * b.m[3 * j + i];
  return t;
}

// The stout generator of one link: Q = -i TA(C U^+) (Hermitian, traceless),
// its square, and the invariants c0, c1.
struct StoutQ {
  M3 Q, Q2;
  double c0, c1;
};

__device__ __forceinline__ StoutQ stout_q(const M3& C, const M3& U) {
  StoutQ q;
  M3 a = mul_nd(C, U);
  at3(a);                                    // a = i Q
#pragma unroll
  for (int k = 0; k < 9; ++k) q.Q.m[k] = cx(a.m[k].i, -a.m[k].r);
  q.Q2 = mul_nn(q.Q, q.Q);
  q.c1 = 0.5 * (q.Q2.m[0].r + q.Q2.m[4].r + q.Q2.m[8].r);
  q.c0 = tr_mul(q.Q, q.Q2).r / 3.0;
  return q;
}

// The reference treats a link whose generator is negligible as unsmeared:
// exp(iQ) = 1 and no Lambda term in the force, when |iQ|^2 = tr(Q^2) = 2 c1
// is at most 1e-10 (Projection_Stout_SU3::force_recursive / project,
// src/lib/Smear/projection_Stout_SU3.cpp); the same cut keeps results equal
// on (near-)cold links.
__device__ __forceinline__ bool stout_negligible(const StoutQ& q) { return 2.0 * q.c1 <= 1.0e-10; }

struct StoutParams {
  const double* u;     // links of this level (input of the smearing step)
  double* u_out;       // smeared links
  const double* sigp;  // force w.r.t. the smeared links
  double* sig;         // force w.r.t. u (output)
  double* itheta;      // per-link Theta (recursive -> force_each)
  double rho;
  LexGeom g;
};

// U' = exp(iQ) U, one thread per link
__global__ void stout_smear_kernel(StoutParams p) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 4 * p.g.vol) return;
  const int mu = (int)(idx / p.g.vol);
  const size_t site = idx % p.g.vol;
  const M3 U = load3(p.u, idx);
  const StoutQ q = stout_q(staple_sum(p.u, p.g, site, mu, p.rho), U);
  if (stout_negligible(q)) {
    store3(p.u_out, idx, U);
    return;
  }
  const ExpCoef k = expi_coef<false>(q.c0, q.c1);
  store3(p.u_out, idx, mul_nn(qpoly(k.f, q.Q, q.Q2), U));
}

// One backward step of the stout chain for link (x, mu): with M = U Sigma'
//   Gamma  = tr(M B1) Q + tr(M B2) Q^2 + f1 M + f2 (Q M + M Q)
//   iLambda = TA(i Gamma),   iTheta = iLambda U   (kept for force_each)
//   Sigma  = Sigma' exp(iQ) + C^+ iLambda
// (paper eqs. 69-75); the staple derivative terms follow in force_each.
__global__ void stout_recursive_kernel(StoutParams p) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 4 * p.g.vol) return;
  const int mu = (int)(idx / p.g.vol);
  const size_t site = idx % p.g.vol;
  const M3 U = load3(p.u, idx);
  const M3 C = staple_sum(p.u, p.g, site, mu, p.rho);
  const M3 Sp = load3(p.sigp, idx);
  const StoutQ q = stout_q(C, U);
  M3 e, il;
  if (stout_negligible(q)) {
    e = unit3();
    il = zero3();
  } else {
    const ExpCoef k = expi_coef<true>(q.c0, q.c1);
    e = qpoly(k.f, q.Q, q.Q2);
    const M3 M = mul_nn(U, Sp);
    const Cx g1 = tr_mul(M, qpoly(k.d1, q.Q, q.Q2));
    const Cx g0 = tr_mul(M, qpoly(k.d0, q.Q, q.Q2));
    const M3 QM = mul_nn(q.Q, M);
    const M3 MQ = mul_nn(M, q.Q);
#pragma unroll
    for (int n = 0; n < 9; ++n) {
      const Cx gam = g1 * q.Q.m[n] + g0 * q.Q2.m[n] + k.f[1] * M.m[n] + k.f[2] * (QM.m[n] + MQ.m[n]);
      il.m[n] = imul(1.0, gam);
    }
    at3(il);
  }
  store3(p.itheta, idx, mul_nn(il, U));
  M3 sig = mul_nn(Sp, e);
  add_to(sig, mul_dn(C, il));
  store3(p.sig, idx, sig);
}

// ForceSmear_APE::force_each summed over nu != mu, times rho, added to sig
__global__ void stout_force_each_kernel(StoutParams p) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 4 * p.g.vol) return;
  const int mu = (int)(idx / p.g.vol);
  const size_t x = idx % p.g.vol;
  const size_t V = p.g.vol;
  const double* U = p.u;
  const double* T = p.itheta;
  M3 acc = zero3();
  const size_t xmu = p.g.shift(x, mu, 1);
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    const size_t xnu = p.g.shift(x, nu, 1);
    const size_t xmn = p.g.shift(x, nu, -1);          // x - nu
    const size_t xmn_mu = p.g.shift(xmn, mu, 1);      // x - nu + mu
    const M3 Vnu_xmu = load3(U, xmu + V * nu);
    const M3 Vmu_xnu = load3(U, xnu + V * mu);
    const M3 Vnu_x = load3(U, x + V * nu);
    M3 s = zero3();
    // V_nu(x+mu) V_mu(x+nu)^+ iT_nu(x)^+
    add_to(s, mul_nd(mul_nd(Vnu_xmu, Vmu_xnu), load3(T, x + V * nu)));
    // V_nu(x-nu+mu)^+ iT_mu(x-nu)^+ V_nu(x-nu)
    const M3 Vnu_xmnmu = load3(U, xmn_mu + V * nu);
    const M3 Vnu_xmn = load3(U, xmn + V * nu);
    add_to(s, mul_dn(Vnu_xmnmu, mul_dn(load3(T, xmn + V * mu), Vnu_xmn)));
    // V_nu(x-nu+mu)^+ V_mu(x-nu)^+ iT_nu(x-nu)
    const M3 Vmu_xmn = load3(U, xmn + V * mu);
    add_to(s, mul_dn(Vnu_xmnmu, mul_dn(Vmu_xmn, load3(T, xmn + V * nu))));
    // iT_nu(x+mu) V_mu(x+nu)^+ V_nu(x)^+
    add_to(s, mul_nd(mul_nd(load3(T, xmu + V * nu), Vmu_xnu), Vnu_x));
    // iT_nu(x-nu+mu)^+ V_mu(x-nu)^+ V_nu(x-nu)
    add_to(s, mul_nn(mul_dd(load3(T, xmn_mu + V * nu), Vmu_xmn), Vnu_xmn));
    // V_nu(x+mu) iT_mu(x+nu)^+ V_nu(x)^+
    add_to(s, mul_nd(mul_nd(Vnu_xmu, load3(T, xnu + V * mu)), Vnu_x));
    add_to(acc, s, p.rho);
  }
  M3 out = load3(p.sig, idx);
  add_to(out, acc);
  store3(p.sig, idx, out);
}

// AForce_F<ACCEL>::mult_generator (src/lib_alt_Accel/Force/Fermion/aforce_F.cpp:62-75):
// F_mu(x) <- -2 at(U_mu(x) F_mu(x))
__global__ void mult_generator_kernel(double* f, const double* u, size_t nlink) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nlink) return;
  M3 m = mul_nn(load3(u, idx), load3(f, idx));
  at3(m);
#pragma unroll
  for (int k = 0; k < 9; ++k) m.m[k] = -2.0 * m.m[k];
  store3(f, idx, m);
}

}  // namespace b200

// ------------------------------------------------------------ smearing plan
using namespace b200;

struct b200_smear {
  LexGeom g;
  double rho;
  int nsmear;
  double* levels = nullptr;   // (nsmear + 1) configs, level 0 = thin links
  double* itheta = nullptr;
  double* sig_tmp = nullptr;
  bool have_config = false;
};

namespace b200 {
void set_last_error(int code, const char* fmt, ...);
}

#define B200_SMEAR_CHECK(call)                                                      \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      set_last_error(B200_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));          \
      return B200_ECUDA;                                                            \
    }                                                                               \
  } while (0)

static size_t nreal_cfg(const b200_smear* sm) { return 18 * 4 * sm->g.vol; }

extern "C" {

int b200_smear_create(b200_smear_t** out, const int lattice[4], double rho, int nsmear) {
  if (!out || !lattice || nsmear < 0 || nsmear > 16) {
    set_last_error(B200_EINVAL, "smear_create: invalid argument");
    return B200_EINVAL;
  }
  b200_smear* sm = new b200_smear();
  for (int mu = 0; mu < 4; ++mu) {
    if (lattice[mu] < 1) { delete sm; set_last_error(B200_EINVAL, "invalid lattice"); return B200_EINVAL; }
    sm->g.n[mu] = lattice[mu];
  }
  sm->g.vol = (size_t)lattice[0] * lattice[1] * lattice[2] * lattice[3];
  sm->rho = rho;
  sm->nsmear = nsmear;
  const size_t n = nreal_cfg(sm) * sizeof(double);
  if (cudaMalloc(&sm->levels, (nsmear + 1) * n) != cudaSuccess ||
      cudaMalloc(&sm->itheta, n) != cudaSuccess || cudaMalloc(&sm->sig_tmp, n) != cudaSuccess) {
    cudaFree(sm->levels); cudaFree(sm->itheta); cudaFree(sm->sig_tmp);
    delete sm;
    set_last_error(B200_ENOMEM, "smear_create: device allocation failed");
    return B200_ENOMEM;
  }
  *out = sm;
  return 0;
}

int b200_smear_destroy(b200_smear_t* sm) {
  if (!sm) return 0;
  cudaFree(sm->levels);
  cudaFree(sm->itheta);
  cudaFree(sm->sig_tmp);
  delete sm;
  return 0;
}

int b200_smear_set_config(b200_smear_t* sm, const double* u, int on_device, void* stream) {
  if (!sm || !u) { set_last_error(B200_EINVAL, "smear_set_config: invalid argument"); return B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = nreal_cfg(sm);
  B200_SMEAR_CHECK(cudaMemcpyAsync(sm->levels, u, n * sizeof(double),
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  const int grid = (int)((4 * sm->g.vol + 127) / 128);
  for (int i = 0; i < sm->nsmear; ++i) {
    StoutParams p{};
    p.u = sm->levels + i * n;
    p.u_out = sm->levels + (i + 1) * n;
    p.rho = sm->rho;
    p.g = sm->g;
    stout_smear_kernel<<<grid, 128, 0, st>>>(p);
    B200_SMEAR_CHECK(cudaGetLastError());
  }
  B200_SMEAR_CHECK(cudaStreamSynchronize(st));
  sm->have_config = true;
  return 0;
}

const double* b200_smear_config(b200_smear_t* sm, int level) {
  if (!sm || level < 0 || level > sm->nsmear || !sm->have_config) return nullptr;
  return sm->levels + (size_t)level * nreal_cfg(sm);
}

int b200_smear_get_config(b200_smear_t* sm, int level, double* host_out, void* stream) {
  const double* src = b200_smear_config(sm, level);
  if (!src || !host_out) { set_last_error(B200_EINVAL, "smear_get_config: invalid level or no config"); return B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  B200_SMEAR_CHECK(cudaMemcpyAsync(host_out, src, nreal_cfg(sm) * sizeof(double), cudaMemcpyDeviceToHost, st));
  B200_SMEAR_CHECK(cudaStreamSynchronize(st));
  return 0;
}

int b200_smear_jacobian(b200_smear_t* sm, double* sigma, void* stream) {
  if (!sm || !sigma || !sm->have_config) {
    set_last_error(B200_EINVAL, "smear_jacobian: invalid argument or no config");
    return B200_EINVAL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = nreal_cfg(sm);
  const int grid = (int)((4 * sm->g.vol + 127) / 128);
  for (int i = sm->nsmear - 1; i >= 0; --i) {
    // Sigma_i = J_i^T Sigma_(i+1): sig_tmp <- recursion(sigma), then force_each
    B200_SMEAR_CHECK(cudaMemcpyAsync(sm->sig_tmp, sigma, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    StoutParams p{};
    p.u = sm->levels + (size_t)i * n;
    p.sigp = sm->sig_tmp;
    p.sig = sigma;
    p.itheta = sm->itheta;
    p.rho = sm->rho;
    p.g = sm->g;
    stout_recursive_kernel<<<grid, 128, 0, st>>>(p);
    B200_SMEAR_CHECK(cudaGetLastError());
    stout_force_each_kernel<<<grid, 128, 0, st>>>(p);
    B200_SMEAR_CHECK(cudaGetLastError());
  }
  return 0;
}

int b200_force_mult_generator(const int lattice[4], double* force, const double* u, void* stream) {
  if (!lattice || !force || !u) { set_last_error(B200_EINVAL, "mult_generator: invalid argument"); return B200_EINVAL; }
  const size_t nlink = 4 * (size_t)lattice[0] * lattice[1] * lattice[2] * lattice[3];
  mult_generator_kernel<<<(int)((nlink + 127) / 128), 128, 0, (cudaStream_t)stream>>>(force, u, nlink);
  B200_SMEAR_CHECK(cudaGetLastError());
  return 0;
}

}  // extern "C"
