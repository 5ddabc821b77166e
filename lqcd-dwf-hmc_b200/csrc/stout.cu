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

__device__ __forceinline__ double xi0f(double w) { return (w == 0.0) ? 1.0 : sin(w) / w; }
__device__ __forceinline__ double xi1f(double w) {
  if (w < 0.25) {
    const double w2 = w * w;
    const double c0 = -1.0 / 3.0, c1 = 1.0 / 30.0, c2 = -1.0 / 840.0, c3 = 1.0 / 45360.0,
                 c4 = -1.0 / 3991680.0;
    return c0 + w2 * (c1 + w2 * (c2 + w2 * (c3 + w2 * c4)));
  }
  return (w * cos(w) - sin(w)) / (w * w * w);
}

// Cayley-Hamilton coefficients of exp(iQ) (set_uw, set_fj)
__device__ void uw_fj(const M3& iQ2, const M3& iQ3, double& u, double& w, Cx& f0, Cx& f1, Cx& f2) {
  const double c0 = -(iQ3.m[0].i + iQ3.m[4].i + iQ3.m[8].i) / 3.0;
  const double c1 = -0.5 * (iQ2.m[0].r + iQ2.m[4].r + iQ2.m[8].r);
  const double c13r = sqrt(c1 / 3.0);
  const double c0max = 2.0 * c13r * c13r * c13r;
  const double theta = acos(c0 / c0max);
  u = c13r * cos(theta / 3.0);
  w = sqrt(c1) * sin(theta / 3.0);
  const double xi0 = xi0f(w);
  const double u2 = u * u, w2 = w * w, cos_w = cos(w);
  const double cos_u = cos(u), sin_u = sin(u);
  const Cx emiu = cx(cos_u, -sin_u);
  const Cx e2iu = cx(cos_u * cos_u - sin_u * sin_u, 2.0 * sin_u * cos_u);
  const Cx h0 = e2iu * cx(u2 - w2, 0.0) + emiu * cx(8.0 * u2 * cos_w, 2.0 * u * (3.0 * u2 + w2) * xi0);
  const Cx h1 = e2iu * cx(2 * u, 0.0) - emiu * cx(2.0 * u * cos_w, -(3.0 * u2 - w2) * xi0);
  const Cx h2 = e2iu - emiu * cx(cos_w, 3.0 * u * xi0);
  const double fden = 1.0 / (9.0 * u2 - w2);
  f0 = fden * h0;
  f1 = fden * h1;
  f2 = fden * h2;
}

// f0 + f1 Q + f2 Q^2 with Q = -i iQ1 and Q^2 = -iQ2
__device__ __forceinline__ M3 ch_combine(Cx f0, Cx f1, Cx f2, const M3& iQ1, const M3& iQ2) {
  M3 e;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const Cx id = (k == 0 || k == 4 || k == 8) ? cx(1, 0) : cx(0, 0);
    e.m[k] = f0 * id + f1 * cx(iQ1.m[k].i, -iQ1.m[k].r) - f2 * iQ2.m[k];
  }
  return e;
}

struct StoutParams {
  const double* u;     // links of this level (input of the smearing step)
  double* u_out;       // smeared links
  const double* sigp;  // force w.r.t. the smeared links
  double* sig;         // force w.r.t. u (output)
  double* itheta;      // per-link Theta (recursive -> force_each)
  double rho;
  LexGeom g;
};

__global__ void stout_smear_kernel(StoutParams p) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 4 * p.g.vol) return;
  const int mu = (int)(idx / p.g.vol);
  const size_t site = idx % p.g.vol;
  const M3 U = load3(p.u, idx);
  const M3 C = staple_sum(p.u, p.g, site, mu, p.rho);
  M3 iQ1 = mul_nd(C, U);
  at3(iQ1);
  const M3 iQ2 = mul_nn(iQ1, iQ1);
  const M3 iQ3 = mul_nn(iQ1, iQ2);
  M3 e;
  if (norm2_3(iQ1) > 1.0e-10) {
    double u, w;
    Cx f0, f1, f2;
    uw_fj(iQ2, iQ3, u, w, f0, f1, f2);
    e = ch_combine(f0, f1, f2, iQ1, iQ2);
  } else {
    e = unit3();
  }
  store3(p.u_out, idx, mul_nn(e, U));
}

// Projection_Stout_SU3::force_recursive: Xi = Sigma' e^{iQ} + C^+ iGamma, iTheta = iGamma U
__global__ void stout_recursive_kernel(StoutParams p) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 4 * p.g.vol) return;
  const int mu = (int)(idx / p.g.vol);
  const size_t site = idx % p.g.vol;
  const M3 U = load3(p.u, idx);
  const M3 C = staple_sum(p.u, p.g, site, mu, p.rho);
  const M3 Sp = load3(p.sigp, idx);
  M3 iQ1 = mul_nd(C, U);
  at3(iQ1);
  const M3 iQ2 = mul_nn(iQ1, iQ1);
  const M3 iQ3 = mul_nn(iQ1, iQ2);
  M3 e, iG;
  if (norm2_3(iQ1) > 1.0e-10) {
    double u, w;
    Cx f0, f1, f2;
    uw_fj(iQ2, iQ3, u, w, f0, f1, f2);
    e = ch_combine(f0, f1, f2, iQ1, iQ2);
    const double xi0 = xi0f(w), xi1 = xi1f(w);
    const double u2 = u * u, w2 = w * w, cos_w = cos(w);
    const Cx emiu = cx(cos(u), -sin(u));
    const Cx e2iu = cx(cos(2.0 * u), sin(2.0 * u));
    const Cx r01 = cx(2.0 * u, 2.0 * (u2 - w2)) * e2iu +
                   emiu * cx(16.0 * u * cos_w + 2.0 * u * (3.0 * u2 + w2) * xi0,
                             -8.0 * u2 * cos_w + 2.0 * (9.0 * u2 + w2) * xi0);
    const Cx r11 = cx(2.0, 4.0 * u) * e2iu +
                   emiu * cx(-2.0 * cos_w + (3.0 * u2 - w2) * xi0, 2.0 * u * cos_w + 6.0 * u * xi0);
    const Cx r21 = cx(0.0, 2.0) * e2iu + emiu * cx(-3.0 * u * xi0, cos_w - 3.0 * xi0);
    const Cx r02 = cx(-2.0, 0.0) * e2iu +
                   emiu * cx(-8.0 * u2 * xi0, 2.0 * u * (cos_w + xi0 + 3.0 * u2 * xi1));
    const Cx r12 = emiu * cx(2.0 * u * xi0, -cos_w - xi0 + 3.0 * u2 * xi1);
    const Cx r22 = emiu * cx(xi0, -3.0 * u * xi1);
    const double fden = 1.0 / (2 * (9.0 * u2 - w2) * (9.0 * u2 - w2));
    const double c2u = 2.0 * u, c3 = 3.0 * u2 - w2, c30 = 30.0 * u2 + 2.0 * w2;
    const Cx b10 = fden * (c2u * r01 + c3 * r02 - c30 * f0);
    const Cx b11 = fden * (c2u * r11 + c3 * r12 - c30 * f1);
    const Cx b12 = fden * (c2u * r21 + c3 * r22 - c30 * f2);
    const Cx b20 = fden * (r01 - (3.0 * u) * r02 - (24.0 * u) * f0);
    const Cx b21 = fden * (r11 - (3.0 * u) * r12 - (24.0 * u) * f1);
    const Cx b22 = fden * (r21 - (3.0 * u) * r22 - (24.0 * u) * f2);
    const M3 B1 = ch_combine(b10, b11, b12, iQ1, iQ2);
    const M3 B2 = ch_combine(b20, b21, b22, iQ1, iQ2);
    const M3 US = mul_nn(U, Sp);
    const M3 t1 = mul_nn(US, B1);
    const M3 t2 = mul_nn(US, B2);
    const Cx tr1 = t1.m[0] + t1.m[4] + t1.m[8];
    const Cx tr2 = t2.m[0] + t2.m[4] + t2.m[8];
    const M3 iQUS = mul_nn(iQ1, US);
    const M3 iUSQ = mul_nn(US, iQ1);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const Cx qt = tr1 * cx(iQ1.m[k].i, -iQ1.m[k].r) - tr2 * iQ2.m[k] + f1 * US.m[k] +
                    f2 * cx(iQUS.m[k].i, -iQUS.m[k].r) + f2 * cx(iUSQ.m[k].i, -iUSQ.m[k].r);
      iG.m[k] = cx(-qt.i, qt.r);
    }
  } else {
    iG = zero3();
    e = unit3();
  }
  at3(iG);
  store3(p.itheta, idx, mul_nn(iG, U));
  M3 xi = mul_nn(Sp, e);
  add_to(xi, mul_dn(C, iG));
  store3(p.sig, idx, xi);
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
