// Gauge-field side of the HMC step on the device (FP64): the Iwasaki /
// rectangle gauge force and action, the link update exp(alpha iP) U and the
// momentum update and kinetic energy.
//
// Reference (the corelib runs these on the host in every build):
//   Force_G_Rectangle::force_core  src/lib/Force/Gauge/force_G_Rectangle.cpp:84-220
//   Action_G_Rectangle::calcH      src/lib/Action/Gauge/action_G_Rectangle.cpp:97-200
//   Integrator_UpdateU::evolve     src/lib/HMC/integrator_UpdateU.cpp:79-86
//     -> mult_exp_Field_G (src/lib/Field/Imp/field_G_imp.cpp:496-522)
//     -> SU_N::mat_exp + Mat_SU_N::reunit_SU3 (src/lib/Tools/mat_SU_N.h:637-657,
//        src/lib/Tools/mat_SU_N.cpp:18-88)
//   Integrator_UpdateP::evolve     src/lib/HMC/integrator_UpdateP.cpp:44-66
//   HMC_General::calcH_P           src/lib/HMC/hmc_General.cpp:340-346
//
// One thread per link (site, mu) for the force and the update, one per site
// for the action; every staple and rectangle is formed from the links it
// touches (no shifted copies of the field are made).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/b200dwf.h"
#include "dwf_kernels.h"
#include "su3_lex.cuh"

namespace b200 {

void set_last_error(int code, const char* fmt, ...);

namespace {

struct GaugeGeom {
  LexGeom g;
  __device__ M3 U(const double* u, size_t site, int mu) const { return load3(u, site + g.vol * mu); }
  __device__ size_t sh(size_t site, int mu, int d) const { return g.shift(site, mu, d); }
};

// Sum over nu != mu of the staples of U_mu(x) in the rectangle action:
// c_plaq (upper + lower plaquette staples) + c_rect (the six 2x1 rectangles
// through U_mu(x)), each a product S with U_mu(x) S^+ a closed loop at x.
__device__ M3 rect_staples(const double* u, const GaugeGeom& G, size_t x, int mu, double cp, double cr) {
  // links are re-read from global memory (L1/L2 hits) instead of being kept
  // live, which keeps the register footprint of the 3x3 products small
  M3 f = zero3();
  const size_t xpm = G.sh(x, mu, 1);
  const size_t xmm = G.sh(x, mu, -1);
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    const size_t xpn = G.sh(x, nu, 1), xmn = G.sh(x, nu, -1);
    const size_t xpmmn = G.sh(xpm, nu, -1);                    // x+mu-nu
    // upper: U_nu(x) U_mu(x+nu) U_nu(x+mu)^+ ; lower: U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu)
    add_to(f, mul_nd(mul_nn(G.U(u, x, nu), G.U(u, xpn, mu)), G.U(u, xpm, nu)), cp);
    add_to(f, mul_nn(mul_dn(G.U(u, xmn, nu), G.U(u, xmn, mu)), G.U(u, xpmmn, nu)), cp);
    if (cr == 0.0) continue;
    const size_t xpmpn = G.sh(xpm, nu, 1);                     // x+mu+nu
    const size_t xp2m = G.sh(xpm, mu, 1);                      // x+2mu
    const size_t xp2n = G.sh(xpn, nu, 1);                      // x+2nu
    const size_t xm2n = G.sh(xmn, nu, -1);                     // x-2nu
    const size_t xmmpn = G.sh(xmm, nu, 1);                     // x-mu+nu
    const size_t xmmmn = G.sh(xmm, nu, -1);                    // x-mu-nu
    const size_t xp2mmn = G.sh(xp2m, nu, -1);                  // x+2mu-nu
    const size_t xm2npm = G.sh(xm2n, mu, 1);                   // x-2nu+mu
    // R1 = U_nu(x) U_mu(x+nu) U_mu(x+mu+nu) U_nu(x+2mu)^+ U_mu(x+mu)^+
    add_to(f, mul_nd(mul_nd(mul_nn(mul_nn(G.U(u, x, nu), G.U(u, xpn, mu)), G.U(u, xpmpn, mu)),
                            G.U(u, xp2m, nu)), G.U(u, xpm, mu)), cr);
    // R2 = U_nu(x) U_nu(x+nu) U_mu(x+2nu) U_nu(x+mu+nu)^+ U_nu(x+mu)^+
    add_to(f, mul_nd(mul_nd(mul_nn(mul_nn(G.U(u, x, nu), G.U(u, xpn, nu)), G.U(u, xp2n, mu)),
                            G.U(u, xpmpn, nu)), G.U(u, xpm, nu)), cr);
    // R3 = U_mu(x-mu)^+ U_nu(x-mu) U_mu(x-mu+nu) U_mu(x+nu) U_nu(x+mu)^+
    add_to(f, mul_nd(mul_nn(mul_nn(mul_dn(G.U(u, xmm, mu), G.U(u, xmm, nu)), G.U(u, xmmpn, mu)),
                            G.U(u, xpn, mu)), G.U(u, xpm, nu)), cr);
    // R4 = U_nu(x-nu)^+ U_mu(x-nu) U_mu(x-nu+mu) U_nu(x-nu+2mu) U_mu(x+mu)^+
    add_to(f, mul_nd(mul_nn(mul_nn(mul_dn(G.U(u, xmn, nu), G.U(u, xmn, mu)), G.U(u, xpmmn, mu)),
                            G.U(u, xp2mmn, nu)), G.U(u, xpm, mu)), cr);
    // R5 = U_nu(x-nu)^+ U_nu(x-2nu)^+ U_mu(x-2nu) U_nu(x-2nu+mu) U_nu(x-nu+mu)
    add_to(f, mul_nn(mul_nn(mul_nn(mul_dd(G.U(u, xmn, nu), G.U(u, xm2n, nu)), G.U(u, xm2n, mu)),
                            G.U(u, xm2npm, nu)), G.U(u, xpmmn, nu)), cr);
    // R6 = U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_mu(x-nu) U_nu(x-nu+mu)
    add_to(f, mul_nn(mul_nn(mul_nn(mul_dd(G.U(u, xmm, mu), G.U(u, xmmmn, nu)), G.U(u, xmmmn, mu)),
                            G.U(u, xmn, mu)), G.U(u, xpmmn, nu)), cr);
  }
  return f;
}

__global__ void gauge_force_kernel(const double* u, double* force, LexGeom g, double beta, double cp,
                                   double cr) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= 4 * g.vol) return;
  const int mu = (int)(idx / g.vol);
  const size_t x = idx - (size_t)mu * g.vol;
  GaugeGeom G{g};
  const M3 f = rect_staples(u, G, x, mu, cp, cr);
  M3 w = mul_nd(G.U(u, x, mu), f);
  at3(w);
  M3 out = zero3();
  add_to(out, w, -beta / 3.0);
  store3(force, idx, out);
}

__device__ __forceinline__ double retr_nd(const M3& a, const M3& b) {   // Re tr(a b^+)
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) t += a.m[k].r * b.m[k].r + a.m[k].i * b.m[k].i;
  return t;
}

// per-block partial sums of the plaquette and rectangle traces of calcH
__global__ void gauge_action_kernel(const double* u, LexGeom g, double* partial) {
  __shared__ double sp[256], sr[256];
  const size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  double pl = 0.0, re = 0.0;
  if (x < g.vol) {
    GaugeGeom G{g};
    for (int mu = 0; mu < 4; ++mu) {
      const M3 umu = G.U(u, x, mu);
      const size_t xpm = G.sh(x, mu, 1);
      for (int nu = mu + 1; nu < 4; ++nu) {
        const size_t xpn = G.sh(x, nu, 1);
        pl += retr_nd(umu, mul_nd(mul_nn(G.U(u, x, nu), G.U(u, xpn, mu)), G.U(u, xpm, nu)));
        const size_t xpmpn = G.sh(xpm, nu, 1);
        re += retr_nd(umu, mul_nd(mul_nd(mul_nn(mul_nn(G.U(u, x, nu), G.U(u, xpn, mu)), G.U(u, xpmpn, mu)),
                                         G.U(u, G.sh(xpm, mu, 1), nu)), G.U(u, xpm, mu)));
        re += retr_nd(umu, mul_nd(mul_nd(mul_nn(mul_nn(G.U(u, x, nu), G.U(u, xpn, nu)),
                                                G.U(u, G.sh(xpn, nu, 1), mu)), G.U(u, xpmpn, nu)),
                                  G.U(u, xpm, nu)));
      }
    }
  }
  sp[threadIdx.x] = pl;
  sr[threadIdx.x] = re;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sp[threadIdx.x] += sp[threadIdx.x + o]; sr[threadIdx.x] += sr[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = sp[0]; partial[2 * blockIdx.x + 1] = sr[0]; }
}

// Back onto SU(3) after the link update, as Mat_SU_N::reunit_SU3 does
// (src/lib/Tools/mat_SU_N.cpp:18-88): Gram-Schmidt on the first two rows,
// then the third row completes a unit-determinant matrix.  With rows a, b:
//   a <- a / |a|;   b <- b - <a, b> a,  b <- b / |b|;   c = conj(a x b).
__device__ void reunit3(M3& m) {
  Cx* a = m.m;
  Cx* b = m.m + 3;
  Cx* c = m.m + 6;
  const double ia = 1.0 / sqrt(a[0].r * a[0].r + a[0].i * a[0].i + a[1].r * a[1].r + a[1].i * a[1].i +
                               a[2].r * a[2].r + a[2].i * a[2].i);
#pragma unroll
  for (int j = 0; j < 3; ++j) a[j] = ia * a[j];
  const Cx ab = conj(a[0]) * b[0] + conj(a[1]) * b[1] + conj(a[2]) * b[2];   // <a, b>
#pragma unroll
  for (int j = 0; j < 3; ++j) b[j] = b[j] - ab * a[j];
  const double ib = 1.0 / sqrt(b[0].r * b[0].r + b[0].i * b[0].i + b[1].r * b[1].r + b[1].i * b[1].i +
                               b[2].r * b[2].r + b[2].i * b[2].i);
#pragma unroll
  for (int j = 0; j < 3; ++j) b[j] = ib * b[j];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int k = (j + 1) % 3, l = (j + 2) % 3;
    c[j] = conj(a[k] * b[l] - a[l] * b[k]);
  }
}

// u <- reunit( (u + a iP (u + a/2 iP ( ... (u + a/n iP u) ...))) ), n = nprec
__global__ void link_update_kernel(double* u, const double* ip, size_t nlink, double alpha, int nprec) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= nlink) return;
  const M3 u0 = load3(u, idx);
  const M3 iv = load3(ip, idx);
  M3 t = u0;
  for (int k = 0; k < nprec; ++k) {
    const double f = alpha / (double)(nprec - k);
    M3 p = mul_nn(iv, t);
    t = u0;
    add_to(t, p, f);
  }
  reunit3(t);
  store3(u, idx, t);
}

__global__ void axpy_links_kernel(double* y, const double* x, size_t n, double a) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

// y = a x + b y over link fields (b = 0: y = a x, y not read)
__global__ void axpby_links_kernel(double* y, const double* x, size_t n, double a, double b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = (b == 0.0) ? a * x[i] : fma(a, x[i], b * y[i]);
}

// iP = i sum_a h_a lambda_a on every link (Langevin_Momentum::set_iP_SU3,
// src/lib/HMC/langevin_Momentum.cpp:150-210) from h = Field(8, Nvol, 4) of
// Gaussians, written into the Field_G layout entry by entry: the Gell-Mann
// matrices lambda_1..8 have at most two non-zero entries per position, and
// lambda_8's 1/sqrt(3) is passed in (s).  Diagonal: i (h_3 +- s h_8) and
// -2 i s h_8; off-diagonal (r, c) / (c, r): i h for the symmetric lambdas,
// +-h for the antisymmetric ones.
__global__ void momentum_from_gauss_kernel(const double* h, double* ip, size_t nlink, double s) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= nlink) return;
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = h[8 * idx + k];
  double* o = ip + 18 * idx;
  const double d8 = __dmul_rn(s, a[7]);
  o[0] = 0.0;    o[1] = __dadd_rn(a[2], d8);               // (0,0)
  o[2] = a[1];   o[3] = a[0];                               // (0,1)
  o[4] = a[4];   o[5] = a[3];                               // (0,2)
  o[6] = -a[1];  o[7] = a[0];                               // (1,0)
  o[8] = 0.0;    o[9] = __dadd_rn(-a[2], d8);              // (1,1)
  o[10] = a[6];  o[11] = a[5];                              // (1,2)
  o[12] = -a[4]; o[13] = a[3];                              // (2,0)
  o[14] = -a[6]; o[15] = a[5];                              // (2,1)
  o[16] = 0.0;   o[17] = __dmul_rn(-2.0 * s, a[7]);        // (2,2)
}

__global__ void norm2_links_kernel(const double* x, size_t n, double* partial) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc = fma(x[i], x[i], acc);
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

bool geom_ok(const int* L, LexGeom* g) {
  if (!L) return false;
  size_t v = 1;
  for (int mu = 0; mu < 4; ++mu) {
    if (L[mu] < 1) return false;
    g->n[mu] = L[mu];
    v *= (size_t)L[mu];
  }
  g->vol = v;
  return true;
}

int fail_code(int code, const char* msg) {
  set_last_error(code, "%s", msg);
  return code;
}

#define G_CHECK(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      set_last_error(B200_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                     cudaGetErrorString(e_));                                          \
      return B200_ECUDA;                                                               \
    }                                                                                  \
  } while (0)

}  // namespace
}  // namespace b200

using namespace b200;

extern "C" {

int b200_gauge_force_rect(const int lattice[4], double beta, double c_plaq, double c_rect, double* force,
                          const double* u, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !force || !u) return fail_code(B200_EINVAL, "invalid argument");
  const size_t n = 4 * g.vol;
  gauge_force_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(u, force, g, beta, c_plaq,
                                                                                     c_rect);
  G_CHECK(cudaGetLastError());
  return 0;
}

int b200_gauge_action_rect(const int lattice[4], double beta, double c_plaq, double c_rect, const double* u,
                           double* H, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !u || !H) return fail_code(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)((g.vol + 255) / 256);
  double* part = nullptr;
  G_CHECK(cudaMalloc(&part, sizeof(double) * 2 * nb));
  gauge_action_kernel<<<nb, 256, 0, st>>>(u, g, part);
  std::vector<double> h(2 * (size_t)nb);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(part);
  G_CHECK(e);
  double plaqF = 0.0, rectF = 0.0;
  for (int b = 0; b < nb; ++b) { plaqF += h[2 * b]; rectF += h[2 * b + 1]; }
  const double V = (double)g.vol;
  *H = beta * (c_plaq * 6.0 * V - c_plaq * plaqF / 3.0 + c_rect * 12.0 * V - c_rect * rectF / 3.0);
  return 0;
}

int b200_link_update(const int lattice[4], double alpha, const double* ip, double* u, int nprec, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !ip || !u || nprec < 1) return fail_code(B200_EINVAL, "invalid argument");
  const size_t n = 4 * g.vol;
  link_update_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(u, ip, n, alpha, nprec);
  G_CHECK(cudaGetLastError());
  return 0;
}

int b200_momentum_update(const int lattice[4], double eps, const double* force, double* ip, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !force || !ip) return fail_code(B200_EINVAL, "invalid argument");
  const size_t n = 18 * 4 * g.vol;
  axpy_links_kernel<<<592, 256, 0, (cudaStream_t)stream>>>(ip, force, n, eps);
  G_CHECK(cudaGetLastError());
  return 0;
}

int b200_momentum_energy(const int lattice[4], const double* ip, double* H, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !ip || !H) return fail_code(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = 592;
  double* part = nullptr;
  G_CHECK(cudaMalloc(&part, sizeof(double) * nb));
  norm2_links_kernel<<<nb, 256, 0, st>>>(ip, 18 * 4 * g.vol, part);
  std::vector<double> h(nb);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * nb, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(part);
  G_CHECK(e);
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += h[b];
  *H = 0.5 * s;
  return 0;
}

int b200_links_axpby(const int lattice[4], double a, const double* x, double b, double* y, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !x || !y) return fail_code(B200_EINVAL, "invalid argument");
  axpby_links_kernel<<<592, 256, 0, (cudaStream_t)stream>>>(y, x, 18 * 4 * g.vol, a, b);
  G_CHECK(cudaGetLastError());
  return 0;
}

int b200_momentum_from_gauss(const int lattice[4], const double* h, double* ip, void* stream) {
  LexGeom g;
  if (!geom_ok(lattice, &g) || !h || !ip) return fail_code(B200_EINVAL, "invalid argument");
  const size_t n = 4 * g.vol;
  momentum_from_gauss_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
      h, ip, n, 1.0 / std::sqrt(3.0));
  G_CHECK(cudaGetLastError());
  return 0;
}

}  // extern "C"
