// Fused fermion-force kernel of the even/odd 5D domain-wall operator.
//
// The reference (src/lib/Force/Fermion/force_F_Domainwall_eo.cpp:190-318;
// GPU form src/lib_alt_Accel/Force/Fermion/aforce_F_Domainwall_5din-tmpl.h:
// 341-1217 + tensorProd_5din) forms, per direction mu and site x of one
// parity, F_mu(x) = sum_s sum_spin [U_mu(x)^+ D_mu(x)]_c1 conj(v(x))_c2 where
// D_mu is the forward-mu part of D_eo (or of its dagger).  U^+ U = 1 removes
// the link, and the fifth-dimension chain of the dagger moves onto v as its
// adjoint, so every term has the form
//     F_mu(x) += coef * sum_s sum_spin [(1 -+ g_mu) Y(x+mu, s)]_c1 conj(Z(x, s))_c2
// with the boundary phase of the x -> x+mu hop.  This kernel computes up to
// two such terms (term 1 with (1 - g_mu), term 2 with (1 + g_mu)) for all four
// directions in one pass over the sites of one
// parity, never materialising shifted fields: one thread per (site, s), the
// spin sum done on projected half spinors, the s sum reduced on a
// shared-memory tile, and the 3x3 result written into the lexical
// Field_G(Nvol, 4) force (18 reals per (site, mu)).
#include "dwf_hop.cuh"
#include "dwf_kernels.h"

namespace b200 {

template <int LS, bool T1, bool T2>
__global__ void __launch_bounds__(128) force_kernel(ForceParams p) {
  using St = Store<PREC_F64>;
  using R = double;
  constexpr int G = 32 / LS;
  constexpr int WARPS = 4;
  extern __shared__ unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw) + (size_t)(threadIdx.x >> 5) * G * LS * 18;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane / LS;
  const int s = lane - g * LS;
  const int site = (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.vh);
  const size_t vh = p.vh;

  int x = 0, y = 0, z = 0, t = 0, ix2 = 0, iyzt = 0, keo = 0;
  if (active) {
    ix2 = site % p.nx2;
    iyzt = site / p.nx2;
    y = iyzt % p.ny;
    const int izt = iyzt / p.ny;
    z = izt % p.nz;
    t = izt / p.nz;
    keo = (p.ieo + y + z + t) & 1;
    x = 2 * ix2 + keo;
  }
  R z1[24], z2[24];
  if (active) {
    if (T1) St::load(p.z1, vh, LS, site, s, z1);
    if (T2) St::load(p.z2, vh, LS, site, s, z2);
  }

#define B200_FORCE_MU(MU, COORD, EXT, NBP)                                            \
  {                                                                                   \
    R f[18];                                                                          \
    _Pragma("unroll") for (int i = 0; i < 18; ++i) f[i] = 0;                          \
    if (active) {                                                                     \
      const R ph = (COORD == EXT - 1) ? (R)p.bc[MU] : R(1);                           \
      const int nb = NBP;                                                             \
      const R half_t = (MU == 3) ? R(0.5) : R(1);                                     \
      R w[24], h[12], gz[12];                                                         \
      if (T1) {                                                                       \
        St::load(p.y1, vh, LS, nb, s, w);                                             \
        project<R, MU, 1>(w, h);                                                      \
        project<R, MU, 1>(z1, gz);                                                    \
        _Pragma("unroll") for (int a = 0; a < 2; ++a)                                 \
        _Pragma("unroll") for (int c1 = 0; c1 < 3; ++c1)                              \
        _Pragma("unroll") for (int c2 = 0; c2 < 3; ++c2) {                            \
          const R hr = h[6 * a + 2 * c1], hi = h[6 * a + 2 * c1 + 1];                 \
          const R gr = gz[6 * a + 2 * c2], gi = gz[6 * a + 2 * c2 + 1];               \
          f[2 * (c2 + 3 * c1)] += ph * half_t * (hr * gr + hi * gi);                  \
          f[2 * (c2 + 3 * c1) + 1] += ph * half_t * (hi * gr - hr * gi);              \
        }                                                                             \
      }                                                                               \
      if (T2) {                                                                       \
        St::load(p.y2, vh, LS, nb, s, w);                                             \
        project<R, MU, -1>(w, h);                                                     \
        project<R, MU, -1>(z2, gz);                                                   \
        _Pragma("unroll") for (int a = 0; a < 2; ++a)                                 \
        _Pragma("unroll") for (int c1 = 0; c1 < 3; ++c1)                              \
        _Pragma("unroll") for (int c2 = 0; c2 < 3; ++c2) {                            \
          const R hr = h[6 * a + 2 * c1], hi = h[6 * a + 2 * c1 + 1];                 \
          const R gr = gz[6 * a + 2 * c2], gi = gz[6 * a + 2 * c2 + 1];               \
          f[2 * (c2 + 3 * c1)] += ph * half_t * (hr * gr + hi * gi);                  \
          f[2 * (c2 + 3 * c1) + 1] += ph * half_t * (hi * gr - hr * gi);              \
        }                                                                             \
      }                                                                               \
    }                                                                                 \
    __syncwarp();                                                                     \
    if (g < G) {                                                                      \
      _Pragma("unroll") for (int i = 0; i < 18; ++i) tile[(g * LS + s) * 18 + i] = f[i]; \
    }                                                                                 \
    __syncwarp();                                                                     \
    for (int o = lane; o < 18 * G; o += 32) {                                         \
      const int gg = o / 18, i = o - 18 * gg;                                         \
      const int st = (blockIdx.x * WARPS + warp) * G + gg;                            \
      if (st < p.vh) {                                                                \
        R sum = 0;                                                                    \
        for (int q = 0; q < LS; ++q) sum += tile[(gg * LS + q) * 18 + i];             \
        const int sx2 = st % p.nx2, syzt = st / p.nx2;                                \
        const int sy = syzt % p.ny, sz = (syzt / p.ny) % p.nz, stt = syzt / (p.ny * p.nz); \
        const int sxx = 2 * sx2 + ((p.ieo + sy + sz + stt) & 1);                      \
        const size_t lex = sxx + (size_t)(2 * p.nx2) *                                \
                           (sy + (size_t)p.ny * (sz + (size_t)p.nz * stt));           \
        double* dst = p.force + 18 * (lex + (size_t)2 * vh * MU) + i;                 \
        *dst = (p.beta != 0.0 ? p.beta * (*dst) : 0.0) + p.coef * sum;               \
      }                                                                               \
    }                                                                                 \
  }

  const int row = p.nx2 * iyzt;
  B200_FORCE_MU(0, x, 2 * p.nx2, row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo))
  B200_FORCE_MU(1, y, p.ny, (y == p.ny - 1) ? site - (p.ny - 1) * p.nx2 : site + p.nx2)
  const int sz_ = p.nx2 * p.ny;
  B200_FORCE_MU(2, z, p.nz, (z == p.nz - 1) ? site - (p.nz - 1) * sz_ : site + sz_)
  const int st_ = p.nx2 * p.ny * p.nz;
  B200_FORCE_MU(3, t, p.nt, (t == p.nt - 1) ? site - (p.nt - 1) * st_ : site + st_)
#undef B200_FORCE_MU
}

template <int LS>
cudaError_t run_force(const ForceParams& p, cudaStream_t st) {
  constexpr size_t smem = sizeof(double) * 4 * (32 / LS) * LS * 18;
  const int grid = hop_grid(LS, p.vh);
  if (p.y1 && p.y2) force_kernel<LS, true, true><<<grid, 128, smem, st>>>(p);
  else if (p.y1) force_kernel<LS, true, false><<<grid, 128, smem, st>>>(p);
  else if (p.y2) force_kernel<LS, false, true><<<grid, 128, smem, st>>>(p);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_force(const ForceParams& p, cudaStream_t st) {
  switch (p.ls) {
    case 4: return run_force<4>(p, st);
    case 6: return run_force<6>(p, st);
    case 8: return run_force<8>(p, st);
    case 12: return run_force<12>(p, st);
    case 16: return run_force<16>(p, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace b200
