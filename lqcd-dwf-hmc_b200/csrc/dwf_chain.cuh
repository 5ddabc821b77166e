// Fifth-dimension operator chains of the even/odd DWF matrix, applied in
// registers to one chirality column x[Ls] (x+- = v_p +- v_(p+2), Dirac basis).
//
// Each primitive is the O(Ls) recurrence of the reference, restated in the
// chiral basis (the reference applies the same maps with (1 +- gamma5)
// projections on full spinors):
//   m5pre   : D_eo pre-factor  b*Wf(x) + c*(Fup(1-g5)x(s+1) + Fdn(1+g5)x(s-1))
//             (src/lib/Fopr/afopr_Domainwall_eo-tmpl.h:764-826;
//              src/lib_alt_Accel/BridgeOpenACC/src/mult_Domainwall_5din_eo_openacc-inc.h:122-227)
//   m5dag   : its adjoint, applied after the dagger hop (:830-898; :346-447)
//   lu_inv  : M_ee^-1 = U^-1 L^-1 (afopr_Domainwall_eo-tmpl.h:1022-1119;
//             mult_Domainwall_5din_LUinv_openacc-inc.h:14-200)
//   ludag   : (M_ee^-1)^+ = L^-+ U^-+ (afopr_Domainwall_eo-tmpl.h:1124-1240;
//             mult_Domainwall_5din_LUinv_openacc-inc.h:204-398)
//   g5r     : gamma5 R (s -> Ls-1-s)
#pragma once

#include "dwf_common.cuh"

namespace b200 {

// Coefficients, passed by value in kernel parameter space (uniform loads).
template <typename R>
struct ChainCoef {
  R wb[kMaxLs];      // b_s
  R wc2[kMaxLs];     // 2*c_s
  R rl[kMaxLs];      // dm_s / dp_(s-1)            (s >= 1)
  R rld[kMaxLs];     // dm_(s+1) / dp_s            (s <= Ls-2)
  R dm[kMaxLs];      // dm_s
  R dpinv[kMaxLs];   // 1/dp_s
  R e[kMaxLs];       // e_s
  R f[kMaxLs];       // f_s
  R alpha, half_alpha, mhalf_mq, dpg_inv;   // alpha, alpha/2, -mq/2, 1/(dp_(Ls-1)+g)
};

template <typename R, int LS, int CHI>
__device__ __forceinline__ void chain_m5pre(const ChainCoef<R>& k, R* x) {
  R y[LS];
#pragma unroll
  for (int s = 0; s < LS; ++s) {
    R wf, hop;
    if (CHI == 0) {
      wf = (s == LS - 1) ? R(1) : k.alpha;
      const R fdn = (s == 0) ? k.mhalf_mq : k.half_alpha;
      hop = k.wc2[s] * fdn * x[(s - 1 + LS) % LS];
    } else {
      wf = (s == 0) ? R(1) : k.alpha;
      const R fup = (s == LS - 1) ? k.mhalf_mq : k.half_alpha;
      hop = k.wc2[s] * fup * x[(s + 1) % LS];
    }
    y[s] = fma(k.wb[s] * wf, x[s], hop);
  }
#pragma unroll
  for (int s = 0; s < LS; ++s) x[s] = y[s];
}

template <typename R, int LS, int CHI>
__device__ __forceinline__ void chain_m5dag(const ChainCoef<R>& k, R* x) {
  R y[LS];
#pragma unroll
  for (int s = 0; s < LS; ++s) {
    R wf, hop;
    if (CHI == 0) {
      wf = (s == LS - 1) ? R(1) : k.alpha;
      const int sp = (s + 1) % LS;
      const R fdn = (sp == 0) ? k.mhalf_mq : k.half_alpha;
      hop = k.wc2[sp] * fdn * x[sp];
    } else {
      wf = (s == 0) ? R(1) : k.alpha;
      const int sm = (s - 1 + LS) % LS;
      const R fup = (sm == LS - 1) ? k.mhalf_mq : k.half_alpha;
      hop = k.wc2[sm] * fup * x[sm];
    }
    y[s] = fma(k.wb[s] * wf, x[s], hop);
  }
#pragma unroll
  for (int s = 0; s < LS; ++s) x[s] = y[s];
}

template <typename R, int LS, int CHI>
__device__ __forceinline__ void chain_lu_inv(const ChainCoef<R>& k, R* x) {
  if (CHI == 0) {
#pragma unroll
    for (int s = 1; s < LS; ++s) x[s] = fma(k.rl[s], x[s - 1], x[s]);
    x[LS - 1] = k.alpha * x[LS - 1] * k.dpg_inv;
    const R Y = x[LS - 1];
#pragma unroll
    for (int s = 0; s < LS - 1; ++s) x[s] = fma(-k.f[s], Y, x[s]) * k.dpinv[s];
  } else {
    R Y = 0;
#pragma unroll
    for (int s = 0; s < LS - 1; ++s) Y = fma(k.e[s], x[s], Y);
    x[LS - 1] = (x[LS - 1] - Y) * k.dpg_inv;
#pragma unroll
    for (int s = LS - 2; s >= 0; --s) x[s] = fma(k.dm[s], x[s + 1], x[s]) * k.dpinv[s];
    x[0] *= k.alpha;
  }
}

template <typename R, int LS, int CHI>
__device__ __forceinline__ void chain_ludag(const ChainCoef<R>& k, R* x) {
  if (CHI == 0) {
    R Y = 0;
#pragma unroll
    for (int s = 0; s < LS - 1; ++s) {
      x[s] *= k.dpinv[s];
      Y = fma(k.f[s], x[s], Y);
    }
    x[LS - 1] = k.alpha * (x[LS - 1] - Y) * k.dpg_inv;
#pragma unroll
    for (int s = LS - 2; s >= 0; --s) x[s] = fma(k.rld[s], x[s + 1], x[s]);
  } else {
    x[0] = k.alpha * x[0] * k.dpinv[0];
#pragma unroll
    for (int s = 1; s < LS - 1; ++s) x[s] = fma(k.dm[s - 1], x[s - 1], x[s]) * k.dpinv[s];
    x[LS - 1] = fma(k.dm[LS - 2], x[LS - 2], x[LS - 1]) * k.dpg_inv;
    const R Y = x[LS - 1];
#pragma unroll
    for (int s = 0; s < LS - 1; ++s) x[s] = fma(-k.e[s], Y, x[s]);
  }
}

template <typename R, int LS, int CHI>
__device__ __forceinline__ void chain_g5r(R* x) {
  R y[LS];
#pragma unroll
  for (int s = 0; s < LS; ++s) y[s] = (CHI == 0) ? x[LS - 1 - s] : -x[LS - 1 - s];
#pragma unroll
  for (int s = 0; s < LS; ++s) x[s] = y[s];
}

template <typename R, int LS>
__device__ __forceinline__ void chain_scale(R* x, R a) {
#pragma unroll
  for (int s = 0; s < LS; ++s) x[s] *= a;
}

// Epilogue chains used by the fused hop kernel (E applied to the hop result).
enum EpiKind {
  EPI_HALF = 0,    // -1/2                         (D_eo after a separate M5 pre-factor)
  EPI_DDAGEO = 1,  // M5^+ (-1/2 g5)               (D_eo^+)
  EPI_K1 = 2,      // M5pre M_ee^-1 (-1/2)         (D chain, first hop)
  EPI_K2N = 3,     // -M_ee^-1 (-1/2)              (D chain, second hop: o = w + this)
  EPI_K3 = 4,      // M_ee^-+ M5^+ (-1/2 g5)       (D^+ chain, first hop)
  EPI_K4N = 5,     // -M5^+ (-1/2 g5)              (D^+ chain, second hop)
  EPI_COUNT = 6
};
// Second maps F applied to o1.
enum FKind { F_NONE = 0, F_LUDAG = 1, F_G5R = 2 };

template <int EPI> struct EpiIsDag { static constexpr bool v = (EPI == EPI_DDAGEO || EPI == EPI_K3 || EPI == EPI_K4N); };

template <typename R, int LS, int CHI, int EPI>
__device__ __forceinline__ void apply_epi(const ChainCoef<R>& k, R* x) {
  // gamma5 in the chiral basis: +1 on chi=0, -1 on chi=1
  const R g5 = (CHI == 0) ? R(1) : R(-1);
  if (EPI == EPI_HALF) {
    chain_scale<R, LS>(x, R(-0.5));
  } else if (EPI == EPI_DDAGEO) {
    chain_scale<R, LS>(x, R(-0.5) * g5);
    chain_m5dag<R, LS, CHI>(k, x);
  } else if (EPI == EPI_K1) {
    chain_scale<R, LS>(x, R(-0.5));
    chain_lu_inv<R, LS, CHI>(k, x);
    chain_m5pre<R, LS, CHI>(k, x);
  } else if (EPI == EPI_K2N) {
    chain_scale<R, LS>(x, R(0.5));
    chain_lu_inv<R, LS, CHI>(k, x);
  } else if (EPI == EPI_K3) {
    chain_scale<R, LS>(x, R(-0.5) * g5);
    chain_m5dag<R, LS, CHI>(k, x);
    chain_ludag<R, LS, CHI>(k, x);
  } else {  // EPI_K4N
    chain_scale<R, LS>(x, R(0.5) * g5);
    chain_m5dag<R, LS, CHI>(k, x);
  }
}

template <typename R, int LS, int CHI, int FK>
__device__ __forceinline__ void apply_f(const ChainCoef<R>& k, R* x) {
  if (FK == F_LUDAG) chain_ludag<R, LS, CHI>(k, x);
  else if (FK == F_G5R) chain_g5r<R, LS, CHI>(x);
}

// A warp's shared-memory tile holds, per (site g, slice s), the 24 reals of
// one spinor in a row of TileStride<R>::v elements.  The padding (26 doubles,
// 28 floats) makes both the per-thread 16-byte row accesses and the
// per-unit column walks of tile_chiral free of bank conflicts.
template <typename R> struct TileStride { static constexpr int v = 26; };
template <> struct TileStride<float> { static constexpr int v = 28; };

// Elements between the tiles of consecutive sites g of a warp: LS rows plus a
// pad that puts site g+1's columns half a bank cycle away from site g's, so
// the column walks of tile_chiral for two sites do not collide.
template <typename R, int LS> struct TileGroup {
  static constexpr int rows = LS * TileStride<R>::v;
  static constexpr int mod = sizeof(R) == 8 ? 16 : 32;       // elements per bank cycle
  static constexpr int target = sizeof(R) == 8 ? 12 : 16;
  static constexpr int v = rows + ((target - rows % mod) % mod + mod) % mod;
};
template <typename R, int LS, int G> struct TileWarp { static constexpr int v = G * TileGroup<R, LS>::v; };

template <typename R, int LS>
__device__ __forceinline__ R* tile_row(R* tile, int g, int s) {
  return tile + g * TileGroup<R, LS>::v + s * TileStride<R>::v;
}

__device__ __forceinline__ void tile_put(double* row, const double* v) {
#pragma unroll
  for (int k = 0; k < 12; ++k) reinterpret_cast<double2*>(row)[k] = make_double2(v[2 * k], v[2 * k + 1]);
}
__device__ __forceinline__ void tile_put(float* row, const float* v) {
#pragma unroll
  for (int k = 0; k < 6; ++k)
    reinterpret_cast<float4*>(row)[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}
__device__ __forceinline__ void tile_get(const double* row, double* v) {
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const double2 c = reinterpret_cast<const double2*>(row)[k];
    v[2 * k] = c.x; v[2 * k + 1] = c.y;
  }
}
__device__ __forceinline__ void tile_get(const float* row, float* v) {
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float4 c = reinterpret_cast<const float4*>(row)[k];
    v[4 * k] = c.x; v[4 * k + 1] = c.y; v[4 * k + 2] = c.z; v[4 * k + 3] = c.w;
  }
}

// Run `op` on every unit (site g, color, ri, spin pair) of a warp's tile
// [g][s][TileStride]: gather the chirality columns, apply, scatter back in place.
template <typename R, int LS, int G, typename Op>
__device__ __forceinline__ void tile_chiral(R* tile, int lane, Op op) {
  constexpr int TS = TileStride<R>::v;
#pragma unroll 1
  for (int u = lane; u < 12 * G; u += 32) {
    const int g = u / 12;
    const int r = u - 12 * g;
    const int pair = r / 6;
    const int cr = r - 6 * pair;
    R* t = tile + g * TileGroup<R, LS>::v + 6 * pair + cr;
    R xp[LS], xm[LS];
#pragma unroll
    for (int s = 0; s < LS; ++s) {
      const R a = t[s * TS];
      const R b = t[s * TS + 12];
      xp[s] = a + b;
      xm[s] = a - b;
    }
    op(xp, xm);
#pragma unroll
    for (int s = 0; s < LS; ++s) {
      t[s * TS] = R(0.5) * (xp[s] + xm[s]);
      t[s * TS + 12] = R(0.5) * (xp[s] - xm[s]);
    }
  }
}

}  // namespace b200
