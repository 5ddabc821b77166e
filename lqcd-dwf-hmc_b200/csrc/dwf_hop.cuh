// Fused even/odd 5D domain-wall hopping kernel for sm_100a.
//
// One thread per (4D site, s).  A warp holds G = 32/Ls complete 4D sites, so
// every SU(3) link is fetched by one broadcast transaction per site and reused
// by all Ls lanes of that site from registers.  The fifth-dimension operators
// that surround the hop in the reference (the M5 pre-factor of D_eo, M5^+ after
// the dagger hop, M_ee^-1 = U^-1 L^-1 and its dagger, gamma5 R) are all linear
// maps along s that are block-diagonal in chirality, so any chain of them is a
// pair of dense Ls x Ls real matrices (E+, E-).  The kernel applies that pair in
// its epilogue on a shared-memory tile of the site's whole fifth-dimension
// column, then optionally forms o1 = c*X + E(acc), o2 = F(o1), stores o1/o2 and
// reduces |o1|^2 -- the fusions used by the CG iteration.
//
// Reference behaviour (file:line relative to the reference tree):
//   hop with Dirac projections, no -kappa: src/lib_alt_Accel/BridgeOpenACC/src/
//     mult_Domainwall_5din_eo_openacc-inc.h:450-550 (+ inc/ files); jgm5=1
//     gives the gamma5-sandwiched dagger hop.
//   boundary phase applied at the lattice edge in-kernel (inc/*_xyz, bc2).
#pragma once

#include "dwf_common.cuh"
#include "dwf_chain.cuh"
#include "tma_util.cuh"

namespace b200 {

enum LinkFmt {
  LINK_F64_18 = 0, LINK_F64_12 = 1, LINK_F32_12 = 2, LINK_F16_12 = 3, LINK_F32_18 = 4, LINK_F16_18 = 5,
  LINK_NFMT = 6
};

template <int LF> struct LinkLoad;

// kFolded: the plan stores this format with two constant factors of the hop
// already multiplied into the links: the boundary phase bc[mu] on the links
// of the last slice along mu, and the factor 2 of the (1 -+ gamma_4)
// projection on every t link (full 3x3 records only: a reconstructed third
// row would carry neither).  The hop kernels then skip the per-direction
// phase and the doubling of the t projection.
template <> struct LinkLoad<LINK_F64_18> {
  using R = double;
  static constexpr int kChunks = 9;
  static constexpr bool kFolded = true;
  __device__ static void load_plain(const void* rec, double* u) {
    const double2* p = reinterpret_cast<const double2*>(rec);
#pragma unroll
    for (int j = 0; j < 9; ++j) { double2 c = p[j]; u[2 * j] = c.x; u[2 * j + 1] = c.y; }
  }
  __device__ static void load(const void* base, size_t idx, double* u) {
    const double2* p = reinterpret_cast<const double2*>(base) + idx * 9;
#pragma unroll
    for (int j = 0; j < 9; ++j) { double2 c = __ldg(p + j); u[2 * j] = c.x; u[2 * j + 1] = c.y; }
  }
};
template <> struct LinkLoad<LINK_F64_12> {
  using R = double;
  static constexpr int kChunks = 6;
  static constexpr bool kFolded = false;
  __device__ static void load_plain(const void* rec, double* u) {
    const double2* p = reinterpret_cast<const double2*>(rec);
#pragma unroll
    for (int j = 0; j < 6; ++j) { double2 c = p[j]; u[2 * j] = c.x; u[2 * j + 1] = c.y; }
    su3_reconstruct(u);
  }
  __device__ static void load(const void* base, size_t idx, double* u) {
    const double2* p = reinterpret_cast<const double2*>(base) + idx * 6;
#pragma unroll
    for (int j = 0; j < 6; ++j) { double2 c = __ldg(p + j); u[2 * j] = c.x; u[2 * j + 1] = c.y; }
    su3_reconstruct(u);
  }
};
template <> struct LinkLoad<LINK_F32_12> {
  using R = float;
  static constexpr int kChunks = 3;
  static constexpr bool kFolded = false;
  __device__ static void load_plain(const void* rec, float* u) {
    const float4* p = reinterpret_cast<const float4*>(rec);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float4 c = p[j];
      u[4 * j] = c.x; u[4 * j + 1] = c.y; u[4 * j + 2] = c.z; u[4 * j + 3] = c.w;
    }
    su3_reconstruct(u);
  }
  __device__ static void load(const void* base, size_t idx, float* u) {
    const float4* p = reinterpret_cast<const float4*>(base) + idx * 3;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float4 c = __ldg(p + j);
      u[4 * j] = c.x; u[4 * j + 1] = c.y; u[4 * j + 2] = c.z; u[4 * j + 3] = c.w;
    }
    su3_reconstruct(u);
  }
};
template <> struct LinkLoad<LINK_F16_12> {
  using R = float;
  static constexpr int kChunks = 2;
  static constexpr bool kFolded = false;
  __device__ static void load_plain(const void* rec, float* u) {
    const uint4* p = reinterpret_cast<const uint4*>(rec);
    uint4 a = p[0], b = p[1];
    unsigned int w[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      float2 f = HalfOps<__half>::to2(w[j]);
      u[2 * j] = f.x; u[2 * j + 1] = f.y;
    }
    su3_reconstruct(u);
  }
  __device__ static void load(const void* base, size_t idx, float* u) {
    const uint4* p = reinterpret_cast<const uint4*>(base) + idx * 2;
    uint4 a = __ldg(p), b = __ldg(p + 1);
    unsigned int w[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      float2 f = HalfOps<__half>::to2(w[j]);
      u[2 * j] = f.x; u[2 * j + 1] = f.y;
    }
    su3_reconstruct(u);
  }
};

// Full 3x3 records in FP32 (18 floats padded to 5 float4) and in FP16 (18
// halves padded to 3 uint4): no third-row rebuild in the hop (the lanes of a
// site would each repeat it), phase and t factor folded in like LINK_F64_18.
template <> struct LinkLoad<LINK_F32_18> {
  using R = float;
  static constexpr int kChunks = 5;
  static constexpr bool kFolded = true;
  __device__ static void load_plain(const void* rec, float* u) {
    const float4* p = reinterpret_cast<const float4*>(rec);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float4 c = p[j];
      u[4 * j] = c.x; u[4 * j + 1] = c.y; u[4 * j + 2] = c.z; u[4 * j + 3] = c.w;
    }
    const float2 c = reinterpret_cast<const float2*>(p + 4)[0];
    u[16] = c.x; u[17] = c.y;
  }
  __device__ static void load(const void* base, size_t idx, float* u) {
    const float4* p = reinterpret_cast<const float4*>(base) + idx * 5;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float4 c = __ldg(p + j);
      u[4 * j] = c.x; u[4 * j + 1] = c.y; u[4 * j + 2] = c.z; u[4 * j + 3] = c.w;
    }
    const float2 c = __ldg(reinterpret_cast<const float2*>(p + 4));
    u[16] = c.x; u[17] = c.y;
  }
};
template <> struct LinkLoad<LINK_F16_18> {
  using R = float;
  static constexpr int kChunks = 3;
  static constexpr bool kFolded = true;
  __device__ static void decode(uint4 a, uint4 b, uint4 c, float* u) {
    const unsigned int w[9] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x};
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      float2 f = HalfOps<__half>::to2(w[j]);
      u[2 * j] = f.x; u[2 * j + 1] = f.y;
    }
  }
  __device__ static void load_plain(const void* rec, float* u) {
    const uint4* p = reinterpret_cast<const uint4*>(rec);
    decode(p[0], p[1], p[2], u);
  }
  __device__ static void load(const void* base, size_t idx, float* u) {
    const uint4* p = reinterpret_cast<const uint4*>(base) + idx * 3;
    decode(__ldg(p), __ldg(p + 1), __ldg(p + 2), u);
  }
};

// ------------------------------------------------------------ complex helpers
template <typename R>
__device__ __forceinline__ void cmul_acc(R& ore, R& oim, R ar, R ai, R br, R bi) {
  ore = fma(ar, br, ore); ore = fma(-ai, bi, ore);
  oim = fma(ar, bi, oim); oim = fma(ai, br, oim);
}

// out[2] (half spinor, 3 colors each, 12 reals) = U * h  or U^+ * h
template <typename R, bool kDag>
__device__ __forceinline__ void su3_mult_half(const R* u, const R* h, R* o) {
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      R re = 0, im = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const R ur = kDag ? u[2 * (i + 3 * j)] : u[2 * (j + 3 * i)];
        const R ui = kDag ? -u[2 * (i + 3 * j) + 1] : u[2 * (j + 3 * i) + 1];
        cmul_acc(re, im, ur, ui, h[6 * a + 2 * j], h[6 * a + 2 * j + 1]);
      }
      o[6 * a + 2 * i] = re;
      o[6 * a + 2 * i + 1] = im;
    }
  }
}

// Spin projection (1 - sign*gamma_mu) w -> half spinor h (2 spins x 3 colors)
// and reconstruction acc += ph * (1 - sign*gamma_mu)-shaped result from uh.
// Dirac basis (reference src/lib/Tools/gammaMatrixSet_Dirac.cpp:31-60).
// w index: ri + 2*(c + 3*sp).  sign = +1 forward (1-g), -1 backward (1+g).
// kT2 = false: the t links carry the projection's factor 2 (kFolded formats).
template <typename R, int MU, int SIGN, bool kT2 = true>
__device__ __forceinline__ void project(const R* w, R* h) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const R w0r = w[2 * c], w0i = w[2 * c + 1];
    const R w1r = w[2 * (c + 3)], w1i = w[2 * (c + 3) + 1];
    const R w2r = w[2 * (c + 6)], w2i = w[2 * (c + 6) + 1];
    const R w3r = w[2 * (c + 9)], w3i = w[2 * (c + 9) + 1];
    R h0r, h0i, h1r, h1i;
    if (MU == 0) {        // (1 -+ g1): h0 = w0 +- i w3, h1 = w1 +- i w2
      h0r = w0r - SIGN * w3i; h0i = w0i + SIGN * w3r;
      h1r = w1r - SIGN * w2i; h1i = w1i + SIGN * w2r;
    } else if (MU == 1) { // (1 -+ g2): h0 = w0 +- w3, h1 = w1 -+ w2
      h0r = w0r + SIGN * w3r; h0i = w0i + SIGN * w3i;
      h1r = w1r - SIGN * w2r; h1i = w1i - SIGN * w2i;
    } else if (MU == 2) { // (1 -+ g3): h0 = w0 +- i w2, h1 = w1 -+ i w3
      h0r = w0r - SIGN * w2i; h0i = w0i + SIGN * w2r;
      h1r = w1r + SIGN * w3i; h1i = w1i - SIGN * w3r;
    } else {              // (1 - g4) keeps lower spins, (1 + g4) upper, x2
      const R two = kT2 ? R(2) : R(1);
      if (SIGN > 0) { h0r = two * w2r; h0i = two * w2i; h1r = two * w3r; h1i = two * w3i; }
      else          { h0r = two * w0r; h0i = two * w0i; h1r = two * w1r; h1i = two * w1i; }
    }
    h[2 * c] = h0r; h[2 * c + 1] = h0i;
    h[6 + 2 * c] = h1r; h[6 + 2 * c + 1] = h1i;
  }
}

// kUnit: the phase is 1 (phased links), no multiplication is issued.
template <typename R, int MU, int SIGN, bool kUnit = false>
__device__ __forceinline__ void reconstruct_acc(R* acc, const R* o, R ph) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const R a0r = kUnit ? o[2 * c] : ph * o[2 * c], a0i = kUnit ? o[2 * c + 1] : ph * o[2 * c + 1];
    const R a1r = kUnit ? o[6 + 2 * c] : ph * o[6 + 2 * c];
    const R a1i = kUnit ? o[6 + 2 * c + 1] : ph * o[6 + 2 * c + 1];
    R* r0 = acc + 2 * c;
    R* r1 = acc + 2 * (c + 3);
    R* r2 = acc + 2 * (c + 6);
    R* r3 = acc + 2 * (c + 9);
    if (MU == 3) {
      if (SIGN > 0) { r2[0] += a0r; r2[1] += a0i; r3[0] += a1r; r3[1] += a1i; }
      else          { r0[0] += a0r; r0[1] += a0i; r1[0] += a1r; r1[1] += a1i; }
      continue;
    }
    r0[0] += a0r; r0[1] += a0i;
    r1[0] += a1r; r1[1] += a1i;
    if (MU == 0) {        // rows 2,3 = -+ i h1, -+ i h0
      r2[0] += SIGN * a1i; r2[1] -= SIGN * a1r;
      r3[0] += SIGN * a0i; r3[1] -= SIGN * a0r;
    } else if (MU == 1) { // rows 2,3 = -+ h1, +- h0
      r2[0] -= SIGN * a1r; r2[1] -= SIGN * a1i;
      r3[0] += SIGN * a0r; r3[1] += SIGN * a0i;
    } else {              // MU==2: rows 2,3 = -+ i h0, +- i h1
      r2[0] += SIGN * a0i; r2[1] -= SIGN * a0r;
      r3[0] -= SIGN * a1i; r3[1] += SIGN * a1r;
    }
  }
}

// One hop direction for full (18-real) FP64 link records read from shared
// memory, colour by colour: for output colour i only the three link entries
// it needs (row i of U, or column i for U^+) are loaded, multiplied into both
// projected spins and reconstructed into acc, so the live state is the
// accumulator, the projected half spinor and one link row (instead of the
// whole link and the whole product).  Phased links (no edge factor).
template <int MU, int SIGN>
__device__ __forceinline__ void hop_dir_rows_f64(const double2* urec, const double* h, double* acc) {
  constexpr bool kDag = SIGN < 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double2 uc[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) uc[j] = urec[kDag ? (3 * j + i) : (3 * i + j)];
    if (MU == 3) {
      // the t projection keeps one spin pair, so U h lands in it unchanged:
      // the multiply-add chains start from the accumulator itself
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        double* tgt = acc + 2 * (i + 3 * (a + (SIGN > 0 ? 2 : 0)));
        double re = tgt[0], im = tgt[1];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const double ur = uc[j].x;
          const double ui = kDag ? -uc[j].y : uc[j].y;
          cmul_acc(re, im, ur, ui, h[6 * a + 2 * j], h[6 * a + 2 * j + 1]);
        }
        tgt[0] = re;
        tgt[1] = im;
      }
      continue;
    }
    double o[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) o[q] = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double ur = uc[j].x;
        const double ui = kDag ? -uc[j].y : uc[j].y;
        cmul_acc(re, im, ur, ui, h[6 * a + 2 * j], h[6 * a + 2 * j + 1]);
      }
      o[6 * a + 2 * i] = re;
      o[6 * a + 2 * i + 1] = im;
    }
    // reconstruct colour i only (reconstruct_acc's colour loop body)
    const double a0r = o[2 * i], a0i = o[2 * i + 1];
    const double a1r = o[6 + 2 * i], a1i = o[6 + 2 * i + 1];
    double* r0 = acc + 2 * i;
    double* r1 = acc + 2 * (i + 3);
    double* r2 = acc + 2 * (i + 6);
    double* r3 = acc + 2 * (i + 9);
    r0[0] += a0r; r0[1] += a0i;
    r1[0] += a1r; r1[1] += a1i;
    if (MU == 0) {
      r2[0] += SIGN * a1i; r2[1] -= SIGN * a1r;
      r3[0] += SIGN * a0i; r3[1] -= SIGN * a0r;
    } else if (MU == 1) {
      r2[0] -= SIGN * a1r; r2[1] -= SIGN * a1i;
      r3[0] += SIGN * a0r; r3[1] += SIGN * a0i;
    } else {
      r2[0] += SIGN * a0i; r2[1] -= SIGN * a0r;
      r3[0] -= SIGN * a1i; r3[1] += SIGN * a1r;
    }
  }
}

// ------------------------------------------------------------ parameters
struct HopParams {
  const void* in;        // input field (parity 1-ieo)
  const void* links;     // plan links (layout per LinkFmt)
  void* out1;            // o1 store target (nullable)
  void* out2;            // o2 store target (nullable)
  const void* x1;        // axpy operand X (nullable)
  int epi;               // EpiKind applied to the hop result
  int fk;                // FKind second map, o2 = F o1 (F_NONE: no o2)
  int variant;           // occupancy variant (0/1), chosen by the autotuner
  const void* x2;        // second axpy operand (nullable)
  const void* x3;        // third axpy operand (nullable)
  // o1 = ce * E(acc) + c_x1 * X1 + c_x2 * X2 + c_x3 * X3; each scalar is
  // multiplied by the device value behind its _dev pointer when non-null
  double ce, c_x1, c_x2, c_x3;
  const double* ce_dev;
  const double* c_x1_dev;
  const double* c_x2_dev;
  const double* c_x3_dev;
  double* red;           // per-block partials of |o1|^2 (nullable)
  int* err;              // device error word: 1 when a bounded wait gave up, 2 when the
                         // drain of the copies still in flight gave up as well
  int fail_dir;          // host-set test hook: the wait for this hop direction (0..7)
                         // reports failure as if its bound had run out (-1: none)
  unsigned int wait_ns;  // suspend-time hint of the TMA kernels' mbarrier tries (0: none)
  const double* skip;    // when non-null and *skip != 0 the launch does nothing
                         // (lets a captured solver iteration replay as a no-op)
  int vh, nx2, ny, nz, nt, ls;
  int site0, site_end;   // output sites [site0, site_end) of this launch (the plan: 0, vh)
  int ieo;               // output parity (0 even, 1 odd)
  double bc[4];
};

// Epilogue shared by the hop kernels: chain E on the site column, axpy with
// up to three fields, store o1, optional F map -> o2, |o1|^2 block partials.
// Each thread finishes NR rows (slices srow[r]) of its site; GT sites per warp.
// With NR = 2 a block covers the sites of two one-row blocks and writes its
// |o1|^2 partial to red[2*block] (and zero to red[2*block + 1]), so the host
// reduces the same number of partials for either kernel shape.
template <int LS, int P, int EPI, int FK, int NR, int GT>
__device__ __forceinline__ void hop_epilogue_rows(const HopParams& p,
                                                  const ChainCoef<typename Store<P>::R>& k,
                                                  typename Store<P>::R (*acc)[24],
                                                  typename Store<P>::R* tile, double* red_warp,
                                                  int tid, int lane, int warp, int g,
                                                  const int* srow, int site, bool active) {
  using St = Store<P>;
  using R = typename St::R;
  constexpr int WARPS = 4;
  const size_t vh = p.vh;
  R o1[NR][24];
  // ce is uniform over the launch: folded into the constant factor of
  // EPI_HALF, and skipped when it is 1 (both exact, so results are unchanged)
  const R ce = (R)(p.ce * (p.ce_dev ? *p.ce_dev : 1.0));
  bool ce_done = (ce == R(1));
  if (EPI == EPI_HALF) {
    const R c = R(-0.5) * ce;
#pragma unroll
    for (int r = 0; r < NR; ++r)
#pragma unroll
      for (int i = 0; i < 24; ++i) o1[r][i] = c * acc[r][i];
    ce_done = true;
  } else if (NR == 1 && (EPI == EPI_DDAGEO || EPI == EPI_K4N)) {
    // c * M5^+ g5 acc (c = -1/2 or +1/2): in the chiral basis M5^+ couples s
    // only to s+1 (x+) or s-1 (x-) of the same site, whose values sit in the
    // neighbouring lanes, so the chain is two warp shuffles per component and
    // needs no shared-memory tile.  Coefficients as in chain_m5dag, with the
    // g5 sign, the 1/2 of the back transform and c folded in.
    const int s = srow[0];
    const R c = (EPI == EPI_DDAGEO) ? R(-0.5) : R(0.5);
    const int sp = (s + 1 == LS) ? 0 : s + 1;
    const int sm = (s == 0) ? LS - 1 : s - 1;
    const R wf0 = (s == LS - 1) ? R(1) : k.alpha;
    const R wf1 = (s == 0) ? R(1) : k.alpha;
    const R fdn = (sp == 0) ? k.mhalf_mq : k.half_alpha;
    const R fup = (sm == LS - 1) ? k.mhalf_mq : k.half_alpha;
    const R hc = R(0.5) * c;
    const R a0 = hc * k.wb[s] * wf0, b0 = hc * k.wc2[sp] * fdn;
    const R a1 = -hc * k.wb[s] * wf1, b1 = -hc * k.wc2[sm] * fup;
    const int lup = g * LS + sp, ldn = g * LS + sm;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const R xp = acc[0][i] + acc[0][i + 12];
      const R xm = acc[0][i] - acc[0][i + 12];
      const R xpu = __shfl_sync(0xffffffffu, xp, lup);
      const R xmd = __shfl_sync(0xffffffffu, xm, ldn);
      const R yp = fma(a0, xp, b0 * xpu);
      const R ym = fma(a1, xm, b1 * xmd);
      o1[0][i] = yp + ym;
      o1[0][i + 12] = yp - ym;
    }
  } else {
    if (g < GT) {
#pragma unroll
      for (int r = 0; r < NR; ++r) tile_put(tile_row<R, LS>(tile, g, srow[r]), acc[r]);
    }
    __syncwarp();
    tile_chiral<R, LS, GT>(tile, lane, [&](R* xp, R* xm) {
      apply_epi<R, LS, 0, EPI>(k, xp);
      apply_epi<R, LS, 1, EPI>(k, xm);
    });
    __syncwarp();
    if (g < GT) {
#pragma unroll
      for (int r = 0; r < NR; ++r) tile_get(tile_row<R, LS>(tile, g, srow[r]), o1[r]);
    }
  }

  double nrm = 0.0;
  if (active) {
    const R c1 = (R)(p.c_x1 * (p.c_x1_dev ? *p.c_x1_dev : 1.0));
    const R c2 = (R)(p.c_x2 * (p.c_x2_dev ? *p.c_x2_dev : 1.0));
    const R c3 = (R)(p.c_x3 * (p.c_x3_dev ? *p.c_x3_dev : 1.0));
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int s = srow[r];
#pragma unroll
      if (!ce_done)
#pragma unroll
        for (int i = 0; i < 24; ++i) o1[r][i] *= ce;
      if (p.x1) {
        R xv[24];
        St::load(p.x1, vh, LS, site, s, xv);
#pragma unroll
        for (int i = 0; i < 24; ++i) o1[r][i] = fma(c1, xv[i], o1[r][i]);
      }
      if (p.x2) {
        R xv[24];
        St::load(p.x2, vh, LS, site, s, xv);
#pragma unroll
        for (int i = 0; i < 24; ++i) o1[r][i] = fma(c2, xv[i], o1[r][i]);
      }
      if (p.x3) {
        R xv[24];
        St::load(p.x3, vh, LS, site, s, xv);
#pragma unroll
        for (int i = 0; i < 24; ++i) o1[r][i] = fma(c3, xv[i], o1[r][i]);
      }
      if (p.out1) St::store(p.out1, vh, LS, site, s, o1[r]);
      if (p.red) {
#pragma unroll
        for (int i = 0; i < 24; ++i) nrm += (double)o1[r][i] * (double)o1[r][i];
      }
    }
  }
  if (FK != F_NONE) {
    __syncwarp();
    if (g < GT) {
#pragma unroll
      for (int r = 0; r < NR; ++r) tile_put(tile_row<R, LS>(tile, g, srow[r]), o1[r]);
    }
    __syncwarp();
    tile_chiral<R, LS, GT>(tile, lane, [&](R* xp, R* xm) {
      apply_f<R, LS, 0, FK>(k, xp);
      apply_f<R, LS, 1, FK>(k, xm);
    });
    __syncwarp();
    if (active) {
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        R o2[24];
        tile_get(tile_row<R, LS>(tile, g, srow[r]), o2);
        St::store(p.out2, vh, LS, site, srow[r], o2);
      }
    }
  }
  if (p.red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, off);
    if (lane == 0) red_warp[warp] = nrm;
    __syncthreads();
    if (tid == 0) {
      double b = 0.0;
#pragma unroll
      for (int w = 0; w < WARPS; ++w) b += red_warp[w];
      if (NR == 1) {
        p.red[blockIdx.x] = b;
      } else if (32 % LS == 0) {
        const int nb1 = (p.vh + WARPS * (32 / LS) - 1) / (WARPS * (32 / LS));
        p.red[2 * blockIdx.x] = b;
        if (2 * (int)blockIdx.x + 1 < nb1) p.red[2 * blockIdx.x + 1] = 0.0;
      } else {
        // Ls not dividing 32 (6, 12): the host reduces the one-slice kernel's
        // block count of partials, more than this grid has blocks; each block
        // writes its own and clears its share of the rest
        const int nb1 = (p.vh + WARPS * (32 / LS) - 1) / (WARPS * (32 / LS));
        p.red[blockIdx.x] = b;
        for (int j = (int)(gridDim.x + blockIdx.x); j < nb1; j += (int)gridDim.x) p.red[j] = 0.0;
      }
    }
  }
}

template <int LS, int P, int EPI, int FK>
__device__ __forceinline__ void hop_epilogue(const HopParams& p, const ChainCoef<typename Store<P>::R>& k,
                                             typename Store<P>::R* acc,
                                             typename Store<P>::R* tile, double* red_warp,
                                             int tid, int lane, int warp, int g, int s, int site,
                                             bool active) {
  using R = typename Store<P>::R;
  R (*rows)[24] = reinterpret_cast<R (*)[24]>(acc);
  const int srow[1] = {s};
  hop_epilogue_rows<LS, P, EPI, FK, 1, 32 / LS>(p, k, rows, tile, red_warp, tid, lane, warp, g, srow,
                                                site, active);
}

// Occupancy variants (minimum resident 128-thread blocks per SM requested from
// the register allocator); the plan's autotuner times both and keeps the faster.
template <int P> struct HopMinBlocks { static constexpr int v0 = 3, v1 = 4; };
template <> struct HopMinBlocks<PREC_F32> { static constexpr int v0 = 4, v1 = 6; };
template <> struct HopMinBlocks<PREC_F16> { static constexpr int v0 = 4, v1 = 6; };
template <> struct HopMinBlocks<PREC_BF16> { static constexpr int v0 = 4, v1 = 6; };

template <int LS, int P, int LF, int EPI, int FK, int MB>
__global__ void __launch_bounds__(128, MB)
dwf_hop_kernel(const HopParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  if (p.skip && *p.skip != 0.0) return;
  using St = Store<P>;
  using R = typename St::R;
  constexpr bool kDagHop = EpiIsDag<EPI>::v;
  constexpr bool kPh = LinkLoad<LF>::kFolded;
  constexpr int G = 32 / LS;              // sites per warp
  constexpr int WARPS = 4;
  constexpr bool kTile = (EPI != EPI_HALF) || (FK != F_NONE);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile_all = reinterpret_cast<R*>(smem_raw);        // WARPS * TileWarp
  __shared__ double red_warp[WARPS];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane / LS;
  const int s = lane - g * LS;
  const int site = p.site0 + (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.site_end);
  const size_t vh = p.vh;

  R acc[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) acc[i] = 0;

  if (active) {
    const int ix2 = site % p.nx2;
    const int iyzt = site / p.nx2;
    const int y = iyzt % p.ny;
    const int izt = iyzt / p.ny;
    const int z = izt % p.nz;
    const int t = izt / p.nz;
    const int keo = (p.ieo + y + z + t) & 1;
    const int x = 2 * ix2 + keo;
    const int nx = 2 * p.nx2;
    const int ieo = p.ieo;
    const size_t strideMu = vh;          // links: ((ieo + 2*mu)*Vh + site)

#define B200_HOP_DIR(MU, COORD, EXT, NBP, NBM)                                       \
    {                                                                                \
      R w[24], h[12], o[12], u[18];                                                  \
      {                                                                              \
        const R ph = (kPh || COORD != EXT - 1) ? R(1) : (R)p.bc[MU];                 \
        const int nb = NBP;                                                          \
        St::load(p.in, vh, LS, nb, s, w);                                            \
        if (kDagHop) {                                                               \
          _Pragma("unroll") for (int q = 0; q < 12; ++q) {                           \
            R tmp = w[q]; w[q] = w[q + 12]; w[q + 12] = tmp; }                       \
        }                                                                            \
        project<R, MU, 1, !kPh>(w, h);                                               \
        LinkLoad<LF>::load(p.links, (size_t)(ieo + 2 * MU) * strideMu + site, u);    \
        su3_mult_half<R, false>(u, h, o);                                            \
        reconstruct_acc<R, MU, 1, kPh>(acc, o, ph);                                  \
      }                                                                              \
      {                                                                              \
        const R ph = (kPh || COORD != 0) ? R(1) : (R)p.bc[MU];                       \
        const int nb = NBM;                                                          \
        St::load(p.in, vh, LS, nb, s, w);                                            \
        if (kDagHop) {                                                               \
          _Pragma("unroll") for (int q = 0; q < 12; ++q) {                           \
            R tmp = w[q]; w[q] = w[q + 12]; w[q + 12] = tmp; }                       \
        }                                                                            \
        project<R, MU, -1, !kPh>(w, h);                                              \
        LinkLoad<LF>::load(p.links, (size_t)(1 - ieo + 2 * MU) * strideMu + nb, u);  \
        su3_mult_half<R, true>(u, h, o);                                             \
        reconstruct_acc<R, MU, -1, kPh>(acc, o, ph);                                 \
      }                                                                              \
    }

    const int row = p.nx2 * iyzt;
    B200_HOP_DIR(0, x, nx,
                 row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo),
                 row + ((ix2 - 1 + keo < 0) ? p.nx2 - 1 : ix2 - 1 + keo));
    const int sy = p.nx2;
    B200_HOP_DIR(1, y, p.ny,
                 (y == p.ny - 1) ? site - (p.ny - 1) * sy : site + sy,
                 (y == 0) ? site + (p.ny - 1) * sy : site - sy);
    const int sz = p.nx2 * p.ny;
    B200_HOP_DIR(2, z, p.nz,
                 (z == p.nz - 1) ? site - (p.nz - 1) * sz : site + sz,
                 (z == 0) ? site + (p.nz - 1) * sz : site - sz);
    const int st = p.nx2 * p.ny * p.nz;
    B200_HOP_DIR(3, t, p.nt,
                 (t == p.nt - 1) ? site - (p.nt - 1) * st : site + st,
                 (t == 0) ? site + (p.nt - 1) * st : site - st);
#undef B200_HOP_DIR
  }

  hop_epilogue<LS, P, EPI, FK>(p, k, acc, tile_all + (size_t)warp * TileWarp<R, LS, G>::v, red_warp, tid, lane,
                               warp, g, s, site, active);
}

// ---------------------------------------------------------------------------
// Packed variant for FP32 arithmetic (f32, f16, bf16 storage).  One thread per
// (site, slice pair): slices s0 = j and s1 = j + Ls/2 undergo exactly the same
// operations (same links, same projections), so every value is held as a
// float2 (value at s0, value at s1) and the hop runs on Blackwell's packed
// FP32x2 instructions: the SU(3) products and the reconstruction issue half
// the instructions of the one-slice kernel, and each link is loaded and its
// third row rebuilt once per two slices.  The projection is done per slice in
// scalar code so that its outputs land directly in the packed pairs; the
// per-slice scale of f16/bf16 storage is applied to the projected pairs.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// out (half spinor pairs) = U h or U^+ h on both slices
template <bool kDag>
__device__ __forceinline__ void su3_mult_half2(const float* u, const float2* h, float2* o) {
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float2 re = make_float2(0.f, 0.f), im = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float ur = kDag ? u[2 * (i + 3 * j)] : u[2 * (j + 3 * i)];
        const float ui = kDag ? -u[2 * (i + 3 * j) + 1] : u[2 * (j + 3 * i) + 1];
        const float2 hr = h[6 * a + 2 * j], hi = h[6 * a + 2 * j + 1];
        re = __ffma2_rn(f2(ur), hr, re);
        re = __ffma2_rn(f2(-ui), hi, re);
        im = __ffma2_rn(f2(ur), hi, im);
        im = __ffma2_rn(f2(ui), hr, im);
      }
      o[6 * a + 2 * i] = re;
      o[6 * a + 2 * i + 1] = im;
    }
  }
}

// acc (pairs) += m * (1 - sign*gamma_mu)-shaped result, m a per-slice
// multiplier (the edge phase and, for f16/bf16 storage, the neighbour's
// per-(site, s) scale: U (sc h) = sc (U h), so the scale rides on the
// reconstruction's multiply-adds instead of costing its own multiplies);
// same algebra as reconstruct_acc, the factor i only selects the re/im pair.
template <int MU, int SIGN>
__device__ __forceinline__ void reconstruct_acc2(float2* acc, const float2* o, float2 m) {
  const float2 pp = m;
  const float2 sp = SIGN > 0 ? m : make_float2(-m.x, -m.y);
  const float2 sm = SIGN > 0 ? make_float2(-m.x, -m.y) : m;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float2 a0r = o[2 * c], a0i = o[2 * c + 1];
    const float2 a1r = o[6 + 2 * c], a1i = o[6 + 2 * c + 1];
    float2* r0 = acc + 2 * c;
    float2* r1 = acc + 2 * (c + 3);
    float2* r2 = acc + 2 * (c + 6);
    float2* r3 = acc + 2 * (c + 9);
    if (MU == 3) {
      if (SIGN > 0) {
        r2[0] = __ffma2_rn(pp, a0r, r2[0]); r2[1] = __ffma2_rn(pp, a0i, r2[1]);
        r3[0] = __ffma2_rn(pp, a1r, r3[0]); r3[1] = __ffma2_rn(pp, a1i, r3[1]);
      } else {
        r0[0] = __ffma2_rn(pp, a0r, r0[0]); r0[1] = __ffma2_rn(pp, a0i, r0[1]);
        r1[0] = __ffma2_rn(pp, a1r, r1[0]); r1[1] = __ffma2_rn(pp, a1i, r1[1]);
      }
      continue;
    }
    r0[0] = __ffma2_rn(pp, a0r, r0[0]); r0[1] = __ffma2_rn(pp, a0i, r0[1]);
    r1[0] = __ffma2_rn(pp, a1r, r1[0]); r1[1] = __ffma2_rn(pp, a1i, r1[1]);
    if (MU == 0) {        // rows 2,3 = -+ i h1, -+ i h0
      r2[0] = __ffma2_rn(sp, a1i, r2[0]); r2[1] = __ffma2_rn(sm, a1r, r2[1]);
      r3[0] = __ffma2_rn(sp, a0i, r3[0]); r3[1] = __ffma2_rn(sm, a0r, r3[1]);
    } else if (MU == 1) { // rows 2,3 = -+ h1, +- h0
      r2[0] = __ffma2_rn(sm, a1r, r2[0]); r2[1] = __ffma2_rn(sm, a1i, r2[1]);
      r3[0] = __ffma2_rn(sp, a0r, r3[0]); r3[1] = __ffma2_rn(sp, a0i, r3[1]);
    } else {              // MU==2: rows 2,3 = -+ i h0, +- i h1
      r2[0] = __ffma2_rn(sp, a0i, r2[0]); r2[1] = __ffma2_rn(sm, a0r, r2[1]);
      r3[0] = __ffma2_rn(sm, a1i, r3[0]); r3[1] = __ffma2_rn(sp, a1r, r3[1]);
    }
  }
}

template <int LS, int P, int LF, int EPI, int FK, int MB>
__global__ void __launch_bounds__(128, MB)
dwf_hop_pair_kernel(const HopParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  if (p.skip && *p.skip != 0.0) return;
  using St = Store<P>;
  using R = typename St::R;
  static_assert(sizeof(R) == 4, "packed kernel is for FP32 arithmetic");
  static_assert(LS % 2 == 0 && LS / 2 <= 32, "packed kernel: even Ls, at most 64");
  constexpr bool kDagHop = EpiIsDag<EPI>::v;
  constexpr bool kPh = LinkLoad<LF>::kFolded;
  constexpr int H = LS / 2;               // lanes per site
  constexpr int G = 32 / H;               // sites per warp
  constexpr int WARPS = 4;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile_all = reinterpret_cast<R*>(smem_raw);
  __shared__ double red_warp[WARPS];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane / H;
  const int j = lane - g * H;
  const int site = p.site0 + (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.site_end);
  const size_t vh = p.vh;
  const int s0 = j, s1 = j + H;

  float2 acc[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) acc[i] = make_float2(0.f, 0.f);

  if (active) {
    const int ix2 = site % p.nx2;
    const int iyzt = site / p.nx2;
    const int y = iyzt % p.ny;
    const int izt = iyzt / p.ny;
    const int z = izt % p.nz;
    const int t = izt / p.nz;
    const int keo = (p.ieo + y + z + t) & 1;
    const int x = 2 * ix2 + keo;
    const int nx = 2 * p.nx2;
    const int ieo = p.ieo;

#define B200_PAIR_HALF(MU, SIGN, NB, PH, LIDX)                                       \
    {                                                                                \
      float w0[24], w1[24], h0[12], h1[12], u[18];                                   \
      float sc0, sc1;                                                                \
      St::load_raw(p.in, vh, LS, NB, s0, w0, &sc0);                                  \
      St::load_raw(p.in, vh, LS, NB, s1, w1, &sc1);                                  \
      if (kDagHop) {                                                                 \
        _Pragma("unroll") for (int q = 0; q < 12; ++q) {                             \
          float t0 = w0[q]; w0[q] = w0[q + 12]; w0[q + 12] = t0;                     \
          float t1 = w1[q]; w1[q] = w1[q + 12]; w1[q + 12] = t1; }                   \
      }                                                                              \
      project<float, MU, SIGN, !kPh>(w0, h0);                                        \
      project<float, MU, SIGN, !kPh>(w1, h1);                                        \
      float2 h[12], o[12];                                                           \
      _Pragma("unroll") for (int q = 0; q < 12; ++q) h[q] = make_float2(h0[q], h1[q]); \
      const float2 mul = St::kScaled ? make_float2(sc0 * (PH), sc1 * (PH)) : f2(PH); \
      LinkLoad<LF>::load(p.links, LIDX, u);                                          \
      su3_mult_half2<(SIGN < 0)>(u, h, o);                                           \
      reconstruct_acc2<MU, SIGN>(acc, o, mul);                                       \
    }

#define B200_PAIR_DIR(MU, COORD, EXT, NBP, NBM)                                      \
    {                                                                                \
      const int nbp = NBP;                                                           \
      const float php = (kPh || COORD != EXT - 1) ? 1.f : (float)p.bc[MU];           \
      B200_PAIR_HALF(MU, 1, nbp, php, (size_t)(ieo + 2 * MU) * vh + site)            \
      const int nbm = NBM;                                                           \
      const float phm = (kPh || COORD != 0) ? 1.f : (float)p.bc[MU];                 \
      B200_PAIR_HALF(MU, -1, nbm, phm, (size_t)(1 - ieo + 2 * MU) * vh + nbm)        \
    }

    const int row = p.nx2 * iyzt;
    B200_PAIR_DIR(0, x, nx,
                  row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo),
                  row + ((ix2 - 1 + keo < 0) ? p.nx2 - 1 : ix2 - 1 + keo));
    const int sy = p.nx2;
    B200_PAIR_DIR(1, y, p.ny,
                  (y == p.ny - 1) ? site - (p.ny - 1) * sy : site + sy,
                  (y == 0) ? site + (p.ny - 1) * sy : site - sy);
    const int sz = p.nx2 * p.ny;
    B200_PAIR_DIR(2, z, p.nz,
                  (z == p.nz - 1) ? site - (p.nz - 1) * sz : site + sz,
                  (z == 0) ? site + (p.nz - 1) * sz : site - sz);
    const int st = p.nx2 * p.ny * p.nz;
    B200_PAIR_DIR(3, t, p.nt,
                  (t == p.nt - 1) ? site - (p.nt - 1) * st : site + st,
                  (t == 0) ? site + (p.nt - 1) * st : site - st);
#undef B200_PAIR_DIR
#undef B200_PAIR_HALF
  }

  float rows[2][24];
#pragma unroll
  for (int i = 0; i < 24; ++i) { rows[0][i] = acc[i].x; rows[1][i] = acc[i].y; }
  const int srow[2] = {s0, s1};
  hop_epilogue_rows<LS, P, EPI, FK, 2, G>(p, k, rows, tile_all + (size_t)warp * TileWarp<R, LS, G>::v,
                                          red_warp, tid, lane, warp, g, srow, site, active);
}

// Packed kernel for f16/bf16 storage with the next direction's raw data
// (two slices' stored chunks and scales, the link record) fetched into
// registers while the current direction is computed, so every warp keeps two
// directions of loads in flight.
template <int P>
struct PairRaw {
  uint4 c0[3], c1[3];   // stored chunks of slices s0 and s1
  float sc0, sc1;       // their scales
  uint4 l0, l1, l2;     // link record (LINK_F16_18: full 3x3, 18 halves, phase folded in)
};

template <int LS, int P>
__device__ __forceinline__ void pair_fetch(const HopParams& p, int nb, size_t lidx, int s0, int s1,
                                           PairRaw<P>& r) {
  using St = Store<P>;
  const unsigned char* colp = reinterpret_cast<const unsigned char*>(p.in) + (size_t)nb * St::col_bytes(LS);
  const uint4* c = reinterpret_cast<const uint4*>(colp);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r.c0[k] = __ldg(c + k * LS + s0);
    r.c1[k] = __ldg(c + k * LS + s1);
  }
  const float* scp = reinterpret_cast<const float*>(c + 3 * LS);
  r.sc0 = __ldg(scp + s0);
  r.sc1 = __ldg(scp + s1);
  const uint4* lp = reinterpret_cast<const uint4*>(p.links) + lidx * 3;
  r.l0 = __ldg(lp);
  r.l1 = __ldg(lp + 1);
  r.l2 = __ldg(lp + 2);
}

template <int P>
__device__ __forceinline__ void pair_decode(const uint4 (&c)[3], float* v) {
  using HO = HalfOps<typename Store<P>::Half>;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float2 a = HO::to2(c[k].x), b = HO::to2(c[k].y), d = HO::to2(c[k].z), e = HO::to2(c[k].w);
    v[8 * k + 0] = a.x; v[8 * k + 1] = a.y; v[8 * k + 2] = b.x; v[8 * k + 3] = b.y;
    v[8 * k + 4] = d.x; v[8 * k + 5] = d.y; v[8 * k + 6] = e.x; v[8 * k + 7] = e.y;
  }
}

// The Dirac-basis projection (1 - sign*gamma_mu) of project(), applied to the
// stored (re, im) half-precision pairs before any conversion to FP32: each
// projected colour is one paired multiply-add, h = w_a + f * w_b or
// w_a + f * swap(w_b) with f = (+-1, +-1), so a slice converts 6 pairs instead
// of 12 and issues 6 paired operations instead of 12 FP32 adds.  The rounding
// this adds is that of the storage format itself.  w[c + 3*spin],
// h[c + 3*a]; t projection without its factor 2 (folded into the links).
template <typename H2> struct Half2Ops;
template <> struct Half2Ops<__half2> {
  __device__ static __half2 k(float a, float b) { return __floats2half2_rn(a, b); }
  __device__ static float2 f2(__half2 h) { return __half22float2(h); }
};
template <> struct Half2Ops<__nv_bfloat162> {
  __device__ static __nv_bfloat162 k(float a, float b) { return __floats2bfloat162_rn(a, b); }
  __device__ static float2 f2(__nv_bfloat162 h) { return __bfloat1622float2(h); }
};

template <typename H2, int MU, int SIGN>
__device__ __forceinline__ void project_half2(const H2* w, H2* h) {
  using O = Half2Ops<H2>;
  constexpr float S = SIGN > 0 ? 1.f : -1.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const H2 w0 = w[c], w1 = w[c + 3], w2 = w[c + 6], w3 = w[c + 9];
    H2 h0, h1;
    if (MU == 0) {        // h0 = w0 -+ i w3, h1 = w1 -+ i w2 (as project)
      h0 = __hfma2(__lowhigh2highlow(w3), O::k(-S, S), w0);
      h1 = __hfma2(__lowhigh2highlow(w2), O::k(-S, S), w1);
    } else if (MU == 1) { // h0 = w0 +- w3, h1 = w1 -+ w2
      h0 = __hfma2(w3, O::k(S, S), w0);
      h1 = __hfma2(w2, O::k(-S, -S), w1);
    } else if (MU == 2) { // h0 = w0 -+ i w2, h1 = w1 +- i w3
      h0 = __hfma2(__lowhigh2highlow(w2), O::k(-S, S), w0);
      h1 = __hfma2(__lowhigh2highlow(w3), O::k(S, -S), w1);
    } else {              // (1 - g4) keeps the lower spins, (1 + g4) the upper
      h0 = SIGN > 0 ? w2 : w0;
      h1 = SIGN > 0 ? w3 : w1;
    }
    h[c] = h0;
    h[c + 3] = h1;
  }
}

template <int P> struct Half2Of;
template <> struct Half2Of<PREC_F16> { using T = __half2; };
template <> struct Half2Of<PREC_BF16> { using T = __nv_bfloat162; };

// the 12 stored pairs of one slice (three 16-byte chunks), spins swapped for
// the gamma5-sandwiched dagger hop
template <int P, bool kDagHop>
__device__ __forceinline__ void pair_unpack(const uint4 (&c)[3], typename Half2Of<P>::T* w) {
  using H2 = typename Half2Of<P>::T;
  unsigned int u[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[4 * k] = c[k].x; u[4 * k + 1] = c[k].y; u[4 * k + 2] = c[k].z; u[4 * k + 3] = c[k].w;
  }
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const unsigned int v = kDagHop ? u[(q + 6) % 12] : u[q];
    w[q] = *reinterpret_cast<const H2*>(&v);
  }
}

template <int P, int MU, int SIGN, bool kDagHop>
__device__ __forceinline__ void pair_compute(const PairRaw<P>& r, float ph, float2* acc) {
  using H2 = typename Half2Of<P>::T;
  using O = Half2Ops<H2>;
  float u[18];
  H2 w0[12], w1[12], p0[6], p1[6];
  pair_unpack<P, kDagHop>(r.c0, w0);
  pair_unpack<P, kDagHop>(r.c1, w1);
  project_half2<H2, MU, SIGN>(w0, p0);
  project_half2<H2, MU, SIGN>(w1, p1);
  float2 h[12], o[12];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const float2 a = O::f2(p0[q]), b = O::f2(p1[q]);
    h[2 * q] = make_float2(a.x, b.x);
    h[2 * q + 1] = make_float2(a.y, b.y);
  }
  LinkLoad<LINK_F16_18>::decode(r.l0, r.l1, r.l2, u);
  su3_mult_half2<(SIGN < 0)>(u, h, o);
  reconstruct_acc2<MU, SIGN>(acc, o, make_float2(r.sc0 * ph, r.sc1 * ph));
}

template <int LS, int P, int EPI, int FK, int MB>
__global__ void __launch_bounds__(128, MB)
dwf_hop_pair_pf_kernel(const HopParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  if (p.skip && *p.skip != 0.0) return;
  using St = Store<P>;
  using R = typename St::R;
  static_assert(St::kScaled, "prefetching packed kernel is for f16/bf16 storage");
  static_assert(LS % 2 == 0 && LS / 2 <= 32, "packed kernel: even Ls, at most 64");
  constexpr bool kDagHop = EpiIsDag<EPI>::v;
  constexpr int H = LS / 2;
  constexpr int G = 32 / H;
  constexpr int WARPS = 4;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile_all = reinterpret_cast<R*>(smem_raw);
  __shared__ double red_warp[WARPS];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane / H;
  const int j = lane - g * H;
  const int site = p.site0 + (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.site_end);
  const size_t vh = p.vh;
  const int s0 = j, s1 = j + H;

  float2 acc[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) acc[i] = make_float2(0.f, 0.f);

  if (active) {
    const int ix2 = site % p.nx2;
    const int iyzt = site / p.nx2;
    const int y = iyzt % p.ny;
    const int izt = iyzt / p.ny;
    const int z = izt % p.nz;
    const int t = izt / p.nz;
    const int keo = (p.ieo + y + z + t) & 1;
    const int x = 2 * ix2 + keo;
    const int ieo = p.ieo;
    int nb[8];
    float ph[8];
    const int row = p.nx2 * iyzt;
    nb[0] = row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo);
    nb[1] = row + ((ix2 - 1 + keo < 0) ? p.nx2 - 1 : ix2 - 1 + keo);
    ph[0] = 1.f;
    ph[1] = 1.f;
    const int sy = p.nx2, sz = p.nx2 * p.ny, st4 = p.nx2 * p.ny * p.nz;
    nb[2] = (y == p.ny - 1) ? site - (p.ny - 1) * sy : site + sy;
    nb[3] = (y == 0) ? site + (p.ny - 1) * sy : site - sy;
    ph[2] = 1.f;
    ph[3] = 1.f;
    nb[4] = (z == p.nz - 1) ? site - (p.nz - 1) * sz : site + sz;
    nb[5] = (z == 0) ? site + (p.nz - 1) * sz : site - sz;
    ph[4] = 1.f;
    ph[5] = 1.f;
    nb[6] = (t == p.nt - 1) ? site - (p.nt - 1) * st4 : site + st4;
    nb[7] = (t == 0) ? site + (p.nt - 1) * st4 : site - st4;
    ph[6] = 1.f;
    ph[7] = 1.f;
    auto lidx = [&](int d) -> size_t {
      const int mu = d >> 1;
      return (d & 1) ? (size_t)(1 - ieo + 2 * mu) * vh + nb[d] : (size_t)(ieo + 2 * mu) * vh + site;
    };
    PairRaw<P> ra, rb;
    pair_fetch<LS, P>(p, nb[0], lidx(0), s0, s1, ra);
#define B200_PF_STEP(D, MU, SIGN, CUR, NXT)                                          \
    if ((D) < 7) pair_fetch<LS, P>(p, nb[(D) + 1], lidx((D) + 1), s0, s1, NXT);      \
    pair_compute<P, MU, SIGN, kDagHop>(CUR, ph[D], acc);
    B200_PF_STEP(0, 0, 1, ra, rb)
    B200_PF_STEP(1, 0, -1, rb, ra)
    B200_PF_STEP(2, 1, 1, ra, rb)
    B200_PF_STEP(3, 1, -1, rb, ra)
    B200_PF_STEP(4, 2, 1, ra, rb)
    B200_PF_STEP(5, 2, -1, rb, ra)
    B200_PF_STEP(6, 3, 1, ra, rb)
    B200_PF_STEP(7, 3, -1, rb, ra)
#undef B200_PF_STEP
  }

  float rows[2][24];
#pragma unroll
  for (int i = 0; i < 24; ++i) { rows[0][i] = acc[i].x; rows[1][i] = acc[i].y; }
  const int srow[2] = {s0, s1};
  hop_epilogue_rows<LS, P, EPI, FK, 2, G>(p, k, rows, tile_all + (size_t)warp * TileWarp<R, LS, G>::v,
                                          red_warp, tid, lane, warp, g, srow, site, active);
}

template <int LS, int P>
constexpr size_t hop_pair_smem_bytes() {
  using R = typename Store<P>::R;
  return sizeof(R) * (4 * TileWarp<R, LS, 64 / LS>::v);
}

// Blocks of the packed kernel: 4 warps of 64/Ls sites each.
inline int hop_pair_grid(int ls, int vh) {
  const int per_block = 4 * (64 / ls);
  return (vh + per_block - 1) / per_block;
}

// ---------------------------------------------------------------------------
// TMA-staged variant.  Each warp keeps an S-deep pipeline over the 8 hop
// directions: for every one of its G sites the lane with s == 0 issues two
// bulk asynchronous copies per direction -- the neighbour site's whole
// fifth-dimension column (site-major field layout) and the link -- into the
// warp's shared-memory stage, completing on that stage's mbarrier.  While
// direction d is computed from shared memory, directions d+1..d+S-1 are in
// flight, without holding registers.  Stage buffers are reused after the
// warp's lanes have finished reading them (__syncwarp + proxy fence).
// All waits are bounded; on timeout the kernel sets p.err and skips its work.
// After a failed wait: wait for the stages this warp issued but has not seen
// complete (directions ndone .. nissued-1), each with the drain bound; if even
// that runs out, the error word says so (2).
template <int S>
__device__ __forceinline__ void drain_copies(uint64_t* bars, int ndone, int nissued, int lane, int* err) {
  bool all = true;
  for (int d = ndone; d < nissued; ++d)
    all = mbar_wait_drain(smem_u32(&bars[d % S]), (d / S) & 1) && all;
  if (!__all_sync(0xffffffffu, all) && lane == 0 && err) atomicExch(err, 2);
}

template <int LS, int P, int LF, int GS = 32 / LS> struct TmaGeom {
  static constexpr int G = GS;              // sites per warp
  static constexpr int COL = (int)Store<P>::col_bytes(LS);
  static constexpr int LNK = LinkLoad<LF>::kChunks * 16;
  static constexpr int SLOT = COL + LNK;                       // one site, one direction
  template <int S> static constexpr int warp_bytes() {
    // stages, and the epilogue tile (reuses the stage area)
    using R = typename Store<P>::R;
    return (S * G * SLOT > TileWarp<R, LS, G>::v * (int)sizeof(R))
               ? S * G * SLOT
               : TileWarp<R, LS, G>::v * (int)sizeof(R);
  }
};

template <int LS, int P, int LF, int EPI, int FK, int S, int MB>
__global__ void __launch_bounds__(128, MB)
dwf_hop_tma_kernel(const HopParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  if (p.skip && *p.skip != 0.0) return;
  using St = Store<P>;
  using R = typename St::R;
  using TG = TmaGeom<LS, P, LF>;
  constexpr bool kDagHop = EpiIsDag<EPI>::v;
  constexpr bool kPh = LinkLoad<LF>::kFolded;
  constexpr int NPH = kPh ? 1 : 8;        // edge phases kept in registers
  constexpr int G = TG::G;
  constexpr int WARPS = 4;
  constexpr int WB = TG::template warp_bytes<S>();
  constexpr int WBA = (WB + 127) / 128 * 128;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ double red_warp[WARPS];
  __shared__ __align__(8) uint64_t bars[WARPS][S];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane / LS;
  const int s = lane - g * LS;
  const int site = p.site0 + (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.site_end);
  const bool issuer = (g < G) && (s == 0);
  unsigned char* wbase = smem_raw + (size_t)warp * WBA;
  const size_t vh = p.vh;

  if (lane == 0) {
#pragma unroll
    for (int st = 0; st < S; ++st) mbar_init(smem_u32(&bars[warp][st]), G);
    mbar_fence_init();
  }
  __syncwarp();

  // neighbour sites and edge phases of the 8 directions (x+, x-, y+, ..., t-)
  int nb[8];
  R ph[NPH];
#pragma unroll
  for (int d = 0; d < NPH; ++d) ph[d] = R(1);
  if (active) {
    const int ix2 = site % p.nx2;
    const int iyzt = site / p.nx2;
    const int y = iyzt % p.ny;
    const int izt = iyzt / p.ny;
    const int z = izt % p.nz;
    const int t = izt / p.nz;
    const int keo = (p.ieo + y + z + t) & 1;
    const int x = 2 * ix2 + keo;
    const int row = p.nx2 * iyzt;
    nb[0] = row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo);
    nb[1] = row + ((ix2 - 1 + keo < 0) ? p.nx2 - 1 : ix2 - 1 + keo);
    const int sy = p.nx2, sz = p.nx2 * p.ny, st4 = p.nx2 * p.ny * p.nz;
    nb[2] = (y == p.ny - 1) ? site - (p.ny - 1) * sy : site + sy;
    nb[3] = (y == 0) ? site + (p.ny - 1) * sy : site - sy;
    nb[4] = (z == p.nz - 1) ? site - (p.nz - 1) * sz : site + sz;
    nb[5] = (z == 0) ? site + (p.nz - 1) * sz : site - sz;
    nb[6] = (t == p.nt - 1) ? site - (p.nt - 1) * st4 : site + st4;
    nb[7] = (t == 0) ? site + (p.nt - 1) * st4 : site - st4;
    if constexpr (!kPh) {
      ph[0 % NPH] = (x == 2 * p.nx2 - 1) ? (R)p.bc[0] : R(1);
      ph[1 % NPH] = (x == 0) ? (R)p.bc[0] : R(1);
      ph[2 % NPH] = (y == p.ny - 1) ? (R)p.bc[1] : R(1);
      ph[3 % NPH] = (y == 0) ? (R)p.bc[1] : R(1);
      ph[4 % NPH] = (z == p.nz - 1) ? (R)p.bc[2] : R(1);
      ph[5 % NPH] = (z == 0) ? (R)p.bc[2] : R(1);
      ph[6 % NPH] = (t == p.nt - 1) ? (R)p.bc[3] : R(1);
      ph[7 % NPH] = (t == 0) ? (R)p.bc[3] : R(1);
    }
  } else {
#pragma unroll
    for (int d = 0; d < 8; ++d) nb[d] = 0;
  }

  auto col_ptr = [&](int st) { return wbase + (size_t)(st * G + g) * TG::SLOT; };
  int nissued = 0;   // directions issued by this warp (uniform across its lanes)
  auto issue = [&](int d, int st) {
    ++nissued;
    if (!issuer) return;
    const uint32_t bar = smem_u32(&bars[warp][st]);
    if (!active) { mbar_arrive(bar); return; }
    const int mu = d >> 1;
    const bool fwd = (d & 1) == 0;
    const size_t lidx = fwd ? (size_t)(p.ieo + 2 * mu) * vh + site : (size_t)(1 - p.ieo + 2 * mu) * vh + nb[d];
    unsigned char* dst = col_ptr(st);
    mbar_arrive_expect_tx(bar, TG::SLOT);
    bulk_g2s(smem_u32(dst), reinterpret_cast<const unsigned char*>(p.in) + (size_t)nb[d] * TG::COL,
             TG::COL, bar);
    bulk_g2s(smem_u32(dst + TG::COL), reinterpret_cast<const unsigned char*>(p.links) + lidx * TG::LNK,
             TG::LNK, bar);
  };

#pragma unroll
  for (int d = 0; d < S; ++d) issue(d, d);

  R acc[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) acc[i] = 0;
  bool ok = true;
  int ndone = 0;     // directions whose copies this warp has seen complete

#define B200_TMA_STEP(D, MU, SIGN)                                                   \
  {                                                                                  \
    constexpr int st = (D) % S;                                                      \
    const uint32_t parity = ((D) / S) & 1;                                           \
    if (ok) {                                                                        \
      const bool got = ((D) != p.fail_dir) &&                                      \
                       mbar_wait_bounded(smem_u32(&bars[warp][st]), parity, p.wait_ns); \
      ok = __all_sync(0xffffffffu, got);                                             \
      if (ok) ndone = (D) + 1;                                                       \
      else if (lane == 0 && p.err) atomicExch(p.err, 1);                             \
    }                                                                                \
    if (ok && active) {                                                              \
      R w[24], h[12], o[12], u[18];                                                  \
      const unsigned char* c = col_ptr(st);                                          \
      St::load_col(c, LS, s, w);                                                     \
      if (kDagHop) {                                                                 \
        _Pragma("unroll") for (int q = 0; q < 12; ++q) {                             \
          R tmp = w[q]; w[q] = w[q + 12]; w[q + 12] = tmp; }                         \
      }                                                                              \
      project<R, MU, SIGN, !kPh>(w, h);                                              \
      if constexpr (LF == LINK_F64_18) {                                             \
        hop_dir_rows_f64<MU, SIGN>(reinterpret_cast<const double2*>(c + TG::COL),    \
                                   reinterpret_cast<const double*>(h),               \
                                   reinterpret_cast<double*>(acc));                  \
      } else {                                                                       \
        LinkLoad<LF>::load_plain(c + TG::COL, u);                                    \
        su3_mult_half<R, (SIGN < 0)>(u, h, o);                                       \
        reconstruct_acc<R, MU, SIGN, kPh>(acc, o, ph[(D) % NPH]);                    \
      }                                                                              \
    }                                                                                \
    __syncwarp();                                                                    \
    if ((D) + S < 8 && ok) {                                                         \
      fence_proxy_async_smem();                                                      \
      issue((D) + S, st);                                                            \
    }                                                                                \
  }

  B200_TMA_STEP(0, 0, 1)
  B200_TMA_STEP(1, 0, -1)
  B200_TMA_STEP(2, 1, 1)
  B200_TMA_STEP(3, 1, -1)
  B200_TMA_STEP(4, 2, 1)
  B200_TMA_STEP(5, 2, -1)
  B200_TMA_STEP(6, 3, 1)
  B200_TMA_STEP(7, 3, -1)
#undef B200_TMA_STEP

  // A warp that gave up waits for the copies it still has in flight (with a
  // bound far longer than the first wait's, so that no bulk copy is left
  // writing into shared memory when the CTA exits), then the whole CTA
  // returns without touching its outputs; the host sees p.err.
  if (!ok) drain_copies<S>(&bars[warp][0], ndone, nissued, lane, p.err);
  if (!__syncthreads_and(ok ? 1 : 0)) return;
  hop_epilogue<LS, P, EPI, FK>(p, k, acc, reinterpret_cast<R*>(wbase), red_warp, tid, lane, warp, g, s,
                               site, active);
}

// TMA-staged packed kernel: the bulk-copy pipeline of dwf_hop_tma_kernel
// (neighbour column + link per site and direction, S-deep per warp, bounded
// mbarrier waits, device error word on timeout) feeding the two-slice FP32x2
// arithmetic of dwf_hop_pair_kernel.  64/Ls sites per warp.
template <int LS, int P, int LF, int EPI, int FK, int S, int MB>
__global__ void __launch_bounds__(128, MB)
dwf_hop_tma_pair_kernel(const HopParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  if (p.skip && *p.skip != 0.0) return;
  using St = Store<P>;
  using R = typename St::R;
  static_assert(sizeof(R) == 4, "packed kernel is for FP32 arithmetic");
  static_assert(LS % 2 == 0 && LS / 2 <= 32, "packed kernel: even Ls, at most 64");
  constexpr int H = LS / 2;
  constexpr int G = 32 / H;
  using TG = TmaGeom<LS, P, LF, G>;
  constexpr bool kDagHop = EpiIsDag<EPI>::v;
  constexpr bool kPh = LinkLoad<LF>::kFolded;
  constexpr int WARPS = 4;
  constexpr int WB = TG::template warp_bytes<S>();
  constexpr int WBA = (WB + 127) / 128 * 128;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ double red_warp[WARPS];
  __shared__ __align__(8) uint64_t bars[WARPS][S];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane / H;
  const int j = lane - g * H;
  const int site = p.site0 + (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.site_end);
  const bool issuer = (g < G) && (j == 0);
  unsigned char* wbase = smem_raw + (size_t)warp * WBA;
  const size_t vh = p.vh;
  const int s0 = j, s1 = j + H;

  if (lane == 0) {
#pragma unroll
    for (int st = 0; st < S; ++st) mbar_init(smem_u32(&bars[warp][st]), G);
    mbar_fence_init();
  }
  __syncwarp();

  int nb[8];
  float ph[8];
  if (active) {
    const int ix2 = site % p.nx2;
    const int iyzt = site / p.nx2;
    const int y = iyzt % p.ny;
    const int izt = iyzt / p.ny;
    const int z = izt % p.nz;
    const int t = izt / p.nz;
    const int keo = (p.ieo + y + z + t) & 1;
    const int x = 2 * ix2 + keo;
    const int row = p.nx2 * iyzt;
    nb[0] = row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo);
    nb[1] = row + ((ix2 - 1 + keo < 0) ? p.nx2 - 1 : ix2 - 1 + keo);
    ph[0] = (!kPh && (x == 2 * p.nx2 - 1)) ? (float)p.bc[0] : 1.f;
    ph[1] = (!kPh && (x == 0)) ? (float)p.bc[0] : 1.f;
    const int sy = p.nx2, sz = p.nx2 * p.ny, st4 = p.nx2 * p.ny * p.nz;
    nb[2] = (y == p.ny - 1) ? site - (p.ny - 1) * sy : site + sy;
    nb[3] = (y == 0) ? site + (p.ny - 1) * sy : site - sy;
    ph[2] = (!kPh && (y == p.ny - 1)) ? (float)p.bc[1] : 1.f;
    ph[3] = (!kPh && (y == 0)) ? (float)p.bc[1] : 1.f;
    nb[4] = (z == p.nz - 1) ? site - (p.nz - 1) * sz : site + sz;
    nb[5] = (z == 0) ? site + (p.nz - 1) * sz : site - sz;
    ph[4] = (!kPh && (z == p.nz - 1)) ? (float)p.bc[2] : 1.f;
    ph[5] = (!kPh && (z == 0)) ? (float)p.bc[2] : 1.f;
    nb[6] = (t == p.nt - 1) ? site - (p.nt - 1) * st4 : site + st4;
    nb[7] = (t == 0) ? site + (p.nt - 1) * st4 : site - st4;
    ph[6] = (!kPh && (t == p.nt - 1)) ? (float)p.bc[3] : 1.f;
    ph[7] = (!kPh && (t == 0)) ? (float)p.bc[3] : 1.f;
  } else {
#pragma unroll
    for (int d = 0; d < 8; ++d) { nb[d] = 0; ph[d] = 0.f; }
  }

  auto col_ptr = [&](int st) { return wbase + (size_t)(st * G + g) * TG::SLOT; };
  int nissued = 0;
  auto issue = [&](int d, int st) {
    ++nissued;
    if (!issuer) return;
    const uint32_t bar = smem_u32(&bars[warp][st]);
    if (!active) { mbar_arrive(bar); return; }
    const int mu = d >> 1;
    const bool fwd = (d & 1) == 0;
    const size_t lidx = fwd ? (size_t)(p.ieo + 2 * mu) * vh + site : (size_t)(1 - p.ieo + 2 * mu) * vh + nb[d];
    unsigned char* dst = col_ptr(st);
    mbar_arrive_expect_tx(bar, TG::SLOT);
    bulk_g2s(smem_u32(dst), reinterpret_cast<const unsigned char*>(p.in) + (size_t)nb[d] * TG::COL,
             TG::COL, bar);
    bulk_g2s(smem_u32(dst + TG::COL), reinterpret_cast<const unsigned char*>(p.links) + lidx * TG::LNK,
             TG::LNK, bar);
  };

#pragma unroll
  for (int d = 0; d < S; ++d) issue(d, d);

  float2 acc[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) acc[i] = make_float2(0.f, 0.f);
  bool ok = true;
  int ndone = 0;

#define B200_TMAP_STEP(D, MU, SIGN)                                                  \
  {                                                                                  \
    constexpr int st = (D) % S;                                                      \
    const uint32_t parity = ((D) / S) & 1;                                           \
    if (ok) {                                                                        \
      const bool got = ((D) != p.fail_dir) &&                                      \
                       mbar_wait_bounded(smem_u32(&bars[warp][st]), parity, p.wait_ns); \
      ok = __all_sync(0xffffffffu, got);                                             \
      if (ok) ndone = (D) + 1;                                                       \
      else if (lane == 0 && p.err) atomicExch(p.err, 1);                             \
    }                                                                                \
    if (ok && active) {                                                              \
      float w0[24], w1[24], h0[12], h1[12], u[18];                                   \
      float sc0, sc1;                                                                \
      const unsigned char* c = col_ptr(st);                                          \
      St::load_col_raw(c, LS, s0, w0, &sc0);                                         \
      St::load_col_raw(c, LS, s1, w1, &sc1);                                         \
      if (kDagHop) {                                                                 \
        _Pragma("unroll") for (int q = 0; q < 12; ++q) {                             \
          float t0 = w0[q]; w0[q] = w0[q + 12]; w0[q + 12] = t0;                     \
          float t1 = w1[q]; w1[q] = w1[q + 12]; w1[q + 12] = t1; }                   \
      }                                                                              \
      project<float, MU, SIGN, !kPh>(w0, h0);                                        \
      project<float, MU, SIGN, !kPh>(w1, h1);                                        \
      float2 h[12], o[12];                                                           \
      _Pragma("unroll") for (int q = 0; q < 12; ++q) h[q] = make_float2(h0[q], h1[q]); \
      const float2 mul = St::kScaled ? make_float2(sc0 * ph[D], sc1 * ph[D]) : f2(ph[D]); \
      LinkLoad<LF>::load_plain(c + TG::COL, u);                                      \
      su3_mult_half2<(SIGN < 0)>(u, h, o);                                           \
      reconstruct_acc2<MU, SIGN>(acc, o, mul);                                       \
    }                                                                                \
    __syncwarp();                                                                    \
    if ((D) + S < 8 && ok) {                                                         \
      fence_proxy_async_smem();                                                      \
      issue((D) + S, st);                                                            \
    }                                                                                \
  }

  B200_TMAP_STEP(0, 0, 1)
  B200_TMAP_STEP(1, 0, -1)
  B200_TMAP_STEP(2, 1, 1)
  B200_TMAP_STEP(3, 1, -1)
  B200_TMAP_STEP(4, 2, 1)
  B200_TMAP_STEP(5, 2, -1)
  B200_TMAP_STEP(6, 3, 1)
  B200_TMAP_STEP(7, 3, -1)
#undef B200_TMAP_STEP

  if (!ok) drain_copies<S>(&bars[warp][0], ndone, nissued, lane, p.err);
  if (!__syncthreads_and(ok ? 1 : 0)) return;
  float rows[2][24];
#pragma unroll
  for (int i = 0; i < 24; ++i) { rows[0][i] = acc[i].x; rows[1][i] = acc[i].y; }
  const int srow[2] = {s0, s1};
  hop_epilogue_rows<LS, P, EPI, FK, 2, G>(p, k, rows, reinterpret_cast<R*>(wbase), red_warp, tid, lane,
                                          warp, g, srow, site, active);
}

template <int LS, int P, int LF, int S>
constexpr size_t hop_tma_pair_smem_bytes() {
  return (size_t)4 * ((TmaGeom<LS, P, LF, 64 / LS>::template warp_bytes<S>() + 127) / 128 * 128);
}

template <int LS, int P, int LF, int S>
constexpr size_t hop_tma_smem_bytes() {
  return (size_t)4 * ((TmaGeom<LS, P, LF>::template warp_bytes<S>() + 127) / 128 * 128);
}

template <int LS, int P>
constexpr size_t hop_smem_bytes() {
  using R = typename Store<P>::R;
  return sizeof(R) * (4 * TileWarp<R, LS, 32 / LS>::v);
}

}  // namespace b200
