// Learned gauge-covariant preconditioner N(r) ~ (D^+D)^-1 r for the even/odd
// domain-wall system: a 3-layer linear 5D convolution network whose layers
// mix channels with complex weights (never color) and move data between sites
// only by parallel transport with the gauge links, so N commutes with gauge
// transformations.  Channels 4 -> H -> 4 per color (the 4 input channels are
// the spins of the residual); each layer has 11 paths (identity, s+-1 with
// open ends, and the 8 link-transported 4D hops).  The residual lives on one
// parity (even); layers 1-2 produce both parities, layer 3 only the even one,
// so the network reaches 3 hops in 4D and 3 slices in s.
//
// The deployed weights are the FP32 master weights rounded to BF16 (held as
// FP32 values that BF16 represents exactly); every kernel accumulates in
// FP32.  Training runs entirely in these kernels: forward, the loss
// L = |A (N r - e)|^2 / |r|^2 on a pair with A e = r (A = DdagD applied by
// the operator's own FP32 kernels; measuring the error in the residual norm
// makes A N ~ 1 on every mode, which is what a Krylov solver needs -- the
// plain error norm lets N neglect the high modes, and the flexible solver
// then stagnates on them), backward through the layers, weight gradients as
// site-reduced outer products, and Adam on the FP32 master copy.  The
// network has no counterpart in the reference; it plugs in where its solver
// framework takes a preconditioner
// (APrecond<AFIELD>::mult, src/lib_alt/Solver/aprecond.h:28-47) and is used by
// the flexible CG in dwf_plan.cu.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/b200dwf.h"
#include "dwf_hop.cuh"
#include "learned.h"
#include "umma.cuh"

namespace b200 {

void set_last_error(int code, const char* fmt, ...);

namespace {

// ------------------------------------------------------------ device helpers
template <int C>
__device__ __forceinline__ void lp_load(const float4* base, int ls, int site, int s,
                                        float2 (&v)[C][3]) {
  constexpr int K = 3 * C / 2;
  const float4* col = base + (size_t)site * K * ls + s;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float4 c = __ldg(col + (size_t)k * ls);
    v[(2 * k) / 3][(2 * k) % 3] = make_float2(c.x, c.y);
    v[(2 * k + 1) / 3][(2 * k + 1) % 3] = make_float2(c.z, c.w);
  }
}

template <int C>
__device__ __forceinline__ void lp_store(float4* base, int ls, int site, int s,
                                         const float2 (&v)[C][3]) {
  constexpr int K = 3 * C / 2;
  float4* col = base + (size_t)site * K * ls + s;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float2 a = v[(2 * k) / 3][(2 * k) % 3];
    const float2 b = v[(2 * k + 1) / 3][(2 * k + 1) % 3];
    col[(size_t)k * ls] = make_float4(a.x, a.y, b.x, b.y);
  }
}

template <int C>
__device__ __forceinline__ void lp_zero(float2 (&v)[C][3]) {
#pragma unroll
  for (int b = 0; b < C; ++b)
#pragma unroll
    for (int c = 0; c < 3; ++c) v[b][c] = make_float2(0.f, 0.f);
}

// o[b] = ph * U v[b] (DAG = false) or ph * U^+ v[b] (DAG = true) on every channel.
template <int C, bool DAG>
__device__ __forceinline__ void lp_transport(const float* u, float ph, const float2 (&v)[C][3],
                                             float2 (&o)[C][3]) {
#pragma unroll
  for (int b = 0; b < C; ++b)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float ur = DAG ? u[2 * (i + 3 * j)] : u[2 * (j + 3 * i)];
        const float ui = DAG ? -u[2 * (i + 3 * j) + 1] : u[2 * (j + 3 * i) + 1];
        re = fmaf(ur, v[b][j].x, re); re = fmaf(-ui, v[b][j].y, re);
        im = fmaf(ur, v[b][j].y, im); im = fmaf(ui, v[b][j].x, im);
      }
      o[b][i] = make_float2(ph * re, ph * im);
    }
}

// Neighbour of (site, parity ieo) in direction mu (fwd: +mu), the boundary
// phase of that hop and the index of the link record it uses -- the hop
// kernel's conventions (dwf_hop.cuh).
template <typename PP>
__device__ __forceinline__ void lp_neighbour(const PP& p, int site, int mu, bool fwd, int* nb,
                                             float* ph, size_t* lidx) {
  const int ix2 = site % p.nx2;
  const int iyzt = site / p.nx2;
  const int y = iyzt % p.ny;
  const int izt = iyzt / p.ny;
  const int z = izt % p.nz;
  const int t = izt / p.nz;
  const int keo = (p.ieo + y + z + t) & 1;
  const int x = 2 * ix2 + keo;
  int coord, ext, stride = 0;
  if (mu == 0) {
    const int row = p.nx2 * iyzt;
    *nb = fwd ? row + ((ix2 + keo == p.nx2) ? 0 : ix2 + keo)
              : row + ((ix2 - 1 + keo < 0) ? p.nx2 - 1 : ix2 - 1 + keo);
    coord = x; ext = 2 * p.nx2;
  } else {
    if (mu == 1) { coord = y; ext = p.ny; stride = p.nx2; }
    else if (mu == 2) { coord = z; ext = p.nz; stride = p.nx2 * p.ny; }
    else { coord = t; ext = p.nt; stride = p.nx2 * p.ny * p.nz; }
    *nb = fwd ? ((coord == ext - 1) ? site - (ext - 1) * stride : site + stride)
              : ((coord == 0) ? site + (ext - 1) * stride : site - stride);
  }
  *ph = (fwd ? (coord == ext - 1) : (coord == 0)) ? p.bc[mu] : 1.f;
  *lidx = fwd ? (size_t)(p.ieo + 2 * mu) * p.vh + site : (size_t)(1 - p.ieo + 2 * mu) * p.vh + *nb;
}

// Transported input of one path at (site, s); zero where the path leaves the
// fifth dimension or the input is absent.
template <int C, typename PP>
__device__ __forceinline__ void lp_path_input(const PP& p, const float4* in_same,
                                              const float4* in_other, int path, int site, int s,
                                              float2 (&u)[C][3]) {
  if (path < 3) {
    const int ss = (path == 0) ? s : (path == 1 ? s + 1 : s - 1);
    if (in_same && ss >= 0 && ss < p.ls) lp_load<C>(in_same, p.ls, site, ss, u);
    else lp_zero<C>(u);
    return;
  }
  if (!in_other) { lp_zero<C>(u); return; }
  const int d = path - 3;
  const int mu = d >> 1;
  const bool fwd = (d & 1) == 0;
  int nb; float ph; size_t lidx;
  lp_neighbour(p, site, mu, fwd, &nb, &ph, &lidx);
  float2 v[C][3];
  lp_load<C>(in_other, p.ls, nb, s, v);
  float U[18];
  LinkLoad<LINK_F32_12>::load(p.links, lidx, U);
  if (fwd) lp_transport<C, false>(U, ph, v, u);
  else lp_transport<C, true>(U, ph, v, u);
}

// ------------------------------------------------------------ forward layer
// One thread per (output site, s): acc = sum_path W_path (T_path in).  The
// channel mixing runs on packed FP32x2 instructions over pairs of output
// channels (a, a+1): the weights sit in shared memory as float4
// (Re W[a][b], Re W[a+1][b], Im W[a][b], Im W[a+1][b]) and each input
// component is broadcast to a pair, so one complex multiply-add of two output
// channels is four FFMA2.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) lp_conv_kernel(const __grid_constant__ LpConvParams p) {
  static_assert(COUT % 2 == 0, "output channels are processed in pairs");
  constexpr int NA = COUT / 2;
  constexpr int NW = kLpPaths * NA * CIN;
  __shared__ float4 w[NW];                       // [path][a/2][b]
  for (int i = threadIdx.x; i < NW; i += blockDim.x) {
    const int path = i / (NA * CIN);
    const int a2 = (i / CIN) % NA;
    const int b = i % CIN;
    const float2 lo = p.w[(path * COUT + 2 * a2) * CIN + b];
    const float2 hi = p.w[(path * COUT + 2 * a2 + 1) * CIN + b];
    w[i] = make_float4(lo.x, hi.x, lo.y, hi.y);
  }
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= p.vh * p.ls) return;
  const int site = idx / p.ls;
  const int s = idx - site * p.ls;

  float2 accr[NA][3], acci[NA][3];   // (channel 2a, channel 2a+1) real / imaginary parts
#pragma unroll
  for (int a = 0; a < NA; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) { accr[a][c] = make_float2(0.f, 0.f); acci[a][c] = accr[a][c]; }
#pragma unroll 1
  for (int path = 0; path < kLpPaths; ++path) {
    if (path < 3 && !p.in_same) continue;
    if (path >= 3 && !p.in_other) break;
    float2 u[CIN][3];
    lp_path_input<CIN>(p, p.in_same, p.in_other, path, site, s, u);
    const float4* wp = w + path * NA * CIN;
#pragma unroll
    for (int b = 0; b < CIN; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 ur = make_float2(u[b][c].x, u[b][c].x);
        const float2 ui = make_float2(u[b][c].y, u[b][c].y);
        const float2 mui = make_float2(-u[b][c].y, -u[b][c].y);
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const float4 wv = wp[a * CIN + b];
          const float2 wr = make_float2(wv.x, wv.y), wi = make_float2(wv.z, wv.w);
          accr[a][c] = __ffma2_rn(wr, ur, accr[a][c]);
          accr[a][c] = __ffma2_rn(wi, mui, accr[a][c]);
          acci[a][c] = __ffma2_rn(wr, ui, acci[a][c]);
          acci[a][c] = __ffma2_rn(wi, ur, acci[a][c]);
        }
      }
  }
  float2 acc[COUT][3];
#pragma unroll
  for (int a = 0; a < NA; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      acc[2 * a][c] = make_float2(accr[a][c].x, acci[a][c].x);
      acc[2 * a + 1][c] = make_float2(accr[a][c].y, acci[a][c].y);
    }
  lp_store<COUT>(p.out, p.ls, site, s, acc);
}

// ------------------------------------------------------------ gathers of the tensor-core layer
// o[b] = U v[b] (DAG = false) or U^+ v[b] on every channel, two channels per
// packed FP32x2 instruction.
template <int C, bool DAG>
__device__ __forceinline__ void lp_transport2(const float* u, const float2 (&v)[C][3],
                                              float2 (&o)[C][3]) {
  static_assert(C % 2 == 0, "channels in pairs");
#pragma unroll
  for (int b2 = 0; b2 < C / 2; ++b2)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float2 re = make_float2(0.f, 0.f), im = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float ur = DAG ? u[2 * (i + 3 * j)] : u[2 * (j + 3 * i)];
        const float ui = DAG ? -u[2 * (i + 3 * j) + 1] : u[2 * (j + 3 * i) + 1];
        const float2 vx = make_float2(v[2 * b2][j].x, v[2 * b2 + 1][j].x);
        const float2 vy = make_float2(v[2 * b2][j].y, v[2 * b2 + 1][j].y);
        re = __ffma2_rn(make_float2(ur, ur), vx, re);
        re = __ffma2_rn(make_float2(-ui, -ui), vy, re);
        im = __ffma2_rn(make_float2(ur, ur), vy, im);
        im = __ffma2_rn(make_float2(ui, ui), vx, im);
      }
      o[2 * b2][i] = make_float2(re.x, im.x);
      o[2 * b2 + 1][i] = make_float2(re.y, im.y);
    }
}

// Coordinates of a site of parity ieo, computed once per tile row.
struct LpSite {
  int site, ix2, iyzt, y, z, t, keo;
};

template <typename PP>
__device__ __forceinline__ LpSite lp_site(const PP& p, int site) {
  LpSite c;
  c.site = site;
  c.ix2 = site % p.nx2;
  c.iyzt = site / p.nx2;
  c.y = c.iyzt % p.ny;
  const int izt = c.iyzt / p.ny;
  c.z = izt % p.nz;
  c.t = izt / p.nz;
  c.keo = (p.ieo + c.y + c.z + c.t) & 1;
  return c;
}

// Input of one path at (site, s) for the tensor-core layer: the same-parity
// paths read in_same at s, s+1, s-1 (zero past the walls); the hops read
// in_other at the neighbour and transport it with the folded full-record
// links (boundary phase inside; the t links carry the hop's factor 2, which
// the layer's t-path weights undo).
template <int C, typename PP>
__device__ __forceinline__ void lp_tc_path_input(const PP& p, int path, const LpSite& c, int s,
                                                 float2 (&u)[C][3]) {
  if (path < 3) {
    const int ss = (path == 0) ? s : (path == 1 ? s + 1 : s - 1);
    if (ss >= 0 && ss < p.ls) lp_load<C>(p.in_same, p.ls, c.site, ss, u);
    else lp_zero<C>(u);
    return;
  }
  const int d = path - 3;
  const int mu = d >> 1;
  const bool fwd = (d & 1) == 0;
  int nb;
  if (mu == 0) {
    const int row = p.nx2 * c.iyzt;
    nb = fwd ? row + ((c.ix2 + c.keo == p.nx2) ? 0 : c.ix2 + c.keo)
             : row + ((c.ix2 - 1 + c.keo < 0) ? p.nx2 - 1 : c.ix2 - 1 + c.keo);
  } else {
    const int coord = (mu == 1) ? c.y : (mu == 2 ? c.z : c.t);
    const int ext = (mu == 1) ? p.ny : (mu == 2 ? p.nz : p.nt);
    const int stride = (mu == 1) ? p.nx2 : (mu == 2 ? p.nx2 * p.ny : p.nx2 * p.ny * p.nz);
    nb = fwd ? ((coord == ext - 1) ? c.site - (ext - 1) * stride : c.site + stride)
             : ((coord == 0) ? c.site + (ext - 1) * stride : c.site - stride);
  }
  const size_t lidx = fwd ? (size_t)(p.ieo + 2 * mu) * p.vh + c.site : (size_t)(1 - p.ieo + 2 * mu) * p.vh + nb;
  float2 v[C][3];
  lp_load<C>(p.in_other, p.ls, nb, s, v);
  float U[18];
  LinkLoad<LINK_F32_18>::load(p.links_folded, lidx, U);
  if (fwd) lp_transport2<C, false>(U, v, u);
  else lp_transport2<C, true>(U, v, u);
}

// ------------------------------------------------------------ forward layer on the tensor cores
// The same layer as a GEMM on the fifth-generation tensor cores (tcgen05).
// A CTA owns tiles of 128 (site, s) rows; for each color c the layer is
//   out_c[row][n] = sum_k A_c[row][k] B[n][k],
// k running over (path, input channel b, re/im) of the transported inputs and
// n over (output channel a, re/im).  B is the real form of the complex
// weights: row 2a holds (Re W[a][b], -Im W[a][b]) and row 2a+1
// (Im W[a][b], Re W[a][b]) against the (re, im) columns of input b; rows past
// 2*COUT are zero (N = 16 is the smallest MMA width at M = 128).  K is walked
// in steps of 16, one MMA deep: 8/CIN paths per step, the three paths on the
// output parity (identity, s+-1) first, then the eight hops.
//
// The threads gather and transport a step's inputs (the CUDA-core part: the
// SU(3) products), round each FP32 value to NSPLIT BF16 parts (NSPLIT = 2:
// hi + lo, 16 significant bits; NSPLIT = 1: BF16 activations, 8 bits, half
// the shared memory and twice the resident CTAs), and write them as the
// step's A operand into one of two shared-memory stages; one thread then
// issues 3 x NSPLIT MMAs (M = 128, N = 16, K = 16: 3 colors x parts)
// accumulating into three FP32 tiles in tensor memory and commits them to
// the stage's mbarrier, so the tensor core multiplies step j while the
// threads build step j+1.  The weights are BF16 values, so B is exact and,
// with NSPLIT = 2, the result differs from FP32 arithmetic only by the
// rounding of lo (2^-17 relative) and the accumulation order.  The epilogue
// reads the accumulators back (warp w: tensor-memory lanes 32w.., one row
// per thread) and stores the output column.
//
// Every mbarrier wait is bounded; a wait that gives up sets the plan's error
// word (1), skips its row's store, and the CTA drains the MMAs it issued
// (longer bound) before it frees its tensor memory.
constexpr int kTcRows = 128;
constexpr uint32_t kTcTile = kTcRows * 16 * 2;   // one 128 x 16 BF16 operand tile
template <int NSPLIT> constexpr uint32_t tc_stage() { return 3u * NSPLIT * kTcTile; }  // 3 colors x parts
constexpr uint32_t kTcCols = 64;                 // tensor-memory columns (3 x 16 used)

template <int CIN> struct TcShape {
  static constexpr int PPS = 8 / CIN;                   // paths per K step
  static constexpr int NS_SAME = (3 + PPS - 1) / PPS;   // steps of paths 0-2
  static constexpr int NS = NS_SAME + 8 / PPS;          // + steps of the 8 hops
  static constexpr uint32_t B_BYTES = 16u * 16u * 2u * NS;
  static constexpr uint32_t SBO_B = 2u * NS * 128u;     // between the two 8-row groups of B
};

template <int CIN, int NSPLIT>
constexpr size_t lp_conv_tc_smem() {
  return 2 * (size_t)tc_stage<NSPLIT>() + TcShape<CIN>::B_BYTES;
}

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 h) {
  return *reinterpret_cast<uint32_t*>(&h);
}

template <int CIN, int COUT, int NSPLIT>
__global__ void __launch_bounds__(128, NSPLIT == 1 ? 5 : 4)
lp_conv_tc_kernel(const __grid_constant__ LpConvParams p) {
  using TS = TcShape<CIN>;
  constexpr int PPS = TS::PPS, NS_SAME = TS::NS_SAME, NS = TS::NS;
  constexpr uint32_t kTcStage = tc_stage<NSPLIT>();
  static_assert(NSPLIT == 1 || NSPLIT == 2, "BF16 parts per value: 1 or 2");
  constexpr uint32_t IDESC = umma_idesc_bf16_f32(kTcRows, 16);
  static_assert(CIN == 4 || CIN == 8, "input channels: 4 or 8");
  static_assert(2 * COUT <= 16, "output channels: at most 8");
  extern __shared__ __align__(1024) unsigned char smem[];
  // stage s free again (MMAs of its last use complete: tcgen05.commit), tile
  // done (every MMA of the tile complete), stage s written (every thread
  // arrived)
  __shared__ __align__(8) uint64_t bars[5];    // empty 0, empty 1, done, full 0, full 1
  __shared__ uint32_t tmem_base;

  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bbase = sbase + 2 * kTcStage;

  if (warp == 0) {
    tmem_alloc(smem_u32(&tmem_base), kTcCols);
    tmem_relinquish();
  }
  if (tid == 0) {
#pragma unroll
    for (int i = 0; i < 3; ++i) mbar_init(smem_u32(&bars[i]), 1);
    mbar_init(smem_u32(&bars[3]), kTcRows);
    mbar_init(smem_u32(&bars[4]), kTcRows);
    mbar_fence_init();
  }
  // B, K-major without swizzle: element (n, k) at (n%8)*16 + (n/8)*SBO_B +
  // (k/8)*128 + (k%8)*2 bytes.
  for (int e = tid; e < 16 * NS * 16; e += blockDim.x) {
    const int n = e / (NS * 16), k = e - n * (NS * 16);
    const int j = k >> 4, kk = k & 15;
    const int q = kk / (2 * CIN), b = (kk >> 1) % CIN, ri = kk & 1;
    const int path = (j < NS_SAME) ? j * PPS + q : 3 + (j - NS_SAME) * PPS + q;
    const int a = n >> 1;
    float val = 0.f;
    if ((j >= NS_SAME || path < 3) && a < COUT) {
      const float2 w = p.w[(path * COUT + a) * CIN + b];
      val = (n & 1) ? (ri ? w.x : w.y) : (ri ? -w.y : w.x);
      if (path >= 9) val *= 0.5f;   // the folded t links carry a factor 2 (exact)
    }
    const uint32_t off = (n & 7) * 16 + (n >> 3) * TS::SBO_B + (k >> 3) * 128 + (k & 7) * 2;
    *reinterpret_cast<__nv_bfloat16*>(smem + 2 * kTcStage + off) = __float2bfloat16_rn(val);
  }
  fence_proxy_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t taddr = tmem_base;

  const int rows = p.vh * p.ls;
  const int ntiles = (rows + kTcRows - 1) / kTcRows;
  const int j0 = p.in_same ? 0 : NS_SAME;
  const int j1 = p.in_other ? NS : NS_SAME;
  const uint32_t row_off = (uint32_t)(tid & 7) * 16 + (uint32_t)(tid >> 3) * 256;
  int g = 0;        // K steps this CTA has built; stage g & 1
  int ndone = 0;    // tile-done commits
  bool bad = false;
  // One thread issues step h's MMAs once every thread has written its stage
  // (full barrier of the stage, phase h / 2), then frees the stage by a
  // commit to its empty barrier.  Issued one step late, so that the wait is
  // for writes that are normally done already and no CTA-wide barrier
  // holds the gathers back.
  auto issue = [&](int h, int jj) {
    const int sh = h & 1;
    if (!mbar_wait_bounded(smem_u32(&bars[3 + sh]), (h >> 1) & 1)) bad = true;
    tc_fence_after_sync();
    const uint64_t bdesc = umma_smem_desc(bbase + (uint32_t)jj * 256, 128, TS::SBO_B);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int part = 0; part < NSPLIT; ++part) {
        const uint64_t adesc =
            umma_smem_desc(sbase + sh * kTcStage + (NSPLIT * c + part) * kTcTile, 128, 256);
        umma_bf16_ss(taddr + (uint32_t)(c * 16), adesc, bdesc, IDESC, jj > j0 || part > 0);
      }
    umma_commit(smem_u32(&bars[sh]));
  };
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int idx = tile * kTcRows + tid;
    const bool active = idx < rows;
    const int site = active ? idx / p.ls : 0;
    const int s = active ? idx - site * p.ls : 0;
    const LpSite cs = lp_site(p, site);
    for (int j = j0; j < j1; ++j, ++g) {
      float v[3][16];
#pragma unroll
      for (int q = 0; q < PPS; ++q) {
        const int path = (j < NS_SAME) ? j * PPS + q : 3 + (j - NS_SAME) * PPS + q;
        float2 u[CIN][3];
        if (active && (j >= NS_SAME || path < 3))
          lp_tc_path_input<CIN>(p, path, cs, s, u);
        else
          lp_zero<CIN>(u);
#pragma unroll
        for (int b = 0; b < CIN; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            v[c][q * 2 * CIN + 2 * b] = u[b][c].x;
            v[c][q * 2 * CIN + 2 * b + 1] = u[b][c].y;
          }
      }
      const int st = g & 1;
      // the stage's previous MMAs (step g - 2) must have read it
      if (g >= 2 && !mbar_wait_bounded(smem_u32(&bars[st]), ((g - 2) >> 1) & 1)) bad = true;
      unsigned char* stage = smem + st * kTcStage;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float x0 = v[c][2 * i], x1 = v[c][2 * i + 1];
          const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
          hi[i] = bf16x2_bits(h);
          if (NSPLIT == 2)
            lo[i] = bf16x2_bits(__floats2bfloat162_rn(x0 - __low2float(h), x1 - __high2float(h)));
        }
        uint4* th = reinterpret_cast<uint4*>(stage + (NSPLIT * c) * kTcTile + row_off);
        th[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);   // K 0-7
        th[8] = make_uint4(hi[4], hi[5], hi[6], hi[7]);   // K 8-15, 128 bytes on
        if (NSPLIT == 2) {
          uint4* tl = reinterpret_cast<uint4*>(stage + (2 * c + 1) * kTcTile + row_off);
          tl[0] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
          tl[8] = make_uint4(lo[4], lo[5], lo[6], lo[7]);
        }
      }
      fence_proxy_async_smem();
      tc_fence_before_sync();
      mbar_arrive(smem_u32(&bars[3 + st]));
      if (tid == 0 && j > j0) issue(g - 1, j - 1);
    }
    if (tid == 0) {
      issue(g - 1, j1 - 1);
      umma_commit(smem_u32(&bars[2]));
    }
    if (!mbar_wait_bounded(smem_u32(&bars[2]), ndone & 1)) bad = true;
    ++ndone;
    tc_fence_after_sync();
    float2 acc[COUT][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float d[16];
      tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 16), d);
#pragma unroll
      for (int a = 0; a < COUT; ++a) acc[a][c] = make_float2(d[2 * a], d[2 * a + 1]);
    }
    if (active && !bad) lp_store<COUT>(p.out, p.ls, site, s, acc);
    tc_fence_before_sync();
  }
  if (__syncthreads_or(bad)) {
    if (tid == 0) {
      if (p.err) atomicExch(p.err, 1);
      umma_commit(smem_u32(&bars[2]));
    }
    mbar_wait_drain(smem_u32(&bars[2]), ndone & 1);
    tc_fence_before_sync();
    __syncthreads();
  }
  if (warp == 0) {
    tc_fence_after_sync();
    tmem_dealloc(taddr, kTcCols);
  }
}

// ------------------------------------------------------------ weight gradient
// G_path[a][b] = sum over (site, s, color) of delta[a] * conj((T_path in)[b]).
// A block walks tiles of kGradTile (site, s) rows: the transported inputs of
// all paths and the deltas of the tile go to shared memory, then each thread
// accumulates its own (path, a, b) entries over the tile.
constexpr int kGradTile = 32;
constexpr int kGradThreads = 256;

template <int CIN, int COUT>
constexpr size_t lp_gradw_smem() {
  return sizeof(float2) * ((size_t)kGradTile * kLpPaths * 3 * CIN + (size_t)kGradTile * 3 * COUT);
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kGradThreads) lp_gradw_kernel(const __grid_constant__ LpGradParams p) {
  constexpr int NE = kLpPaths * COUT * CIN;
  constexpr int EPT = (NE + kGradThreads - 1) / kGradThreads;
  extern __shared__ float2 sm[];
  float2* ut = sm;                                           // [row][path][color][b]
  float2* dt = sm + (size_t)kGradTile * kLpPaths * 3 * CIN;  // [row][color][a]
  float2 g[EPT];
#pragma unroll
  for (int e = 0; e < EPT; ++e) g[e] = make_float2(0.f, 0.f);
  const int rows = p.vh * p.ls;

  for (int base = blockIdx.x * kGradTile; base < rows; base += gridDim.x * kGradTile) {
    // path-major jobs: a warp handles one path for 32 consecutive rows
    for (int job = threadIdx.x; job < kGradTile * kLpPaths; job += blockDim.x) {
      const int path = job / kGradTile;
      const int r = job - path * kGradTile;
      const int idx = base + r;
      float2 u[CIN][3];
      if (idx < rows) {
        const int site = idx / p.ls;
        lp_path_input<CIN>(p, p.in_same, p.in_other, path, site, idx - site * p.ls, u);
      } else {
        lp_zero<CIN>(u);
      }
      float2* dst = ut + ((size_t)(r * kLpPaths + path) * 3) * CIN;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int b = 0; b < CIN; ++b) dst[c * CIN + b] = u[b][c];
    }
    for (int r = threadIdx.x; r < kGradTile; r += blockDim.x) {
      const int idx = base + r;
      float2 d[COUT][3];
      if (idx < rows) {
        const int site = idx / p.ls;
        lp_load<COUT>(p.delta, p.ls, site, idx - site * p.ls, d);
      } else {
        lp_zero<COUT>(d);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < COUT; ++a) dt[(r * 3 + c) * COUT + a] = d[a][c];
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int E = threadIdx.x + e * kGradThreads;
      if (E < NE) {
        const int path = E / (COUT * CIN);
        const int a = (E / CIN) % COUT;
        const int b = E % CIN;
        float re = g[e].x, im = g[e].y;
        for (int r = 0; r < kGradTile; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float2 dv = dt[(r * 3 + c) * COUT + a];
            const float2 uv = ut[((size_t)(r * kLpPaths + path) * 3 + c) * CIN + b];
            // dv * conj(uv)
            re = fmaf(dv.x, uv.x, re); re = fmaf(dv.y, uv.y, re);
            im = fmaf(dv.y, uv.x, im); im = fmaf(-dv.x, uv.y, im);
          }
        g[e] = make_float2(re, im);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int E = threadIdx.x + e * kGradThreads;
    if (E < NE) p.partial[(size_t)blockIdx.x * NE + E] = g[e];
  }
}

// grad[E] (+)= sum over blocks of partial[b][E], summed in double.
__global__ void lp_reduce_kernel(const float2* partial, int nblocks, int ne, float2* grad,
                                 int accumulate) {
  const int E = blockIdx.x * blockDim.x + threadIdx.x;
  if (E >= ne) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    const float2 v = partial[(size_t)b * ne + E];
    re += v.x;
    im += v.y;
  }
  if (accumulate) { re += grad[E].x; im += grad[E].y; }
  grad[E] = make_float2((float)re, (float)im);
}

// ------------------------------------------------------------ loss and norms
__global__ void lp_norm_kernel(const float4* x, size_t n4, double* partial) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const float4 v = x[i];
    acc += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// t = y - e
__global__ void lp_sub_kernel(const float4* y, const float4* e, float4* t, size_t n4) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const float4 a = y[i], b = e[i];
    t[i] = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
  }
}

// out = num * x / den[0] (den a device scalar; zero if den is not positive)
__global__ void lp_scale_kernel(const float4* x, float4* out, size_t n4, const double* den, double num) {
  const float f = (den[0] > 0.0) ? (float)(num / den[0]) : 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const float4 a = x[i];
    out[i] = make_float4(f * a.x, f * a.y, f * a.z, f * a.w);
  }
}

// w *= c[0] / c[1] on n complex weights (c: device scalars)
__global__ void lp_rescale_kernel(float2* w, int n, const double* c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(c[1] > 0.0)) return;
  const float f = (float)(c[0] / c[1]);
  w[i] = make_float2(f * w[i].x, f * w[i].y);
}

// out[0] = Re <x, y> over n4 float4 (complex pairs), per-block partials
__global__ void lp_redot_kernel(const float4* x, const float4* y, size_t n4, double* partial) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const float4 a = x[i], b = y[i];
    acc += (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void lp_sum_kernel(const double* partial, int n, double* out) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

// ------------------------------------------------------------ parameters
__device__ __forceinline__ int lp_swap_path(int path) {
  if (path == 0) return 0;
  if (path == 1) return 2;
  if (path == 2) return 1;
  return ((path - 3) & 1) ? path - 1 : path + 1;
}

// Deployed weights of one layer: BF16-rounded master weights (forward) and the
// adjoint layer's weights, W'_path = (W_swap(path))^H.
__global__ void lp_prep_kernel(const float2* master, float2* wf, float2* wadj, int cin, int cout) {
  const int ne = kLpPaths * cout * cin;
  const int E = blockIdx.x * blockDim.x + threadIdx.x;
  if (E >= ne) return;
  const int path = E / (cout * cin);
  const int a = (E / cin) % cout;
  const int b = E % cin;
  const float2 m = master[E];
  const float re = __bfloat162float(__float2bfloat16_rn(m.x));
  const float im = __bfloat162float(__float2bfloat16_rn(m.y));
  wf[E] = make_float2(re, im);
  wadj[(lp_swap_path(path) * cin + b) * cout + a] = make_float2(re, -im);
}

__global__ void lp_adam_kernel(float2* w, float2* m, float2* v, const float2* g, int n, float lr,
                               float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float2 mm = m[i], vv = v[i], ww = w[i];
  const float2 gg = g[i];
  mm.x = b1 * mm.x + (1.f - b1) * gg.x;
  mm.y = b1 * mm.y + (1.f - b1) * gg.y;
  vv.x = b2 * vv.x + (1.f - b2) * gg.x * gg.x;
  vv.y = b2 * vv.y + (1.f - b2) * gg.y * gg.y;
  ww.x -= lr * (mm.x / c1) / (sqrtf(vv.x / c2) + eps);
  ww.y -= lr * (mm.y / c1) / (sqrtf(vv.y / c2) + eps);
  m[i] = mm; v[i] = vv; w[i] = ww;
}

// The convolution kernel, by B200_LP_CONV: "tc" (default) the tensor-core
// form with BF16 hi + lo inputs, "tc1" the tensor-core form with BF16
// inputs, "ffma2" the packed-FFMA2 form.  All compute the same layer; the
// tensor-core forms round the transported inputs to 16 (tc) or 8 (tc1)
// significant bits before the product.
enum LpConvKind { LP_TC2 = 0, LP_TC1 = 1, LP_FFMA2 = 2 };
LpConvKind lp_conv_kind() {
  const char* e = getenv("B200_LP_CONV");
  if (e && strcmp(e, "ffma2") == 0) return LP_FFMA2;
  if (e && strcmp(e, "tc1") == 0) return LP_TC1;
  return LP_TC2;
}

template <int CIN, int COUT, int NSPLIT>
cudaError_t run_conv_tc(const LpConvParams& p, cudaStream_t st) {
  constexpr size_t smem = lp_conv_tc_smem<CIN, NSPLIT>();
  auto k = lp_conv_tc_kernel<CIN, COUT, NSPLIT>;
  static int grid_cap = 0;
  if (!grid_cap) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the whole unified L1 as shared memory, so that the most CTAs fit an SM
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0, dev = 0, nsm = 0, smem_sm = 0, regs_sm = 0;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess) return e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
      return e;
    if ((e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess)
      return e;
    // resident CTAs per SM from the kernel's own footprint (shared memory
    // with the 1 KB the system reserves per CTA, registers); a grid sized
    // from the occupancy query alone came out at one CTA per SM (148), so
    // the larger of the two counts is used
    const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + 1024);
    const int by_regs = regs_sm / (fa.numRegs * kTcRows);
    per_sm = by_smem < by_regs ? by_smem : by_regs;
    int api = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&api, k, kTcRows, smem) == cudaSuccess && api > per_sm)
      per_sm = api;
    // resident CTAs share the SM's 512 tensor-memory columns: never more than
    // 512 / kTcCols of them, so no allocation has to wait
    per_sm = per_sm < 1 ? 1 : (per_sm > (int)(512 / kTcCols) ? (int)(512 / kTcCols) : per_sm);
    grid_cap = per_sm * nsm;
  }
  const int ntiles = (p.vh * p.ls + kTcRows - 1) / kTcRows;
  k<<<ntiles < grid_cap ? ntiles : grid_cap, kTcRows, smem, st>>>(p);
  return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t run_conv(const LpConvParams& p, cudaStream_t st) {
  const LpConvKind kind = lp_conv_kind();
  if (kind == LP_TC2) return run_conv_tc<CIN, COUT, 2>(p, st);
  if (kind == LP_TC1) return run_conv_tc<CIN, COUT, 1>(p, st);
  const int n = p.vh * p.ls;
  lp_conv_kernel<CIN, COUT><<<(n + 127) / 128, 128, 0, st>>>(p);
  return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t run_gradw(const LpGradParams& p, int max_blocks, int* nblocks, cudaStream_t st) {
  constexpr size_t smem = lp_gradw_smem<CIN, COUT>();
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(lp_gradw_kernel<CIN, COUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const int rows = p.vh * p.ls;
  int nb = (rows + kGradTile - 1) / kGradTile;
  if (nb > max_blocks) nb = max_blocks;
  *nblocks = nb;
  lp_gradw_kernel<CIN, COUT><<<nb, kGradThreads, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_lp_conv(int cin, int cout, const LpConvParams& p, cudaStream_t st) {
  if (cin == 4 && cout == 8) return run_conv<4, 8>(p, st);
  if (cin == 8 && cout == 8) return run_conv<8, 8>(p, st);
  if (cin == 8 && cout == 4) return run_conv<8, 4>(p, st);
  if (cin == 4 && cout == 4) return run_conv<4, 4>(p, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_lp_gradw(int cin, int cout, const LpGradParams& p, int max_blocks, int* nblocks,
                            cudaStream_t st) {
  if (cin == 4 && cout == 8) return run_gradw<4, 8>(p, max_blocks, nblocks, st);
  if (cin == 8 && cout == 8) return run_gradw<8, 8>(p, max_blocks, nblocks, st);
  if (cin == 8 && cout == 4) return run_gradw<8, 4>(p, max_blocks, nblocks, st);
  if (cin == 4 && cout == 4) return run_gradw<4, 4>(p, max_blocks, nblocks, st);
  return cudaErrorInvalidValue;
}

}  // namespace b200

using namespace b200;

// ------------------------------------------------------------ network object
struct b200_lp {
  b200_dwf* op = nullptr;
  int hidden = 0;
  Geom g{};
  float bc[4] = {1, 1, 1, 1};
  int cin[3] = {0, 0, 0}, cout[3] = {0, 0, 0}, off[4] = {0, 0, 0, 0};
  int nparam = 0;                       // complex weights
  float2* master = nullptr;             // FP32 master weights
  float2* adam_m = nullptr;
  float2* adam_v = nullptr;
  float2* grad = nullptr;
  float2* wf = nullptr;                 // deployed (BF16-valued) forward weights
  float2* wadj = nullptr;               // deployed adjoint weights
  bool prepped = false;
  int t = 0;                            // Adam step
  float4* act[12] = {};                 // y1e y1o y2e y2o y3 d3 d2e d2o d1e d1o t ad
  float2* partial = nullptr;
  int max_blocks = 0;
  double* red = nullptr;                // reduction partials
  double* sc = nullptr;                 // device scalars: [0] |e|^2, [1] loss
  double* sc_host = nullptr;
};

namespace {

enum { Y1E = 0, Y1O, Y2E, Y2O, Y3, D3, D2E, D2O, D1E, D1O, T4, AD4, NACT };
constexpr int kRedBlocks = 296;

int lp_fail(int code, const char* msg) {
  set_last_error(code, "%s", msg);
  return code;
}

#define LP_CHECK(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_last_error(B200_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,              \
                     cudaGetErrorString(e_));                                            \
      return B200_ECUDA;                                                                 \
    }                                                                                    \
  } while (0)

size_t act_bytes(const b200_lp* lp, int channels) {
  return (size_t)lp->g.vh * lp->g.ls * 3 * channels * sizeof(float2);
}

int lp_prep(b200_lp* lp, cudaStream_t st) {
  if (lp->prepped) return 0;
  for (int l = 0; l < 3; ++l) {
    const int ne = kLpPaths * lp->cin[l] * lp->cout[l];
    lp_prep_kernel<<<(ne + 255) / 256, 256, 0, st>>>(lp->master + lp->off[l], lp->wf + lp->off[l],
                                                     lp->wadj + lp->off[l], lp->cin[l], lp->cout[l]);
    LP_CHECK(cudaGetLastError());
  }
  lp->prepped = true;
  return 0;
}

LpConvParams conv_base(const b200_lp* lp, const void* links, int ieo) {
  LpConvParams p;
  memset(&p, 0, sizeof(p));
  p.links = links;
  p.err = plan_error_word(lp->op);
  p.vh = lp->g.vh; p.nx2 = lp->g.nx2; p.ny = lp->g.ny; p.nz = lp->g.nz; p.nt = lp->g.nt;
  p.ls = lp->g.ls;
  p.ieo = ieo;
  for (int mu = 0; mu < 4; ++mu) p.bc[mu] = lp->bc[mu];
  return p;
}

int conv(b200_lp* lp, const void* links, int layer, bool adjoint, int ieo, const float4* in_same,
         const float4* in_other, float4* out, cudaStream_t st) {
  LpConvParams p = conv_base(lp, links, ieo);
  int rc;
  if ((rc = plan_links_f32_folded(lp->op, &p.links_folded, st))) return rc;
  p.in_same = in_same;
  p.in_other = in_other;
  p.out = out;
  p.w = (adjoint ? lp->wadj : lp->wf) + lp->off[layer];
  const int ci = adjoint ? lp->cout[layer] : lp->cin[layer];
  const int co = adjoint ? lp->cin[layer] : lp->cout[layer];
  LP_CHECK(launch_lp_conv(ci, co, p, st));
  return 0;
}

int gradw(b200_lp* lp, const void* links, int layer, int ieo, const float4* delta,
          const float4* in_same, const float4* in_other, bool accumulate, cudaStream_t st) {
  LpGradParams p;
  memset(&p, 0, sizeof(p));
  p.delta = delta;
  p.in_same = in_same;
  p.in_other = in_other;
  p.links = links;
  p.partial = lp->partial;
  p.vh = lp->g.vh; p.nx2 = lp->g.nx2; p.ny = lp->g.ny; p.nz = lp->g.nz; p.nt = lp->g.nt;
  p.ls = lp->g.ls;
  p.ieo = ieo;
  for (int mu = 0; mu < 4; ++mu) p.bc[mu] = lp->bc[mu];
  int nb = 0;
  LP_CHECK(launch_lp_gradw(lp->cin[layer], lp->cout[layer], p, lp->max_blocks, &nb, st));
  const int ne = kLpPaths * lp->cin[layer] * lp->cout[layer];
  lp_reduce_kernel<<<(ne + 255) / 256, 256, 0, st>>>(lp->partial, nb, ne, lp->grad + lp->off[layer],
                                                     accumulate ? 1 : 0);
  LP_CHECK(cudaGetLastError());
  return 0;
}

// y3 = N(r): five convolution launches.
int forward(b200_lp* lp, const void* links, const float4* r, float4* y3, cudaStream_t st) {
  int rc;
  if ((rc = lp_prep(lp, st))) return rc;
  float4** a = lp->act;
  if ((rc = conv(lp, links, 0, false, 0, r, nullptr, a[Y1E], st))) return rc;
  if ((rc = conv(lp, links, 0, false, 1, nullptr, r, a[Y1O], st))) return rc;
  if ((rc = conv(lp, links, 1, false, 0, a[Y1E], a[Y1O], a[Y2E], st))) return rc;
  if ((rc = conv(lp, links, 1, false, 1, a[Y1O], a[Y1E], a[Y2O], st))) return rc;
  if ((rc = conv(lp, links, 2, false, 0, a[Y2E], a[Y2O], y3, st))) return rc;
  return 0;
}

// Activations of the backward pass, the loss temporaries and the gradient
// partials, allocated by the first training call.
int ensure_train_buffers(b200_lp* lp) {
  for (int i = Y3; i < NACT; ++i) {
    if (lp->act[i]) continue;
    const int ch = (i == Y3 || i == D3 || i == T4 || i == AD4) ? kLpIn : lp->hidden;
    if (cudaMalloc(&lp->act[i], act_bytes(lp, ch)) != cudaSuccess) {
      lp->act[i] = nullptr;
      return lp_fail(B200_ENOMEM, "allocation of the training buffers failed");
    }
  }
  if (!lp->partial &&
      cudaMalloc(&lp->partial, sizeof(float2) * (size_t)lp->max_blocks * kLpPaths * lp->hidden * lp->hidden) !=
          cudaSuccess) {
    lp->partial = nullptr;
    return lp_fail(B200_ENOMEM, "allocation of the gradient partials failed");
  }
  return 0;
}

bool bad_ptr(const void* p) { return !p || (reinterpret_cast<uintptr_t>(p) & 15u) != 0; }

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double gauss(uint64_t& s) {
  const double u1 = ((splitmix(s) >> 11) + 1.0) / 9007199254740993.0;
  const double u2 = (splitmix(s) >> 11) / 9007199254740992.0;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

}  // namespace

namespace b200 {
int lp_apply_internal(b200_lp* lp, void* z_f32, const void* r_f32, cudaStream_t st) {
  const void* links = nullptr;
  int rc;
  if ((rc = plan_links_f32(lp->op, &links, st))) return rc;
  return forward(lp, links, reinterpret_cast<const float4*>(r_f32), reinterpret_cast<float4*>(z_f32), st);
}
}  // namespace b200

extern "C" {

int b200_lp_create(b200_lp_t** out, b200_dwf_t* op, int hidden, unsigned long long seed,
                   double init_noise) {
  if (!out || !op) return lp_fail(B200_EINVAL, "invalid argument");
  if (hidden != 4 && hidden != 8) return lp_fail(B200_EINVAL, "hidden channels must be 4 or 8");
  if (plan_has_halo(op))
    return lp_fail(B200_EINVAL, "the learned preconditioner needs a plan without a halo exchange hook");
  *out = nullptr;
  b200_lp* lp = new b200_lp();
  lp->op = op;
  lp->hidden = hidden;
  if (plan_geometry(op, &lp->g, lp->bc)) { delete lp; return B200_EINVAL; }
  const int ci[3] = {kLpIn, hidden, hidden}, co[3] = {hidden, hidden, kLpIn};
  for (int l = 0; l < 3; ++l) {
    lp->cin[l] = ci[l];
    lp->cout[l] = co[l];
    lp->off[l + 1] = lp->off[l] + kLpPaths * ci[l] * co[l];
  }
  lp->nparam = lp->off[3];
  // Initial weights: the identity path of each layer carries the identity on
  // the first min(cin, cout) channels, everything else small Gaussian noise.
  std::vector<float2> w(lp->nparam);
  uint64_t s = seed ? seed : 0x1234567ull;
  for (int l = 0; l < 3; ++l)
    for (int path = 0; path < kLpPaths; ++path)
      for (int a = 0; a < co[l]; ++a)
        for (int b = 0; b < ci[l]; ++b) {
          const int E = lp->off[l] + (path * co[l] + a) * ci[l] + b;
          const double nr = init_noise * gauss(s), ni = init_noise * gauss(s);
          w[E] = make_float2((float)(nr + ((path == 0 && a == b) ? 1.0 : 0.0)), (float)ni);
        }
  const size_t pb = sizeof(float2) * lp->nparam;
  bool ok = cudaMalloc(&lp->master, pb) == cudaSuccess && cudaMalloc(&lp->adam_m, pb) == cudaSuccess &&
            cudaMalloc(&lp->adam_v, pb) == cudaSuccess && cudaMalloc(&lp->grad, pb) == cudaSuccess &&
            cudaMalloc(&lp->wf, pb) == cudaSuccess && cudaMalloc(&lp->wadj, pb) == cudaSuccess;
  // the forward pass needs the hidden layers' activations only; the
  // training buffers come with the first training call
  for (int i = Y1E; ok && i <= Y2O; ++i) ok = cudaMalloc(&lp->act[i], act_bytes(lp, hidden)) == cudaSuccess;
  lp->max_blocks = 148 * 3;
  ok = ok && cudaMalloc(&lp->red, sizeof(double) * kRedBlocks) == cudaSuccess;
  ok = ok && cudaMalloc(&lp->sc, sizeof(double) * 4) == cudaSuccess;
  ok = ok && cudaMallocHost(&lp->sc_host, sizeof(double) * 4) == cudaSuccess;
  if (!ok) {
    b200_lp_destroy(lp);
    return lp_fail(B200_ENOMEM, "allocation of the network buffers failed");
  }
  if (cudaMemcpy(lp->master, w.data(), pb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(lp->adam_m, 0, pb) != cudaSuccess || cudaMemset(lp->adam_v, 0, pb) != cudaSuccess ||
      cudaMemset(lp->grad, 0, pb) != cudaSuccess) {
    b200_lp_destroy(lp);
    return lp_fail(B200_ECUDA, "upload of the initial weights failed");
  }
  *out = lp;
  return 0;
}

int b200_lp_destroy(b200_lp_t* lp) {
  if (!lp) return 0;
  cudaFree(lp->master); cudaFree(lp->adam_m); cudaFree(lp->adam_v); cudaFree(lp->grad);
  cudaFree(lp->wf); cudaFree(lp->wadj);
  for (int i = 0; i < NACT; ++i) cudaFree(lp->act[i]);
  cudaFree(lp->partial); cudaFree(lp->red); cudaFree(lp->sc);
  if (lp->sc_host) cudaFreeHost(lp->sc_host);
  delete lp;
  return 0;
}

int b200_lp_nparams(const b200_lp_t* lp) { return lp ? lp->nparam : 0; }

int b200_lp_set_weights(b200_lp_t* lp, const float* w, int nfloat) {
  if (!lp || !w || nfloat != 2 * lp->nparam) return lp_fail(B200_EINVAL, "weights: wrong size");
  LP_CHECK(cudaMemcpy(lp->master, w, sizeof(float) * nfloat, cudaMemcpyHostToDevice));
  LP_CHECK(cudaMemset(lp->adam_m, 0, sizeof(float) * nfloat));
  LP_CHECK(cudaMemset(lp->adam_v, 0, sizeof(float) * nfloat));
  lp->t = 0;
  lp->prepped = false;
  return 0;
}

int b200_lp_get_weights(b200_lp_t* lp, float* w, int nfloat, int deployed) {
  if (!lp || !w || nfloat != 2 * lp->nparam) return lp_fail(B200_EINVAL, "weights: wrong size");
  if (deployed) {
    int rc;
    if ((rc = lp_prep(lp, 0))) return rc;
    LP_CHECK(cudaMemcpy(w, lp->wf, sizeof(float) * nfloat, cudaMemcpyDeviceToHost));
  } else {
    LP_CHECK(cudaMemcpy(w, lp->master, sizeof(float) * nfloat, cudaMemcpyDeviceToHost));
  }
  return 0;
}

int b200_lp_apply(b200_lp_t* lp, void* z_f32, const void* r_f32, void* stream) {
  if (!lp || bad_ptr(z_f32) || bad_ptr(r_f32)) return lp_fail(B200_EINVAL, "invalid argument");
  return lp_apply_internal(lp, z_f32, r_f32, (cudaStream_t)stream);
}

// Forward, loss L = |A (N r - e)|^2 / |r|^2 (A = DdagD, r = A e) and the
// gradient dL/dRe W + i dL/dIm W of every weight (kept on the device;
// b200_lp_get_grad copies it out).  dL/dy = 2 A A (y - e) / |r|^2 since A is
// Hermitian: two FP32 DdagD applications per step.
int b200_lp_loss_grad(b200_lp_t* lp, const void* r_f32, const void* e_f32, double* loss,
                      void* stream) {
  if (!lp || bad_ptr(r_f32) || bad_ptr(e_f32)) return lp_fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const void* links = nullptr;
  int rc;
  if ((rc = ensure_train_buffers(lp))) return rc;
  if ((rc = plan_links_f32(lp->op, &links, st))) return rc;
  const float4* r = reinterpret_cast<const float4*>(r_f32);
  const float4* e = reinterpret_cast<const float4*>(e_f32);
  float4** a = lp->act;
  if ((rc = forward(lp, links, r, a[Y3], st))) return rc;
  const size_t n4 = act_bytes(lp, kLpIn) / sizeof(float4);
  lp_norm_kernel<<<kRedBlocks, 256, 0, st>>>(r, n4, lp->red);
  lp_sum_kernel<<<1, 256, 0, st>>>(lp->red, kRedBlocks, lp->sc);          // |r|^2
  lp_sub_kernel<<<kRedBlocks, 256, 0, st>>>(a[Y3], e, a[T4], n4);         // t = y - e
  LP_CHECK(cudaGetLastError());
  if ((rc = plan_apply_ddagd(lp->op, a[AD4], a[T4], st))) return rc;       // d = A t
  lp_norm_kernel<<<kRedBlocks, 256, 0, st>>>(a[AD4], n4, lp->red);
  lp_sum_kernel<<<1, 256, 0, st>>>(lp->red, kRedBlocks, lp->sc + 1);      // |d|^2
  if ((rc = plan_apply_ddagd(lp->op, a[T4], a[AD4], st))) return rc;       // A d
  lp_scale_kernel<<<kRedBlocks, 256, 0, st>>>(a[T4], a[D3], n4, lp->sc, 2.0);
  LP_CHECK(cudaGetLastError());
  // layer 3 (output even only)
  if ((rc = gradw(lp, links, 2, 0, a[D3], a[Y2E], a[Y2O], false, st))) return rc;
  if ((rc = conv(lp, links, 2, true, 0, a[D3], nullptr, a[D2E], st))) return rc;
  if ((rc = conv(lp, links, 2, true, 1, nullptr, a[D3], a[D2O], st))) return rc;
  // layer 2
  if ((rc = gradw(lp, links, 1, 0, a[D2E], a[Y1E], a[Y1O], false, st))) return rc;
  if ((rc = gradw(lp, links, 1, 1, a[D2O], a[Y1O], a[Y1E], true, st))) return rc;
  if ((rc = conv(lp, links, 1, true, 0, a[D2E], a[D2O], a[D1E], st))) return rc;
  if ((rc = conv(lp, links, 1, true, 1, a[D2O], a[D2E], a[D1O], st))) return rc;
  // layer 1 (input even only)
  if ((rc = gradw(lp, links, 0, 0, a[D1E], r, nullptr, false, st))) return rc;
  if ((rc = gradw(lp, links, 0, 1, a[D1O], nullptr, r, true, st))) return rc;
  LP_CHECK(cudaMemcpyAsync(lp->sc_host, lp->sc, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
  if ((rc = plan_check_error(lp->op, st))) return rc;      // synchronises the stream
  if (!(lp->sc_host[0] > 0.0)) return lp_fail(B200_EINVAL, "residual field r is zero");
  if (loss) *loss = lp->sc_host[1] / lp->sc_host[0];
  return 0;
}

int b200_lp_get_grad(b200_lp_t* lp, float* g, int nfloat) {
  if (!lp || !g || nfloat != 2 * lp->nparam) return lp_fail(B200_EINVAL, "gradient: wrong size");
  LP_CHECK(cudaMemcpy(g, lp->grad, sizeof(float) * nfloat, cudaMemcpyDeviceToHost));
  return 0;
}

int b200_lp_adam_step(b200_lp_t* lp, double lr, void* stream) {
  if (!lp || !(lr > 0.0)) return lp_fail(B200_EINVAL, "invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const float b1 = 0.9f, b2 = 0.999f;
  lp->t += 1;
  const float c1 = 1.f - std::pow(b1, (float)lp->t), c2 = 1.f - std::pow(b2, (float)lp->t);
  lp_adam_kernel<<<(lp->nparam + 255) / 256, 256, 0, st>>>(lp->master, lp->adam_m, lp->adam_v, lp->grad,
                                                          lp->nparam, (float)lr, b1, b2, 1e-8f, c1, c2);
  LP_CHECK(cudaGetLastError());
  lp->prepped = false;
  return 0;
}

// Epochs of Adam over (r_i, e_i) pairs in a seeded shuffled order; returns the
// mean loss of the first and of the last epoch.
int b200_lp_train(b200_lp_t* lp, int npairs, const void* const* r_f32, const void* const* e_f32,
                  int epochs, double lr, unsigned long long seed, double* loss_first,
                  double* loss_last, void* stream) {
  if (!lp || npairs <= 0 || !r_f32 || !e_f32 || epochs <= 0 || !(lr > 0.0))
    return lp_fail(B200_EINVAL, "invalid argument");
  std::vector<int> order(npairs);
  for (int i = 0; i < npairs; ++i) order[i] = i;
  uint64_t s = seed ? seed : 0xABCDEFull;
  if (lp->t == 0) {
    // Fresh network: scale the last layer by the least-squares factor
    // c = Re<A N r, r> / |A N r|^2 on the first pair, so training starts from
    // the best multiple of the initial N.
    cudaStream_t st = (cudaStream_t)stream;
    const void* links = nullptr;
    int rc;
    if ((rc = ensure_train_buffers(lp))) return rc;
    if ((rc = plan_links_f32(lp->op, &links, st))) return rc;
    float4** a = lp->act;
    const size_t n4 = act_bytes(lp, kLpIn) / sizeof(float4);
    if ((rc = forward(lp, links, reinterpret_cast<const float4*>(r_f32[0]), a[Y3], st))) return rc;
    if ((rc = plan_apply_ddagd(lp->op, a[AD4], a[Y3], st))) return rc;
    lp_redot_kernel<<<kRedBlocks, 256, 0, st>>>(a[AD4], reinterpret_cast<const float4*>(r_f32[0]), n4, lp->red);
    lp_sum_kernel<<<1, 256, 0, st>>>(lp->red, kRedBlocks, lp->sc + 2);
    lp_norm_kernel<<<kRedBlocks, 256, 0, st>>>(a[AD4], n4, lp->red);
    lp_sum_kernel<<<1, 256, 0, st>>>(lp->red, kRedBlocks, lp->sc + 3);
    const int n3 = kLpPaths * lp->cin[2] * lp->cout[2];
    lp_rescale_kernel<<<(n3 + 255) / 256, 256, 0, st>>>(lp->master + lp->off[2], n3, lp->sc + 2);
    LP_CHECK(cudaGetLastError());
    lp->prepped = false;
  }
  for (int ep = 0; ep < epochs; ++ep) {
    for (int i = npairs - 1; i > 0; --i) {
      const int j = (int)(splitmix(s) % (uint64_t)(i + 1));
      std::swap(order[i], order[j]);
    }
    double sum = 0.0;
    for (int i = 0; i < npairs; ++i) {
      double l = 0.0;
      int rc = b200_lp_loss_grad(lp, r_f32[order[i]], e_f32[order[i]], &l, stream);
      if (rc) return rc;
      if ((rc = b200_lp_adam_step(lp, lr, stream))) return rc;
      sum += l;
    }
    if (ep == 0 && loss_first) *loss_first = sum / npairs;
    if (ep == epochs - 1 && loss_last) *loss_last = sum / npairs;
  }
  return 0;
}

}  // extern "C"
