// Site-local fifth-dimension kernel, field BLAS, reductions, layout and
// precision conversions of the B200 domain-wall library.
#include "dwf_hop.cuh"
#include "dwf_kernels.h"

#include <type_traits>

namespace b200 {

cudaError_t launch_hop_p0(const HopParams& p, const ChainCoefs& c, cudaStream_t st);
cudaError_t launch_hop_p1(const HopParams& p, const ChainCoefs& c, cudaStream_t st);
cudaError_t launch_hop_p2(const HopParams& p, const ChainCoefs& c, cudaStream_t st);
cudaError_t launch_hop_p3(const HopParams& p, const ChainCoefs& c, cudaStream_t st);

int hop_grid(int ls, int vh) {
  const int g = 32 / ls;
  const int per_block = 4 * g;
  return (vh + per_block - 1) / per_block;
}

int site_s_grid(int ls, int vh) {
  const long n = (long)vh * ls;
  return (int)((n + kSiteSBlock - 1) / kSiteSBlock);
}

cudaError_t launch_hop(int prec, const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (prec) {
    case PREC_F64: return launch_hop_p0(p, c, st);
    case PREC_F32: return launch_hop_p1(p, c, st);
    case PREC_F16: return launch_hop_p2(p, c, st);
    case PREC_BF16: return launch_hop_p3(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------ block reduce
__device__ __forceinline__ void block_reduce_store(double v, double* red) {
  __shared__ double ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) b += ws[w];
    red[blockIdx.x] = b;
  }
}

__device__ __forceinline__ double dev_scale(double c, const double* dev) {
  return dev ? c * (*dev) : c;
}

// ------------------------------------------------------------ sop kernel
// Site-local fifth-dimension map: o1 = ce*A(in) + cx1*X1 + cx2*X2, o2 = B(o1).
template <typename R, int LS, int CHI, int OP>
__device__ __forceinline__ void sop_apply(const ChainCoef<R>& k, const ChainCoef<R>& kee, R* x) {
  switch (OP) {
    case SOP_ID: break;
    case SOP_M5PRE: chain_m5pre<R, LS, CHI>(k, x); break;
    case SOP_M5DAG: chain_m5dag<R, LS, CHI>(k, x); break;
    case SOP_DEE: chain_m5pre<R, LS, CHI>(kee, x); break;
    case SOP_DEE_T: chain_m5dag<R, LS, CHI>(kee, x); break;
    case SOP_LU: chain_lu_inv<R, LS, CHI>(k, x); break;
    case SOP_LUDAG: chain_ludag<R, LS, CHI>(k, x); break;
    case SOP_G5R: chain_g5r<R, LS, CHI>(x); break;
    case SOP_R: {
      R y[LS];
#pragma unroll
      for (int s = 0; s < LS; ++s) y[s] = x[LS - 1 - s];
#pragma unroll
      for (int s = 0; s < LS; ++s) x[s] = y[s];
    } break;
  }
}

template <int LS, int P, int OPA, int OPB>
__global__ void __launch_bounds__(128)
sop_kernel(SopParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k,
           const __grid_constant__ ChainCoef<typename Store<P>::R> kee) {
  using St = Store<P>;
  using R = typename St::R;
  constexpr int G = 32 / LS;
  constexpr int WARPS = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile_all = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane / LS;
  const int s = lane - g * LS;
  const int site = (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.g.vh);
  const size_t vh = p.g.vh;
  R* tile = tile_all + warp * TileWarp<R, LS, G>::v;

  R v[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) v[i] = 0;
  if (active && p.in) St::load(p.in, vh, LS, site, s, v);
  if (OPA != SOP_ID) {
    if (g < G) {
      tile_put(tile_row<R, LS>(tile, g, s), v);
    }
    __syncwarp();
    tile_chiral<R, LS, G>(tile, lane, [&](R* xp, R* xm) {
      sop_apply<R, LS, 0, OPA>(k, kee, xp);
      sop_apply<R, LS, 1, OPA>(k, kee, xm);
    });
    __syncwarp();
    if (g < G) {
      tile_get(tile_row<R, LS>(tile, g, s), v);
    }
  }
  double nrm = 0.0;
  if (active) {
    const R ce = (R)dev_scale(p.ce, p.ce_dev);
#pragma unroll
    for (int i = 0; i < 24; ++i) v[i] *= ce;
    if (p.x1) {
      R xv[24];
      St::load(p.x1, vh, LS, site, s, xv);
      const R c = (R)dev_scale(p.cx1, p.cx1_dev);
#pragma unroll
      for (int i = 0; i < 24; ++i) v[i] = fma(c, xv[i], v[i]);
    }
    if (p.x2) {
      R xv[24];
      St::load(p.x2, vh, LS, site, s, xv);
      const R c = (R)dev_scale(p.cx2, p.cx2_dev);
#pragma unroll
      for (int i = 0; i < 24; ++i) v[i] = fma(c, xv[i], v[i]);
    }
    if (p.out1) St::store(p.out1, vh, LS, site, s, v);
    if (p.red) {
#pragma unroll
      for (int i = 0; i < 24; ++i) nrm += (double)v[i] * (double)v[i];
    }
  }
  if (OPB != SOP_ID) {
    __syncwarp();
    if (g < G) {
      tile_put(tile_row<R, LS>(tile, g, s), v);
    }
    __syncwarp();
    tile_chiral<R, LS, G>(tile, lane, [&](R* xp, R* xm) {
      sop_apply<R, LS, 0, OPB>(k, kee, xp);
      sop_apply<R, LS, 1, OPB>(k, kee, xm);
    });
    __syncwarp();
    if (active) {
      R o2[24];
      tile_get(tile_row<R, LS>(tile, g, s), o2);
      St::store(p.out2, vh, LS, site, s, o2);
    }
  }
  if (p.red) block_reduce_store(nrm, p.red);
}

template <int LS, int P, int OPA, int OPB>
cudaError_t run_sop(const SopParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr size_t smem = sizeof(R) * (4 * TileWarp<R, LS, 32 / LS>::v);
  auto k = sop_kernel<LS, P, OPA, OPB>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const bool dbl = std::is_same<R, double>::value;
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(dbl ? (const void*)&c.d : (const void*)&c.f);
  const ChainCoef<R>& ke = *reinterpret_cast<const ChainCoef<R>*>(dbl ? (const void*)&c.dee_d : (const void*)&c.dee_f);
  k<<<hop_grid(LS, p.g.vh), 128, smem, st>>>(p, kc, ke);
  return cudaGetLastError();
}

template <int LS, int P>
cudaError_t sop_ops(const SopParams& p, const ChainCoefs& c, cudaStream_t st) {
  if (p.opb == SOP_LUDAG) {
    if (p.opa == SOP_G5R) return run_sop<LS, P, SOP_G5R, SOP_LUDAG>(p, c, st);
    return cudaErrorInvalidValue;
  }
  if (p.opb != SOP_ID) return cudaErrorInvalidValue;
  switch (p.opa) {
    case SOP_ID: return run_sop<LS, P, SOP_ID, SOP_ID>(p, c, st);
    case SOP_M5PRE: return run_sop<LS, P, SOP_M5PRE, SOP_ID>(p, c, st);
    case SOP_M5DAG: return run_sop<LS, P, SOP_M5DAG, SOP_ID>(p, c, st);
    case SOP_DEE: return run_sop<LS, P, SOP_DEE, SOP_ID>(p, c, st);
    case SOP_DEE_T: return run_sop<LS, P, SOP_DEE_T, SOP_ID>(p, c, st);
    case SOP_LU: return run_sop<LS, P, SOP_LU, SOP_ID>(p, c, st);
    case SOP_LUDAG: return run_sop<LS, P, SOP_LUDAG, SOP_ID>(p, c, st);
    case SOP_G5R: return run_sop<LS, P, SOP_G5R, SOP_ID>(p, c, st);
    case SOP_R: return run_sop<LS, P, SOP_R, SOP_ID>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int P>
cudaError_t sop_ls(const SopParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (p.g.ls) {
    case 4: return sop_ops<4, P>(p, c, st);
    case 6: return sop_ops<6, P>(p, c, st);
    case 8: return sop_ops<8, P>(p, c, st);
    case 12: return sop_ops<12, P>(p, c, st);
    case 16: return sop_ops<16, P>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_sop(int prec, const SopParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (prec) {
    case PREC_F64: return sop_ls<PREC_F64>(p, c, st);
    case PREC_F32: return sop_ls<PREC_F32>(p, c, st);
    case PREC_F16: return sop_ls<PREC_F16>(p, c, st);
    case PREC_BF16: return sop_ls<PREC_BF16>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------ CG update
template <int LS, int P>
__global__ void __launch_bounds__(128)
cg_update_kernel(CgUpdParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  using St = Store<P>;
  using R = typename St::R;
  constexpr int G = 32 / LS;
  constexpr int WARPS = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile_all = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane / LS;
  const int s = lane - g * LS;
  const int site = (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.g.vh);
  const size_t vh = p.g.vh;
  R* tile = tile_all + warp * TileWarp<R, LS, G>::v;
  R pv[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) pv[i] = 0;
  if (active) {
    const R alpha = (R)(*p.alpha), beta = (R)(*p.beta);
    R xv[24], rv[24];
    St::load(p.x, vh, LS, site, s, xv);
    St::load(p.p, vh, LS, site, s, pv);
    St::load(p.r, vh, LS, site, s, rv);
#pragma unroll
    for (int i = 0; i < 24; ++i) {
      xv[i] = fma(alpha, pv[i], xv[i]);
      pv[i] = fma(beta, pv[i], rv[i]);
    }
    St::store(p.x, vh, LS, site, s, xv);
    St::store(p.p, vh, LS, site, s, pv);
  }
  if (!p.y) return;   // identity pre-factor: the next hop reads p itself
  if (g < G) {
    tile_put(tile_row<R, LS>(tile, g, s), pv);
  }
  __syncwarp();
  tile_chiral<R, LS, G>(tile, lane, [&](R* xp, R* xm) {
    chain_m5pre<R, LS, 0>(k, xp);
    chain_m5pre<R, LS, 1>(k, xm);
  });
  __syncwarp();
  if (active) {
    R o[24];
    tile_get(tile_row<R, LS>(tile, g, s), o);
    St::store(p.y, vh, LS, site, s, o);
  }
}

template <int LS, int P>
cudaError_t run_cgu(const CgUpdParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr size_t smem = sizeof(R) * (4 * TileWarp<R, LS, 32 / LS>::v);
  auto k = cg_update_kernel<LS, P>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(
      std::is_same<R, double>::value ? (const void*)&c.d : (const void*)&c.f);
  k<<<hop_grid(LS, p.g.vh), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

template <int P>
cudaError_t cgu_ls(const CgUpdParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (p.g.ls) {
    case 4: return run_cgu<4, P>(p, c, st);
    case 6: return run_cgu<6, P>(p, c, st);
    case 8: return run_cgu<8, P>(p, c, st);
    case 12: return run_cgu<12, P>(p, c, st);
    case 16: return run_cgu<16, P>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_cg_update(int prec, const CgUpdParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (prec) {
    case PREC_F64: return cgu_ls<PREC_F64>(p, c, st);
    case PREC_F32: return cgu_ls<PREC_F32>(p, c, st);
    case PREC_F16: return cgu_ls<PREC_F16>(p, c, st);
    case PREC_BF16: return cgu_ls<PREC_BF16>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------ multishift
// x_0 -= beta p_0 ; p_0 = r + alpha p_0 ; y_0 = M5pre(p_0) ; |p_0|^2
// for active shifts i >= 1: x_i -= beta_i p_i ; p_i = alpha_i p_i + zeta_i r ; |p_i|^2
// (reference src/lib/Solver/ashiftsolver_CG-tmpl.h:228-262)
template <int LS, int P>
__global__ void __launch_bounds__(128)
ms_update_kernel(MsUpdParams p, const __grid_constant__ ChainCoef<typename Store<P>::R> k) {
  using St = Store<P>;
  using R = typename St::R;
  if (p.st[MS_DONE] != 0.0) return;   // solve finished: replayed iteration is a no-op
  constexpr int G = 32 / LS;
  constexpr int WARPS = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile_all = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane / LS;
  const int s = lane - g * LS;
  const int site = (blockIdx.x * WARPS + warp) * G + g;
  const bool active = (g < G) && (site < p.g.vh);
  const size_t vh = p.g.vh;
  R* tile = tile_all + warp * TileWarp<R, LS, G>::v;
  const int nact = (int)p.st[MS_NACT];
  const R beta = (R)p.st[MS_BETA], alpha = (R)p.st[MS_ALPHA];
  R rv[24], pv[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) { rv[i] = 0; pv[i] = 0; }
  double nrm = 0.0;
  // with p0s set, x_0 is left to the window flush like the other shifts
  const bool defer_x0 = p.p0s != nullptr;
  if (active) {
    R xv[24];
    St::load(p.r, vh, LS, site, s, rv);
    if (!defer_x0) St::load(p.xs[0], vh, LS, site, s, xv);
    St::load(p.ps[0], vh, LS, site, s, pv);
#pragma unroll
    for (int i = 0; i < 24; ++i) {
      if (!defer_x0) xv[i] = fma(-beta, pv[i], xv[i]);
      pv[i] = fma(alpha, pv[i], rv[i]);
      nrm += (double)pv[i] * (double)pv[i];
    }
    if (!defer_x0) St::store(p.xs[0], vh, LS, site, s, xv);
    St::store(p.ps[0], vh, LS, site, s, pv);
  }
  if (p.y0) {         // null: identity pre-factor, the next hop reads p_0
    if (g < G) {
      tile_put(tile_row<R, LS>(tile, g, s), pv);
    }
    __syncwarp();
    tile_chiral<R, LS, G>(tile, lane, [&](R* xp, R* xm) {
      chain_m5pre<R, LS, 0>(k, xp);
      chain_m5pre<R, LS, 1>(k, xm);
    });
    __syncwarp();
    if (active) {
      R o[24];
      tile_get(tile_row<R, LS>(tile, g, s), o);
      St::store(p.y0, vh, LS, site, s, o);
    }
  }
  block_reduce_store(nrm, p.red);
  if (p.win) {
    // windowed mode: keep this iteration's residual; the shifts follow later
    if (active) St::store(p.win[(int)p.st[MS_WIN]], vh, LS, site, s, rv);
    return;
  }
  for (int ish = 1; ish < nact; ++ish) {
    __syncthreads();
    const R bs = (R)p.st[MS_N + MSA_BETAS * kMaxShift + ish];
    const R as = (R)p.st[MS_N + MSA_ALPHAS * kMaxShift + ish];
    const R zt = (R)p.st[MS_N + MSA_ZETA * kMaxShift + ish];
    double n2 = 0.0;
    if (active) {
      R xv[24], qv[24];
      St::load(p.xs[ish], vh, LS, site, s, xv);
      St::load(p.ps[ish], vh, LS, site, s, qv);
#pragma unroll
      for (int i = 0; i < 24; ++i) {
        xv[i] = fma(-bs, qv[i], xv[i]);
        qv[i] = fma(as, qv[i], zt * rv[i]);
        n2 += (double)qv[i] * (double)qv[i];
      }
      St::store(p.xs[ish], vh, LS, site, s, xv);
      St::store(p.ps[ish], vh, LS, site, s, qv);
    }
    block_reduce_store(n2, p.red + (size_t)ish * p.nblocks);
  }
}

template <int LS, int P>
cudaError_t run_msu(const MsUpdParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr size_t smem = sizeof(R) * (4 * TileWarp<R, LS, 32 / LS>::v);
  auto k = ms_update_kernel<LS, P>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(
      std::is_same<R, double>::value ? (const void*)&c.d : (const void*)&c.f);
  k<<<hop_grid(LS, p.g.vh), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

template <int P>
cudaError_t msu_ls(const MsUpdParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (p.g.ls) {
    case 4: return run_msu<4, P>(p, c, st);
    case 6: return run_msu<6, P>(p, c, st);
    case 8: return run_msu<8, P>(p, c, st);
    case 12: return run_msu<12, P>(p, c, st);
    case 16: return run_msu<16, P>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_ms_update(int prec, const MsUpdParams& p, const ChainCoefs& c, cudaStream_t st) {
  switch (prec) {
    case PREC_F64: return msu_ls<PREC_F64>(p, c, st);
    case PREC_F32: return msu_ls<PREC_F32>(p, c, st);
    case PREC_F16: return msu_ls<PREC_F16>(p, c, st);
    case PREC_BF16: return msu_ls<PREC_BF16>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

// deterministic block sum of partials[0..n) into shared memory, returned to thread 0
__device__ double block_sum_partials(const double* partials, int n) {
  __shared__ double ws[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w];
  return s;
}

__global__ void ms_scalar_kernel(int step, const double* partials, int n, double* st, int nshift) {
  if (st[MS_DONE] != 0.0) return;     // solve finished: a replayed iteration is a no-op
  double* zeta1 = st + MS_N + MSA_ZETA1 * kMaxShift;
  double* zeta2 = st + MS_N + MSA_ZETA2 * kMaxShift;
  double* csh2 = st + MS_N + MSA_CSH2 * kMaxShift;
  double* betas = st + MS_N + MSA_BETAS * kMaxShift;
  double* alphas = st + MS_N + MSA_ALPHAS * kMaxShift;
  double* zeta = st + MS_N + MSA_ZETA * kMaxShift;
  double* pp = st + MS_N + MSA_PP * kMaxShift;
  if (step == MSS_BETA) {
    const double pq = block_sum_partials(partials, n);
    if (threadIdx.x == 0) {
      st[MS_PQ] = pq;
      const double pa = pq + st[MS_SIGMA0] * st[MS_PP0];
      st[MS_BETA] = -st[MS_RR] / pa;
    }
  } else if (step == MSS_ALPHA) {
    const double rr = block_sum_partials(partials, n);
    if (threadIdx.x == 0) {
      const double beta = st[MS_BETA];
      const double alpha = rr / st[MS_RR];
      st[MS_ALPHA] = alpha;
      st[MS_RR_NEW] = rr;
      pp[0] = rr;
      const double alpha_h = 1.0 + st[MS_ALPHA_P] * beta / st[MS_BETA_P];
      const int nact = (int)st[MS_NACT];
      for (int i = 1; i < nact; ++i) {
        double z = (alpha_h - csh2[i] * beta) / zeta1[i] + (1.0 - alpha_h) / zeta2[i];
        z = 1.0 / z;
        const double zr = z / zeta1[i];
        betas[i] = beta * zr;
        alphas[i] = alpha * zr * zr;
        zeta[i] = z;
        zeta2[i] = zeta1[i];
        zeta1[i] = z;
      }
      if (st[MS_WSIZE] > 0.0) {
        // deferred form of x_i -= beta_i p_i ; p_i = alpha_i p_i + zeta_i r_w,
        // and |p_i|^2 by its recurrence (the new residual is orthogonal to
        // every earlier direction): pp_i = zeta_i^2 |r|^2 + alpha_i^2 pp_i
        const int w = (int)st[MS_WIN];
        const double rrn = rr * st[MS_SNORM];
        // shift 0 too (beta, alpha, zeta = 1): its p_0 is updated every
        // iteration, its x_0 by the flush where that is deferred
        for (int i = 0; i < nact; ++i) {
          double* pc = st + kMsCoef + i * (kMaxWin + 1);
          double* xc = st + kMsXCoef + i * (kMaxWin + 1);
          const double bs = i ? betas[i] : beta, as = i ? alphas[i] : alpha, zt = i ? zeta[i] : 1.0;
          for (int j = 0; j <= w; ++j) {
            xc[j] -= bs * pc[j];
            pc[j] *= as;
          }
          pc[1 + w] = zt;
          if (i) pp[i] = zt * zt * rrn + as * as * pp[i];
        }
      }
      st[MS_ALPHA_P] = alpha;
      st[MS_BETA_P] = beta;
      st[MS_RR] = rr;
    }
  } else {  // MSS_PRUNE
    const bool windowed = st[MS_WSIZE] > 0.0;
    const int nact = (int)st[MS_NACT];
    for (int i = 0; i < (windowed ? 1 : nact); ++i) {
      const double v = block_sum_partials(partials + (size_t)i * n, n);
      if (threadIdx.x == 0) {
        if (i == 0) st[MS_PP0] = v;
        else pp[i] = v * st[MS_SNORM];
      }
    }
    if (threadIdx.x == 0) {
      int ish1 = nact;
      for (int i = nact - 1; i >= 0; --i) {
        if (pp[i] > st[MS_TOL2]) { ish1 = i + 1; break; }
      }
      st[MS_NACT] = (double)ish1;
      if (windowed) st[MS_WIN] = st[MS_WIN] + 1.0;
      // end of an iteration: count it and decide on the device whether the
      // solve is over, so that iterations can be replayed without the host
      const double it = st[MS_ITER] + 1.0;
      st[MS_ITER] = it;
      const double rel = st[MS_RR] * st[MS_SNORM];
      if (!(rel == rel)) st[MS_DONE] = 2.0;
      else if (rel < st[MS_TOL2]) st[MS_DONE] = 1.0;
      else if (it >= st[MS_MAXITER]) st[MS_DONE] = 3.0;
    }
  }
}

cudaError_t launch_ms_scalar(int step, const double* partials, int n, double* st, int nshift,
                             cudaStream_t stream) {
  ms_scalar_kernel<<<1, 1024, 0, stream>>>(step, partials, n, st, nshift);
  return cudaGetLastError();
}

// Windowed multishift: the window is applied when it is full or when the
// solve has ended with residuals still pending.
__device__ __forceinline__ bool ms_window_due(const double* st) {
  const double w = st[MS_WIN];
  return w > 0.0 && (w >= st[MS_WSIZE] || st[MS_DONE] != 0.0);
}

// p_i = PC0 p_i + sum_l PC_l r_l ; x_i += XC0 p_i(old) + sum_l XC_l r_l for
// every shift active in the window; flat over the FP64 field as double2.
__global__ void __launch_bounds__(256) ms_flush_kernel(MsUpdParams p, long n2) {
  const double* st = p.st;
  if (!ms_window_due(st)) return;
  __shared__ double cs[2 * kMaxShift * (kMaxWin + 1)];
  const int w = (int)st[MS_WIN];
  const int nsh = (int)st[MS_NACTW];
  for (int i = threadIdx.x; i < 2 * kMaxShift * (kMaxWin + 1); i += blockDim.x) cs[i] = st[kMsCoef + i];
  __syncthreads();
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (long)gridDim.x * blockDim.x) {
    double2 rv[kMaxWin];
#pragma unroll
    for (int l = 0; l < kMaxWin; ++l)
      if (l < w) rv[l] = __ldcs(reinterpret_cast<const double2*>(p.win[l]) + e);
    if (p.p0s) {
      // x_0 += XC0 p_0(window start) + sum_l XC_l r_l; p_0 itself is current,
      // and becomes the next window's start
      const double* xc = cs + kMaxShift * (kMaxWin + 1);
      double2* x0p = reinterpret_cast<double2*>(p.xs[0]) + e;
      double2* s0p = reinterpret_cast<double2*>(p.p0s) + e;
      const double2 ps0 = __ldcs(s0p);
      const double2 pc0 = __ldcs(reinterpret_cast<const double2*>(p.ps[0]) + e);
      double2 x = __ldcs(x0p);
      x.x = fma(xc[0], ps0.x, x.x); x.y = fma(xc[0], ps0.y, x.y);
#pragma unroll
      for (int l = 0; l < kMaxWin; ++l) {
        if (l < w) { x.x = fma(xc[1 + l], rv[l].x, x.x); x.y = fma(xc[1 + l], rv[l].y, x.y); }
      }
      __stcs(x0p, x);
      __stcs(s0p, pc0);
    }
    // the next shift's p_i, x_i are loaded while this shift is combined, so
    // every thread keeps two shifts' loads in flight
    double2 pn = make_double2(0.0, 0.0), xn = pn;
    if (nsh > 1) {
      pn = __ldcs(reinterpret_cast<const double2*>(p.ps[1]) + e);
      xn = __ldcs(reinterpret_cast<const double2*>(p.xs[1]) + e);
    }
    for (int i = 1; i < nsh; ++i) {
      const double* pc = cs + i * (kMaxWin + 1);
      const double* xc = cs + kMaxShift * (kMaxWin + 1) + i * (kMaxWin + 1);
      double2* pp = reinterpret_cast<double2*>(p.ps[i]) + e;
      double2* xp = reinterpret_cast<double2*>(p.xs[i]) + e;
      const double2 p0 = pn;
      double2 x = xn;
      if (i + 1 < nsh) {
        pn = __ldcs(reinterpret_cast<const double2*>(p.ps[i + 1]) + e);
        xn = __ldcs(reinterpret_cast<const double2*>(p.xs[i + 1]) + e);
      }
      double2 q;
      q.x = pc[0] * p0.x; q.y = pc[0] * p0.y;
      x.x = fma(xc[0], p0.x, x.x); x.y = fma(xc[0], p0.y, x.y);
#pragma unroll
      for (int l = 0; l < kMaxWin; ++l) {
        if (l < w) {
          q.x = fma(pc[1 + l], rv[l].x, q.x); q.y = fma(pc[1 + l], rv[l].y, q.y);
          x.x = fma(xc[1 + l], rv[l].x, x.x); x.y = fma(xc[1 + l], rv[l].y, x.y);
        }
      }
      __stcs(pp, q);
      __stcs(xp, x);
    }
  }
}

__global__ void ms_window_reset_kernel(double* st) {
  if (threadIdx.x != 0 || !ms_window_due(st)) return;
  for (int i = 0; i < kMaxShift; ++i) {
    double* pc = st + kMsCoef + i * (kMaxWin + 1);
    double* xc = st + kMsXCoef + i * (kMaxWin + 1);
    for (int j = 0; j <= kMaxWin; ++j) { pc[j] = 0.0; xc[j] = 0.0; }
    pc[0] = 1.0;
  }
  st[MS_WIN] = 0.0;
  st[MS_NACTW] = st[MS_NACT];
}

cudaError_t launch_ms_flush(const MsUpdParams& p, cudaStream_t st) {
  const long n2 = (long)12 * p.g.vh * p.g.ls;      // FP64 field as double2
  long blocks = (n2 + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  ms_flush_kernel<<<(int)blocks, 256, 0, st>>>(p, n2);
  return cudaGetLastError();
}

cudaError_t launch_ms_window_reset(double* st, cudaStream_t stream) {
  ms_window_reset_kernel<<<1, 32, 0, stream>>>(st);
  return cudaGetLastError();
}

// ------------------------------------------------------------ BLAS
template <int P>
__global__ void axpby_kernel(Geom g, void* y, const void* x, double a, const double* a_dev,
                             double b, const double* b_dev) {
  using St = Store<P>;
  using R = typename St::R;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)g.vh * g.ls) return;
  const int site = (int)(idx / g.ls), s = (int)(idx % g.ls);
  const R av = (R)dev_scale(a, a_dev), bv = (R)dev_scale(b, b_dev);
  R yv[24], xv[24];
  if (bv != R(0)) St::load(y, g.vh, g.ls, site, s, yv);
  else {
#pragma unroll
    for (int i = 0; i < 24; ++i) yv[i] = 0;
  }
  if (x && av != R(0)) {
    St::load(x, g.vh, g.ls, site, s, xv);
#pragma unroll
    for (int i = 0; i < 24; ++i) yv[i] = fma(av, xv[i], bv * yv[i]);
  } else {
#pragma unroll
    for (int i = 0; i < 24; ++i) yv[i] = bv * yv[i];
  }
  St::store(y, g.vh, g.ls, site, s, yv);
}

template <int P>
__global__ void dot_kernel(Geom g, const void* x, const void* y, double* red) {
  using St = Store<P>;
  using R = typename St::R;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (idx < (long)g.vh * g.ls) {
    const int site = (int)(idx / g.ls), s = (int)(idx % g.ls);
    R xv[24], yv[24];
    St::load(x, g.vh, g.ls, site, s, xv);
    if (y == x) {
#pragma unroll
      for (int i = 0; i < 24; ++i) acc += (double)xv[i] * (double)xv[i];
    } else {
      St::load(y, g.vh, g.ls, site, s, yv);
#pragma unroll
      for (int i = 0; i < 24; ++i) acc += (double)xv[i] * (double)yv[i];
    }
  }
  block_reduce_store(acc, red);
}

template <int PO, int PI>
__global__ void convert_kernel(Geom g, void* out, const void* in) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)g.vh * g.ls) return;
  const int site = (int)(idx / g.ls), s = (int)(idx % g.ls);
  typename Store<PI>::R v[24];
  typename Store<PO>::R w[24];
  Store<PI>::load(in, g.vh, g.ls, site, s, v);
#pragma unroll
  for (int i = 0; i < 24; ++i) w[i] = (typename Store<PO>::R)v[i];
  Store<PO>::store(out, g.vh, g.ls, site, s, w);
}

// corelib Field(24, Vh, Ls): ri + 2*(c + 3*sp) + 24*(site + Vh*s)
template <int P>
__global__ void from_corelib_kernel(Geom g, void* out, const double* in) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)g.vh * g.ls) return;
  const int site = (int)(idx / g.ls), s = (int)(idx % g.ls);
  const double* src = in + 24 * ((size_t)site + (size_t)g.vh * s);
  typename Store<P>::R v[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) v[i] = (typename Store<P>::R)src[i];
  Store<P>::store(out, g.vh, g.ls, site, s, v);
}

// Parity ieo of a full-lattice lexical spinor Field(24, Nvol, Ls), index
// in + 24*(x + Nx*(y + Ny*(z + Nz*t)) + Nvol*s), into the device layout of the
// half lattice (Index_eo::convertField, src/lib/Field/index_eo.cpp).
template <int P>
__global__ void from_lex_parity_kernel(Geom g, void* out, const double* lex, int ieo) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)g.vh * g.ls) return;
  const int site = (int)(idx / g.ls), s = (int)(idx % g.ls);
  const int ix2 = site % g.nx2;
  const int yzt = site / g.nx2;
  const int y = yzt % g.ny, z = (yzt / g.ny) % g.nz, t = yzt / (g.ny * g.nz);
  const int x = 2 * ix2 + ((ieo + y + z + t) & 1);
  const size_t lexsite = x + (size_t)(2 * g.nx2) * (y + (size_t)g.ny * (z + (size_t)g.nz * t));
  const double* src = lex + 24 * (lexsite + (size_t)2 * g.vh * s);
  typename Store<P>::R v[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) v[i] = (typename Store<P>::R)src[i];
  Store<P>::store(out, g.vh, g.ls, site, s, v);
}

template <int P>
__global__ void to_corelib_kernel(Geom g, double* out, const void* in) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)g.vh * g.ls) return;
  const int site = (int)(idx / g.ls), s = (int)(idx % g.ls);
  typename Store<P>::R v[24];
  Store<P>::load(in, g.vh, g.ls, site, s, v);
  double* dst = out + 24 * ((size_t)site + (size_t)g.vh * s);
#pragma unroll
  for (int i = 0; i < 24; ++i) dst[i] = (double)v[i];
}

// links: out index (ieo + 2*mu)*Vh + site_eo  (reference m_Ueo ordering,
// src/lib_alt_Accel/Fopr/afopr_Domainwall_5din_eo-tmpl.h:140-141).
// The full-record formats (LINK_F64_18, LINK_F32_18, LINK_F16_18:
// LinkLoad::kFolded) carry two constant factors of the hop: 2 on every t link
// (the (1 -+ gamma_4) projection), and the boundary phase: links U_mu(x) with
// x_mu = L_mu - 1 are stored times bc[mu], which is the factor the reference
// applies to both hops across that edge (forward from x, backward from
// x + mu).  Real phases only (bc is an integer vector).
struct LinkPhase { double bc[4]; };

template <int LF>
__global__ void links_kernel(Geom g, void* out, const double* u, LinkPhase ph) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)8 * g.vh) return;
  const int site = (int)(idx % g.vh);
  const int pm = (int)(idx / g.vh);       // ieo + 2*mu
  const int ieo = pm & 1, mu = pm >> 1;
  const int ix2 = site % g.nx2;
  const int iyzt = site / g.nx2;
  const int y = iyzt % g.ny;
  const int z = (iyzt / g.ny) % g.nz;
  const int t = iyzt / (g.ny * g.nz);
  const int x = 2 * ix2 + ((ieo + y + z + t) & 1);
  const int nx = 2 * g.nx2;
  const size_t lex = x + (size_t)nx * (y + (size_t)g.ny * (z + (size_t)g.nz * t));
  const size_t vol = (size_t)2 * g.vh;
  const double* m = u + 18 * (lex + vol * mu);
  const int cmu = (mu == 0) ? x : (mu == 1) ? y : (mu == 2) ? z : t;
  const int ext = (mu == 0) ? nx : (mu == 1) ? g.ny : (mu == 2) ? g.nz : g.nt;
  // folded formats only: boundary phase, and the factor 2 of the t projection
  const double f = ((cmu == ext - 1) ? ph.bc[mu] : 1.0) * (mu == 3 ? 2.0 : 1.0);
  if (LF == LINK_F64_18) {
    double2* o = reinterpret_cast<double2*>(out) + idx * 9;
    for (int j = 0; j < 9; ++j) o[j] = make_double2(f * m[2 * j], f * m[2 * j + 1]);
  } else if (LF == LINK_F32_18) {
    float* o = reinterpret_cast<float*>(reinterpret_cast<float4*>(out) + idx * 5);
    for (int j = 0; j < 18; ++j) o[j] = (float)(f * m[j]);
    o[18] = 0.f; o[19] = 0.f;
  } else if (LF == LINK_F16_18) {
    uint4* o = reinterpret_cast<uint4*>(out) + idx * 3;
    unsigned int w[12];
    for (int j = 0; j < 9; ++j) w[j] = HalfOps<__half>::from2((float)(f * m[2 * j]), (float)(f * m[2 * j + 1]));
    w[9] = 0u; w[10] = 0u; w[11] = 0u;
    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
    o[2] = make_uint4(w[8], w[9], w[10], w[11]);
  } else if (LF == LINK_F64_12) {
    double2* o = reinterpret_cast<double2*>(out) + idx * 6;
    for (int j = 0; j < 6; ++j) o[j] = make_double2(m[2 * j], m[2 * j + 1]);
  } else if (LF == LINK_F32_12) {
    float4* o = reinterpret_cast<float4*>(out) + idx * 3;
    for (int j = 0; j < 3; ++j)
      o[j] = make_float4((float)m[4 * j], (float)m[4 * j + 1], (float)m[4 * j + 2], (float)m[4 * j + 3]);
  } else {
    uint4* o = reinterpret_cast<uint4*>(out) + idx * 2;
    unsigned int w[8];
    for (int j = 0; j < 6; ++j) w[j] = HalfOps<__half>::from2((float)m[2 * j], (float)m[2 * j + 1]);
    w[6] = 0u; w[7] = 0u;
    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

size_t link_bytes(int lf, size_t vh) {
  const size_t n = 8 * vh;
  switch (lf) {
    case LINK_F64_18: return n * 9 * 16;
    case LINK_F64_12: return n * 6 * 16;
    case LINK_F32_12: return n * 3 * 16;
    case LINK_F32_18: return n * 5 * 16;
    case LINK_F16_18: return n * 3 * 16;
    default: return n * 2 * 16;
  }
}

__global__ void finalize_kernel(const double* partials, int n, double* out, int op) {
  __shared__ double ws[32];
  double v = 0.0;
  // fixed assignment of partials to threads -> deterministic result
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w];
    if (op == FIN_SUM) {
      out[0] = s;
    } else if (op == FIN_CG_ALPHA) {
      out[SC_PQ] = s;
      out[SC_ALPHA] = out[SC_RR] / s;
    } else if (op == FIN_CG_BETA) {
      out[SC_BETA] = s / out[SC_RR];
      out[SC_RR] = s;
    }
  }
}

// ------------------------------------------------------------ launchers
#define B200_PREC_SWITCH(prec, FN)                          \
  switch (prec) {                                           \
    case PREC_F64: FN(PREC_F64); break;                     \
    case PREC_F32: FN(PREC_F32); break;                     \
    case PREC_F16: FN(PREC_F16); break;                     \
    case PREC_BF16: FN(PREC_BF16); break;                   \
    default: return cudaErrorInvalidValue;                  \
  }

cudaError_t launch_axpby(int prec, const Geom& g, void* y, const void* x, double a,
                         const double* a_dev, double b, const double* b_dev, cudaStream_t st) {
  const int grid = site_s_grid(g.ls, g.vh);
#define L(PP) axpby_kernel<PP><<<grid, kSiteSBlock, 0, st>>>(g, y, x, a, a_dev, b, b_dev)
  B200_PREC_SWITCH(prec, L)
#undef L
  return cudaGetLastError();
}

cudaError_t launch_dot(int prec, const Geom& g, const void* x, const void* y, double* red,
                       cudaStream_t st) {
  const int grid = site_s_grid(g.ls, g.vh);
#define L(PP) dot_kernel<PP><<<grid, kSiteSBlock, 0, st>>>(g, x, y, red)
  B200_PREC_SWITCH(prec, L)
#undef L
  return cudaGetLastError();
}

cudaError_t launch_convert(int pout, void* out, int pin, const void* in, const Geom& g,
                           cudaStream_t st) {
  const int grid = site_s_grid(g.ls, g.vh);
#define L2(PO, PI) convert_kernel<PO, PI><<<grid, kSiteSBlock, 0, st>>>(g, out, in)
#define LIN(PO)                                             \
  switch (pin) {                                            \
    case PREC_F64: L2(PO, PREC_F64); break;                 \
    case PREC_F32: L2(PO, PREC_F32); break;                 \
    case PREC_F16: L2(PO, PREC_F16); break;                 \
    case PREC_BF16: L2(PO, PREC_BF16); break;               \
    default: return cudaErrorInvalidValue;                  \
  }
  B200_PREC_SWITCH(pout, LIN)
#undef LIN
#undef L2
  return cudaGetLastError();
}

cudaError_t launch_from_corelib(int prec, void* out, const double* in_dev, const Geom& g,
                                cudaStream_t st) {
  const int grid = site_s_grid(g.ls, g.vh);
#define L(PP) from_corelib_kernel<PP><<<grid, kSiteSBlock, 0, st>>>(g, out, in_dev)
  B200_PREC_SWITCH(prec, L)
#undef L
  return cudaGetLastError();
}

cudaError_t launch_from_lex_parity(int prec, void* out, const double* lex_dev, int ieo, const Geom& g,
                                  cudaStream_t st) {
  const int grid = site_s_grid(g.ls, g.vh);
#define L(PP) from_lex_parity_kernel<PP><<<grid, kSiteSBlock, 0, st>>>(g, out, lex_dev, ieo)
  B200_PREC_SWITCH(prec, L)
#undef L
  return cudaGetLastError();
}

cudaError_t launch_to_corelib(int prec, double* out_dev, const void* in, const Geom& g,
                              cudaStream_t st) {
  const int grid = site_s_grid(g.ls, g.vh);
#define L(PP) to_corelib_kernel<PP><<<grid, kSiteSBlock, 0, st>>>(g, out_dev, in)
  B200_PREC_SWITCH(prec, L)
#undef L
  return cudaGetLastError();
}

cudaError_t launch_links_from_lex(int lf, void* out, const double* u_lex_dev, const Geom& g,
                                  const int bc[4], cudaStream_t st) {
  const long n = 8L * g.vh;
  const int grid = (int)((n + 127) / 128);
  LinkPhase ph;
  for (int mu = 0; mu < 4; ++mu) ph.bc[mu] = (double)bc[mu];
  switch (lf) {
    case LINK_F64_18: links_kernel<LINK_F64_18><<<grid, 128, 0, st>>>(g, out, u_lex_dev, ph); break;
    case LINK_F64_12: links_kernel<LINK_F64_12><<<grid, 128, 0, st>>>(g, out, u_lex_dev, ph); break;
    case LINK_F32_12: links_kernel<LINK_F32_12><<<grid, 128, 0, st>>>(g, out, u_lex_dev, ph); break;
    case LINK_F16_12: links_kernel<LINK_F16_12><<<grid, 128, 0, st>>>(g, out, u_lex_dev, ph); break;
    case LINK_F32_18: links_kernel<LINK_F32_18><<<grid, 128, 0, st>>>(g, out, u_lex_dev, ph); break;
    case LINK_F16_18: links_kernel<LINK_F16_18><<<grid, 128, 0, st>>>(g, out, u_lex_dev, ph); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_finalize(const double* partials, int n, double* out, int op, cudaStream_t st) {
  finalize_kernel<<<1, 1024, 0, st>>>(partials, n, out, op);
  return cudaGetLastError();
}

// ------------------------------------------------------------ complex BLAS (f64)
// The FP64 field is an array of n complex numbers (double2).  Used by the
// flexible CG, whose step sizes are complex once the preconditioner is not
// Hermitian.
namespace {
constexpr int kZBlocks = 296;

__global__ void zdot_kernel(const double2* x, const double2* y, size_t n, double2* partial) {
  __shared__ double sr[256], si[256];
  double re = 0.0, im = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = x[i], b = y[i];
    re = fma(a.x, b.x, re); re = fma(a.y, b.y, re);   // conj(a) * b
    im = fma(a.x, b.y, im); im = fma(-a.y, b.x, im);
  }
  sr[threadIdx.x] = re; si[threadIdx.x] = im;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sr[threadIdx.x] += sr[threadIdx.x + o]; si[threadIdx.x] += si[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(sr[0], si[0]);
}

// out = sum of partials; with den != nullptr, out = sign * sum / Re(den[0]).
__global__ void zfinal_kernel(const double2* partial, int nb, double2* out, const double2* den,
                              double sign) {
  __shared__ double sr[256], si[256];
  double re = 0.0, im = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) { re += partial[i].x; im += partial[i].y; }
  sr[threadIdx.x] = re; si[threadIdx.x] = im;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sr[threadIdx.x] += sr[threadIdx.x + o]; si[threadIdx.x] += si[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double2 v = make_double2(sr[0], si[0]);
    if (den) {
      const double d = den[0].x;
      const double f = (d != 0.0) ? sign / d : 0.0;
      v = make_double2(f * v.x, f * v.y);
    }
    out[0] = v;
  }
}

// y += c * x  (c complex, read from the device)
__global__ void zaxpy_kernel(double2* y, const double2* x, size_t n, const double2* c) {
  const double2 cc = c[0];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = x[i];
    double2 v = y[i];
    v.x = fma(cc.x, a.x, v.x); v.x = fma(-cc.y, a.y, v.x);
    v.y = fma(cc.x, a.y, v.y); v.y = fma(cc.y, a.x, v.y);
    y[i] = v;
  }
}

// x += alpha p ; r -= alpha q ; per-block |r|^2
__global__ void zcg_update_kernel(double2* x, double2* r, const double2* p, const double2* q, size_t n,
                                  const double2* alpha, double* partial) {
  __shared__ double sh[256];
  const double2 a = alpha[0];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 pv = p[i], qv = q[i];
    double2 xv = x[i], rv = r[i];
    xv.x = fma(a.x, pv.x, xv.x); xv.x = fma(-a.y, pv.y, xv.x);
    xv.y = fma(a.x, pv.y, xv.y); xv.y = fma(a.y, pv.x, xv.y);
    rv.x = fma(-a.x, qv.x, rv.x); rv.x = fma(a.y, qv.y, rv.x);
    rv.y = fma(-a.x, qv.y, rv.y); rv.y = fma(-a.y, qv.x, rv.y);
    x[i] = xv; r[i] = rv;
    acc = fma(rv.x, rv.x, acc); acc = fma(rv.y, rv.y, acc);
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}
// partial[blk * m + j] = sum over the block's elements of conj(Q_j) z, j < m
__global__ void zmdot_kernel(ZMulti q, const double2* z, size_t n, double2* partial) {
  __shared__ double sr[kZMaxMulti][128], si[kZMaxMulti][128];
  double re[kZMaxMulti], im[kZMaxMulti];
#pragma unroll
  for (int j = 0; j < kZMaxMulti; ++j) { re[j] = 0.0; im[j] = 0.0; }
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 b = z[i];
#pragma unroll
    for (int j = 0; j < kZMaxMulti; ++j) {
      if (j < q.m) {
        const double2 a = q.v[j][i];
        re[j] = fma(a.x, b.x, re[j]); re[j] = fma(a.y, b.y, re[j]);
        im[j] = fma(a.x, b.y, im[j]); im[j] = fma(-a.y, b.x, im[j]);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kZMaxMulti; ++j) { sr[j][threadIdx.x] = re[j]; si[j][threadIdx.x] = im[j]; }
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int j = 0; j < kZMaxMulti; ++j) {
        sr[j][threadIdx.x] += sr[j][threadIdx.x + o];
        si[j][threadIdx.x] += si[j][threadIdx.x + o];
      }
    __syncthreads();
  }
  if (threadIdx.x < q.m) partial[blockIdx.x * kZMaxMulti + threadIdx.x] = make_double2(sr[threadIdx.x][0], si[threadIdx.x][0]);
}

// out[j] = sign * (sum over blocks of partial[.][j]) / Re(den[j]), j < m
__global__ void zmfinal_kernel(const double2* partial, int nb, int m, double2* out, const double2* den,
                               double sign) {
  const int j = threadIdx.x;
  if (j >= m) return;
  double re = 0.0, im = 0.0;
  for (int b = 0; b < nb; ++b) { re += partial[b * kZMaxMulti + j].x; im += partial[b * kZMaxMulti + j].y; }
  const double d = den[j].x;
  const double f = (d != 0.0) ? sign / d : 0.0;
  out[j] = make_double2(f * re, f * im);
}

// y = z + sum_j c[j] * P_j
__global__ void zmaxpy_kernel(double2* y, const double2* z, ZMulti pv, const double2* c, size_t n) {
  double2 cc[kZMaxMulti];
#pragma unroll
  for (int j = 0; j < kZMaxMulti; ++j) cc[j] = (j < pv.m) ? c[j] : make_double2(0.0, 0.0);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double2 v = z[i];
#pragma unroll
    for (int j = 0; j < kZMaxMulti; ++j) {
      if (j < pv.m) {
        const double2 a = pv.v[j][i];
        v.x = fma(cc[j].x, a.x, v.x); v.x = fma(-cc[j].y, a.y, v.x);
        v.y = fma(cc[j].x, a.y, v.y); v.y = fma(cc[j].y, a.x, v.y);
      }
    }
    y[i] = v;
  }
}
}  // namespace

int zblas_blocks() { return kZBlocks; }

cudaError_t launch_zmdot(const ZMulti& q, const void* z, size_t n, void* partial, void* out,
                         const void* den, double sign, cudaStream_t st) {
  if (q.m < 1 || q.m > kZMaxMulti) return cudaErrorInvalidValue;
  zmdot_kernel<<<kZBlocks, 128, 0, st>>>(q, (const double2*)z, n, (double2*)partial);
  zmfinal_kernel<<<1, 32, 0, st>>>((const double2*)partial, kZBlocks, q.m, (double2*)out,
                                    (const double2*)den, sign);
  return cudaGetLastError();
}

cudaError_t launch_zmaxpy(void* y, const void* z, const ZMulti& pv, const void* c, size_t n,
                          cudaStream_t st) {
  if (pv.m < 1 || pv.m > kZMaxMulti) return cudaErrorInvalidValue;
  zmaxpy_kernel<<<kZBlocks, 256, 0, st>>>((double2*)y, (const double2*)z, pv, (const double2*)c, n);
  return cudaGetLastError();
}

cudaError_t launch_zdot(const void* x, const void* y, size_t n, void* partial, void* out,
                        const void* den, double sign, cudaStream_t st) {
  zdot_kernel<<<kZBlocks, 256, 0, st>>>((const double2*)x, (const double2*)y, n, (double2*)partial);
  zfinal_kernel<<<1, 256, 0, st>>>((const double2*)partial, kZBlocks, (double2*)out, (const double2*)den, sign);
  return cudaGetLastError();
}

cudaError_t launch_zaxpy(void* y, const void* x, size_t n, const void* c, cudaStream_t st) {
  zaxpy_kernel<<<kZBlocks, 256, 0, st>>>((double2*)y, (const double2*)x, n, (const double2*)c);
  return cudaGetLastError();
}

cudaError_t launch_zcg_update(void* x, void* r, const void* p, const void* q, size_t n,
                              const void* alpha, double* partial, cudaStream_t st) {
  zcg_update_kernel<<<kZBlocks, 256, 0, st>>>((double2*)x, (double2*)r, (const double2*)p,
                                              (const double2*)q, n, (const double2*)alpha, partial);
  return cudaGetLastError();
}

}  // namespace b200
