// Explicit instantiations of the fused hop kernel for one storage precision.
// Compiled once per precision with -DB200_PREC=<0..3> (see the Makefile).
#include "dwf_hop.cuh"
#include "dwf_kernels.h"

#include <type_traits>

#ifndef B200_PREC
#error "B200_PREC must be defined"
#endif

namespace b200 {

template <int P> struct DefaultLink;
template <> struct DefaultLink<PREC_F64> { static constexpr int v = LINK_F64_18; };
template <> struct DefaultLink<PREC_F32> { static constexpr int v = LINK_F32_18; };
template <> struct DefaultLink<PREC_F16> { static constexpr int v = LINK_F16_18; };
template <> struct DefaultLink<PREC_BF16> { static constexpr int v = LINK_F16_18; };

namespace {

template <int LS, int P, int EPI, int FK, int MB>
cudaError_t run_mb(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr int LF = DefaultLink<P>::v;
  constexpr size_t smem = hop_smem_bytes<LS, P>();
  auto k = dwf_hop_kernel<LS, P, LF, EPI, FK, MB>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(
      std::is_same<R, double>::value ? (const void*)&c.d : (const void*)&c.f);
  k<<<hop_grid(LS, p.site_end - p.site0), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

template <int LS, int P, int EPI, int FK, int S, int MB>
cudaError_t run_tma(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr int LF = DefaultLink<P>::v;
  constexpr size_t smem = hop_tma_smem_bytes<LS, P, LF, S>();
  auto k = dwf_hop_tma_kernel<LS, P, LF, EPI, FK, S, MB>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(
      std::is_same<R, double>::value ? (const void*)&c.d : (const void*)&c.f);
  k<<<hop_grid(LS, p.site_end - p.site0), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

template <int LS, int P, int EPI, int FK>
cudaError_t run_pair(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr int LF = DefaultLink<P>::v;
  constexpr size_t smem = hop_pair_smem_bytes<LS, P>();
  auto k = dwf_hop_pair_kernel<LS, P, LF, EPI, FK, HopMinBlocks<P>::v0>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(&c.f);
  k<<<hop_pair_grid(LS, p.site_end - p.site0), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

template <int LS, int P, int EPI, int FK>
cudaError_t run_pair_pf(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr size_t smem = hop_pair_smem_bytes<LS, P>();
  auto k = dwf_hop_pair_pf_kernel<LS, P, EPI, FK, 3>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(&c.f);
  k<<<hop_pair_grid(LS, p.site_end - p.site0), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

template <int LS, int P, int EPI, int FK, int S, int MB>
cudaError_t run_tma_pair(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  using R = typename Store<P>::R;
  constexpr int LF = DefaultLink<P>::v;
  constexpr size_t smem = hop_tma_pair_smem_bytes<LS, P, LF, S>();
  auto k = dwf_hop_tma_pair_kernel<LS, P, LF, EPI, FK, S, MB>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const ChainCoef<R>& kc = *reinterpret_cast<const ChainCoef<R>*>(&c.f);
  k<<<hop_pair_grid(LS, p.site_end - p.site0), 128, smem, st>>>(p, kc);
  return cudaGetLastError();
}

// variant 0: direct loads; 1: TMA-staged, 2 stages; 2: TMA-staged, 3 stages;
// 3: TMA-staged, 2 stages, register budget for HopMinBlocks::v1 resident
// blocks; 4: direct loads with that register budget; 5: packed FP32x2 kernel,
// two slices per thread, direct loads; 6: the packed kernel fed by the TMA
// pipeline; 7: a 4-deep TMA pipeline (FP64: the one-slice kernel; FP32
// arithmetic: the packed kernel) at 2 resident blocks; 8: the packed kernel
// with all 8 directions in flight at once; 9: the packed kernel for f16/bf16
// storage fetching the next direction into registers while computing the
// current one (5-9 packed: FP32 arithmetic only).
template <int LS, int P, int EPI, int FK>
cudaError_t run(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  if (p.variant == 1) return run_tma<LS, P, EPI, FK, 2, 1>(p, c, st);
  if (p.variant == 2) return run_tma<LS, P, EPI, FK, 3, 1>(p, c, st);
  if (p.variant == 3) return run_tma<LS, P, EPI, FK, 2, HopMinBlocks<P>::v1>(p, c, st);
  if (p.variant == 4) return run_mb<LS, P, EPI, FK, HopMinBlocks<P>::v1>(p, c, st);
  if constexpr (P != PREC_F64) {
    if (p.variant == 5) return run_pair<LS, P, EPI, FK>(p, c, st);
    if (p.variant == 6) return run_tma_pair<LS, P, EPI, FK, 2, HopMinBlocks<P>::v0>(p, c, st);
    if (p.variant == 7) return run_tma_pair<LS, P, EPI, FK, 4, 2>(p, c, st);
    if (p.variant == 8) return run_tma_pair<LS, P, EPI, FK, 8, 2>(p, c, st);
    if constexpr (P != PREC_F32)
      if (p.variant == 9) return run_pair_pf<LS, P, EPI, FK>(p, c, st);
  }
  if constexpr (P == PREC_F64)
    if (p.variant == 7) return run_tma<LS, P, EPI, FK, 4, 2>(p, c, st);
  return run_mb<LS, P, EPI, FK, HopMinBlocks<P>::v0>(p, c, st);
}

template <int LS>
cudaError_t dispatch_epi(const HopParams& p, const ChainCoefs& c, cudaStream_t st) {
  constexpr int P = B200_PREC;
  switch (p.epi) {
    case EPI_HALF: return run<LS, P, EPI_HALF, F_NONE>(p, c, st);
    case EPI_DDAGEO: return run<LS, P, EPI_DDAGEO, F_NONE>(p, c, st);
    case EPI_K1: return run<LS, P, EPI_K1, F_NONE>(p, c, st);
    case EPI_K2N:
      if (p.fk == F_LUDAG) return run<LS, P, EPI_K2N, F_LUDAG>(p, c, st);
      if (p.fk == F_G5R) return run<LS, P, EPI_K2N, F_G5R>(p, c, st);
      return run<LS, P, EPI_K2N, F_NONE>(p, c, st);
    case EPI_K3: return run<LS, P, EPI_K3, F_NONE>(p, c, st);
    case EPI_K4N: return run<LS, P, EPI_K4N, F_NONE>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

#define B200_CAT2(a, b) a##b
#define B200_CAT(a, b) B200_CAT2(a, b)
cudaError_t B200_CAT(launch_hop_p, B200_PREC)(const HopParams& p, const ChainCoefs& c,
                                             cudaStream_t st) {
  switch (p.ls) {
    case 4: return dispatch_epi<4>(p, c, st);
    case 6: return dispatch_epi<6>(p, c, st);
    case 8: return dispatch_epi<8>(p, c, st);
    case 12: return dispatch_epi<12>(p, c, st);
    case 16: return dispatch_epi<16>(p, c, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace b200
