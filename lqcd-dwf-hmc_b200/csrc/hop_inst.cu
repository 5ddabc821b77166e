// Explicit instantiations of the fused hop kernel for one storage precision.
// Compiled once per precision with -DB200_PREC=<0..3> (see the Makefile).
#include "dwf_hop.cuh"
#include "dwf_kernels.h"

#ifndef B200_PREC
#error "B200_PREC must be defined"
#endif

namespace b200 {

template <int P> struct DefaultLink;
template <> struct DefaultLink<PREC_F64> { static constexpr int v = LINK_F64_18; };
template <> struct DefaultLink<PREC_F32> { static constexpr int v = LINK_F32_12; };
template <> struct DefaultLink<PREC_F16> { static constexpr int v = LINK_F16_12; };
template <> struct DefaultLink<PREC_BF16> { static constexpr int v = LINK_F16_12; };

namespace {

template <int LS, int P, bool DAG>
cudaError_t run(const HopParams& p, cudaStream_t st) {
  constexpr int LF = DefaultLink<P>::v;
  constexpr size_t smem = hop_smem_bytes<LS, P>();
  auto k = dwf_hop_kernel<LS, P, LF, DAG>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  const int grid = hop_grid(LS, p.vh);
  k<<<grid, 128, smem, st>>>(p);
  return cudaGetLastError();
}

template <bool DAG>
cudaError_t dispatch_ls(const HopParams& p, cudaStream_t st) {
  switch (p.ls) {
    case 4: return run<4, B200_PREC, DAG>(p, st);
    case 6: return run<6, B200_PREC, DAG>(p, st);
    case 8: return run<8, B200_PREC, DAG>(p, st);
    case 12: return run<12, B200_PREC, DAG>(p, st);
    case 16: return run<16, B200_PREC, DAG>(p, st);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

#define B200_CAT2(a, b) a##b
#define B200_CAT(a, b) B200_CAT2(a, b)
cudaError_t B200_CAT(launch_hop_p, B200_PREC)(bool dag, const HopParams& p, cudaStream_t st) {
  return dag ? dispatch_ls<true>(p, st) : dispatch_ls<false>(p, st);
}

}  // namespace b200
