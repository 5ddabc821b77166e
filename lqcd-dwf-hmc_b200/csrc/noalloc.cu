// Allocation-free |x|^2 of a field, for callers that cannot allocate device
// memory.
//
// Who needs it: code that runs where cudaMalloc is forbidden or unsafe -- a
// host framework that owns all device memory through its own pool and counts
// on libraries not to allocate behind its back (an allocation outside the pool
// can fail, or fragment and exhaust what the pool planned for), or a caller on
// a GPU whose memory is already fully committed to resident gauge and fermion
// fields (at 24^3x48 Ls=16 a multishift solve alone holds ~35 GB).  Such a
// caller cannot create an operator plan (which owns its reduction scratch), so
// it gets this one entry point that takes only the field and its size and
// returns the norm.
//
// The block partial sums live in a file-scope __device__ array of fixed size
// (kNoallocMaxBlocks doubles + one result slot, 512 KiB), which every GPU
// that loads this library keeps until the process exits.  One block reduces
// 128 (site, s) pairs, so the largest field is kNoallocMaxBlocks * 128 =
// 8,388,608 (site, s) pairs (e.g. 24^3x48 at Ls=16 fits, 32^3x64 at Ls=12 does
// not); larger sizes are rejected with B200_EINVAL.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/b200dwf.h"
#include "dwf_kernels.h"

namespace b200 {
void set_last_error(int code, const char* fmt, ...);
}

namespace {

constexpr int kNoallocMaxBlocks = 65536;
constexpr int kMaxDevices = 64;

// Shared by every call on a device: slots [0, nblocks) hold the block
// partials of the current call, slot kNoallocMaxBlocks the final sum.
static __device__ __align__(256) double g_noalloc_scratch[kNoallocMaxBlocks + 1];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device with that device current (the array's name in host code is only
// a host-side stand-in for the symbol, not a device address).
int noalloc_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    b200::set_last_error(B200_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    return B200_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    b200::set_last_error(B200_EINVAL, "device index %d out of range", dev);
    return B200_EINVAL;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      b200::set_last_error(B200_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s",
                           cudaGetErrorString(e));
      return B200_ECUDA;
    }
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

}  // namespace

extern "C" int b200_field_norm2_noalloc(int prec, const void* x, long nsite, int ls,
                                        double* result, void* stream) {
  using namespace b200;
  if (!x || !result || prec < 0 || prec > 3 || nsite <= 0 || ls <= 0 || ls > kMaxLs) {
    set_last_error(B200_EINVAL, "norm2_noalloc: invalid argument");
    return B200_EINVAL;
  }
  const long pairs = nsite * (long)ls;
  const long nblocks = (pairs + kSiteSBlock - 1) / kSiteSBlock;
  if (nblocks > kNoallocMaxBlocks) {
    set_last_error(B200_EINVAL,
                   "norm2_noalloc: field of %ld (site, s) pairs exceeds the fixed scratch "
                   "maximum of %ld pairs",
                   pairs, (long)kNoallocMaxBlocks * kSiteSBlock);
    return B200_EINVAL;
  }
  double* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Geom g;
  g.nx2 = 1; g.ny = 1; g.nz = 1; g.nt = 1;
  g.vh = (int)nsite;
  g.ls = ls;
  // every block writes its own partial slot before the final sum reads it, so
  // nothing left over from an earlier call needs clearing
  cudaError_t e = launch_dot(prec, g, x, x, scratch, st);
  if (e == cudaSuccess) e = launch_finalize(scratch, (int)nblocks, scratch + kNoallocMaxBlocks, FIN_SUM, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(result, scratch + kNoallocMaxBlocks, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_last_error(B200_ECUDA, "norm2_noalloc: %s", cudaGetErrorString(e));
    return B200_ECUDA;
  }
  return 0;
}
