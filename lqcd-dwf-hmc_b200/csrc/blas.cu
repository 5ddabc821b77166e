// Plan-free vector kernels on flat device arrays: the AField<REAL, B200>
// methods of the reference-side overlay (set, copy, axpy, aypx, scal, dot,
// dotc, norm2, convert_h) run here.  They replace the BridgeACC vector
// functions of the reference's GPU build (src/lib_alt_Accel/BridgeOpenACC/src/
// afield_openacc-inc.h:14-446: set, axpy, aypx, scal, dot, dotc, norm2) and its
// precision copy (afield_copy_openacc-inc.h:11-54).
//
// The arrays are n reals of one precision (0: double, 1: float) in any order:
// element-wise updates and sums do not depend on the field layout, and a
// complex update acts on (re, im) neighbours, which every layout of this
// library keeps adjacent.  Reductions accumulate in double (the reference
// accumulates dot in the field's precision and norm2 in double) and return
// synchronously, as the reference's do.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/b200dwf.h"
#include "dwf_kernels.h"

namespace b200 {
void set_last_error(int code, const char* fmt, ...);
}

namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 1184;          // 8 blocks on each of the 148 SMs
constexpr int kMaxDevices = 64;

template <typename T>
__global__ void axpby_kernel(size_t n, double a, const T* __restrict__ x, double b, T* __restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double xi = x ? (double)x[i] : 0.0;
    y[i] = (T)((b == 0.0) ? a * xi : fma(a, xi, b * (double)y[i]));
  }
}

// y = (ar + i ai) x + (br + i bi) y on (re, im) pairs
template <typename T>
__global__ void caxpby_kernel(size_t npair, double ar, double ai, const T* __restrict__ x, double br,
                              double bi, T* __restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npair; i += (size_t)gridDim.x * blockDim.x) {
    const double xr = x ? (double)x[2 * i] : 0.0, xi = x ? (double)x[2 * i + 1] : 0.0;
    const double yr = (double)y[2 * i], yi = (double)y[2 * i + 1];
    double outr = ar * xr - ai * xi, outi = ar * xi + ai * xr;
    if (br != 0.0 || bi != 0.0) {
      outr += br * yr - bi * yi;
      outi += br * yi + bi * yr;
    }
    y[2 * i] = (T)outr;
    y[2 * i + 1] = (T)outi;
  }
}

template <typename T>
__global__ void fill_kernel(size_t n, double v, T* y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = (T)v;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += sh[w];
  __syncthreads();
  return s;
}

// kConj = false: partial[b] = sum x_i y_i;  true: (re, im) of sum conj(x) y
// over pairs, partial[2b], partial[2b+1]
template <typename T, bool kConj>
__global__ void dot_partial_kernel(size_t n, const T* __restrict__ x, const T* __restrict__ y,
                                   double* partial) {
  __shared__ double sh[kThreads / 32];
  double re = 0.0, im = 0.0;
  if (!kConj) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
      re = fma((double)x[i], (double)y[i], re);
  } else {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n / 2; i += (size_t)gridDim.x * blockDim.x) {
      const double xr = x[2 * i], xi = x[2 * i + 1], yr = y[2 * i], yi = y[2 * i + 1];
      re = fma(xr, yr, fma(xi, yi, re));
      im = fma(xr, yi, fma(-xi, yr, im));
    }
  }
  const double sr = block_sum(re, sh);
  if (!kConj) {
    if (threadIdx.x == 0) partial[blockIdx.x] = sr;
    return;
  }
  const double si = block_sum(im, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sr;
    partial[2 * blockIdx.x + 1] = si;
  }
}

// out[c] = sum_b partial[ncomp * b + c], one block
__global__ void sum_partials_kernel(const double* partial, int nblocks, int ncomp, double* out) {
  __shared__ double sh[kThreads / 32];
  for (int c = 0; c < ncomp; ++c) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partial[ncomp * b + c];
    const double s = block_sum(v, sh);
    if (threadIdx.x == 0) out[c] = s;
  }
}

// Reduction scratch of the calling device (2 * kBlocks partials + 2 results),
// allocated on the first reduction on that device and kept.  A reduction
// holds its device's lock from the first launch until its result is back,
// so host threads reducing on one device take turns instead of overwriting
// each other's partials.
std::mutex g_mu;
double* g_scratch[kMaxDevices] = {};
std::mutex g_reduce_mu[kMaxDevices];

int scratch(double** out, int* dev_out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    b200::set_last_error(B200_ECUDA, "blas: no usable current device");
    return B200_ECUDA;
  }
  *dev_out = dev;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev] && cudaMalloc(&g_scratch[dev], (2 * kBlocks + 2) * sizeof(double)) != cudaSuccess) {
    g_scratch[dev] = nullptr;
    b200::set_last_error(B200_ENOMEM, "blas: cudaMalloc of the reduction scratch failed");
    return B200_ENOMEM;
  }
  *out = g_scratch[dev];
  return 0;
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return 0;
  b200::set_last_error(B200_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return B200_ECUDA;
}

int bad(const char* what) {
  b200::set_last_error(B200_EINVAL, "%s: invalid argument", what);
  return B200_EINVAL;
}

int blocks_for(size_t n) {
  const size_t b = (n + kThreads - 1) / kThreads;
  return (int)(b < (size_t)kBlocks ? (b ? b : 1) : kBlocks);
}

template <typename T, bool kConj>
int reduce(size_t n, const void* x, const void* y, double* res, int ncomp, cudaStream_t st) {
  double* s = nullptr;
  int dev = 0;
  int rc = scratch(&s, &dev);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_reduce_mu[dev]);
  const int nb = blocks_for(kConj ? n / 2 : n);
  dot_partial_kernel<T, kConj><<<nb, kThreads, 0, st>>>(n, (const T*)x, (const T*)y, s);
  sum_partials_kernel<<<1, kThreads, 0, st>>>(s, nb, ncomp, s + 2 * kBlocks);
  if ((rc = check_launch("blas reduction"))) return rc;
  cudaError_t e = cudaMemcpyAsync(res, s + 2 * kBlocks, ncomp * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    b200::set_last_error(B200_ECUDA, "blas reduction: %s", cudaGetErrorString(e));
    return B200_ECUDA;
  }
  return 0;
}

}  // namespace

extern "C" {

int b200_blas_axpby(int prec, size_t n, double a, const void* x, double b, void* y, void* stream) {
  if (!y || (prec != 0 && prec != 1)) return bad("b200_blas_axpby");
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == 0) axpby_kernel<double><<<blocks_for(n), kThreads, 0, st>>>(n, a, (const double*)x, b, (double*)y);
  else axpby_kernel<float><<<blocks_for(n), kThreads, 0, st>>>(n, a, (const float*)x, b, (float*)y);
  return check_launch("b200_blas_axpby");
}

int b200_blas_caxpby(int prec, size_t n, double ar, double ai, const void* x, double br, double bi, void* y,
                     void* stream) {
  if (!y || (n & 1) || (prec != 0 && prec != 1)) return bad("b200_blas_caxpby");
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == 0)
    caxpby_kernel<double><<<blocks_for(n / 2), kThreads, 0, st>>>(n / 2, ar, ai, (const double*)x, br, bi,
                                                                   (double*)y);
  else
    caxpby_kernel<float><<<blocks_for(n / 2), kThreads, 0, st>>>(n / 2, ar, ai, (const float*)x, br, bi,
                                                                  (float*)y);
  return check_launch("b200_blas_caxpby");
}

int b200_blas_fill(int prec, size_t n, double value, void* y, void* stream) {
  if (!y || (prec != 0 && prec != 1)) return bad("b200_blas_fill");
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == 0) fill_kernel<double><<<blocks_for(n), kThreads, 0, st>>>(n, value, (double*)y);
  else fill_kernel<float><<<blocks_for(n), kThreads, 0, st>>>(n, value, (float*)y);
  return check_launch("b200_blas_fill");
}

int b200_blas_dot(int prec, size_t n, const void* x, const void* y, double* result, void* stream) {
  if (!x || !y || !result || (prec != 0 && prec != 1)) return bad("b200_blas_dot");
  cudaStream_t st = (cudaStream_t)stream;
  return prec == 0 ? reduce<double, false>(n, x, y, result, 1, st) : reduce<float, false>(n, x, y, result, 1, st);
}

int b200_blas_dotc(int prec, size_t n, const void* x, const void* y, double* re, double* im, void* stream) {
  if (!x || !y || !re || !im || (n & 1) || (prec != 0 && prec != 1)) return bad("b200_blas_dotc");
  cudaStream_t st = (cudaStream_t)stream;
  double r[2];
  const int rc = prec == 0 ? reduce<double, true>(n, x, y, r, 2, st) : reduce<float, true>(n, x, y, r, 2, st);
  if (rc) return rc;
  *re = r[0];
  *im = r[1];
  return 0;
}

int b200_field_convert_prec(int prec_out, void* out, int prec_in, const void* in, long nsite, int ls,
                            void* stream) {
  using namespace b200;
  if (!out || !in || prec_out < 0 || prec_out > 3 || prec_in < 0 || prec_in > 3 || nsite <= 0 || ls <= 0 ||
      ls > kMaxLs)
    return bad("b200_field_convert_prec");
  Geom g;
  g.nx2 = 1; g.ny = 1; g.nz = 1; g.nt = 1;
  g.vh = (int)nsite;
  g.ls = ls;
  const cudaError_t e = launch_convert(prec_out, out, prec_in, in, g, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    set_last_error(B200_ECUDA, "b200_field_convert_prec: %s", cudaGetErrorString(e));
    return B200_ECUDA;
  }
  return 0;
}

}  // extern "C"
