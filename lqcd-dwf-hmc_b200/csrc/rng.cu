// The benchmark driver's random-number generator on the device: the parallel
// M-series generator of the reference (random_number_type Mseries_parallel,
// RandomNumbers_parallel<RandomNumbers_Mseries>), stream for stream, so the
// heatbath (Langevin momenta, pseudofermion noise) can be drawn on the GPU
// with the numbers the reference hands out.
//
// Reference behaviour (file:line relative to the reference tree):
//   one stream: RandomNumbers_Mseries, src/lib/Tools/randomNumbers_Mseries.cpp:32-150
//     and randomNumbers_Mseries.h:55-91 -- 521 31-bit words, x_n = x_(n-521) ^
//     x_(n-32), output x_n * 2^-31; the start state is the 69069 LCG bit
//     stream packed into words, advanced by ndelay steps through a polynomial
//     (x^ndelay mod the generator's characteristic polynomial).
//   Gaussian pair: RandomNumbers::gauss, src/lib/Tools/randomNumbers.cpp:53-75.
//   parallel layout: RandomNumbers_parallel init_2d / set_lex_global_2d,
//     src/lib/Tools/randomNumbers_parallel-tmpl.h:160-252 -- one stream per
//     (z, t) plane started with (seed+1)*Lz*Lt + z + Lz*t (as int), 1000
//     numbers discarded; a field Field(Nin, Nvol, Nex) is filled per extra
//     index j, per plane, per y, per x with one block of Nin numbers
//     (get_gauss: Nin Gaussians; get_uniform: one number in component 0,
//     src/lib/Tools/randomNumbers_parallel.h:102-145).
//
// Device mapping: one warp per plane.  The plane's 521-word ring sits in
// shared memory; since every new word depends only on words 32 and 521
// steps back, the warp produces 32 consecutive numbers per step (lane l:
// x_(n+l) = x_(n+l-521) ^ x_(n+l-32)), pairs of lanes form the Box-Muller
// pairs, and each lane stores its number at its (j, y, x, i) position.  The
// stream start states (initset + jump + discarded numbers) are computed on
// the host when the generator is created or reset.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/b200dwf.h"

namespace b200 {
void set_last_error(int code, const char* fmt, ...);
}

namespace {

constexpr int kNp = 521;
constexpr int kNq = 32;
constexpr int kStride = 524;       // words per plane in the device state: ring, jr, kr, pad
constexpr int kThermalization = 1000;

// ---------------------------------------------------------------- host side
struct Stream {
  int w[kNp];
  int jr, kr;

  int get_word() {
    w[jr] ^= w[kr];
    const int v = w[jr];
    jr = (jr + 1 == kNp) ? 0 : jr + 1;
    kr = (kr + 1 == kNp) ? 0 : kr + 1;
    return v;
  }

  // start state: the bit stream of the 69069 congruential sequence (top bit)
  // run through the generator's own recurrence and packed 32 bits a word
  void start(int ndelay) {
    unsigned bits[kNp];
    unsigned ix = 1;
    for (int i = 0; i < kNp; ++i) {
      ix *= 69069u;
      bits[i] = ix >> 31;
    }
    int a = 0, b = kNp - kNq;
    for (int j = 0; j < kNp; ++j) {
      unsigned word = 0;
      for (int i = 0; i < 32; ++i) {
        word = word * 2u + bits[a];
        bits[a] ^= bits[b];
        a = (a + 1 == kNp) ? 0 : a + 1;
        b = (b + 1 == kNp) ? 0 : b + 1;
      }
      w[j] = (int)(word >> 1);
    }
    jr = a;
    kr = b;
    jump(ndelay);
  }

  // advance by ndelay steps: c(x) = x^ndelay mod the characteristic
  // polynomial x^521 + x^489 + 1 (binary square-and-multiply on the exponent,
  // the 40 lowest bits taken as zero as the reference does), then the state
  // words as the c-weighted XOR of the extended word sequence
  void jump(int ndelay) {
    std::vector<unsigned> ext(2 * kNp - 1);
    for (int i = 0; i < kNp; ++i) ext[i] = (unsigned)w[i];
    for (int i = kNp; i < 2 * kNp - 1; ++i) ext[i] = ext[i - kNp] ^ ext[i - kNq];
    std::vector<int> expo(40, 0);
    int m = ndelay;
    while (m > kNp - 1) {
      expo.push_back(m % 2);
      m /= 2;
    }
    std::vector<unsigned char> c(2 * kNp, 0), t(2 * kNp, 0);
    c[m] = 1;
    for (int j = (int)expo.size() - 1; j >= 0; --j) {
      const int e = expo[j];
      for (int i = 0; i < kNp; ++i) {
        t[2 * i + e] = c[i];
        t[2 * i + 1 - e] = 0;
      }
      c.swap(t);
      for (int i = 2 * kNp - 1; i >= kNp; --i) {
        if (c[i]) {
          c[i - kNp] ^= 1;
          c[i - kNq] ^= 1;
        }
      }
    }
    for (int j = 0; j < kNp; ++j) {
      unsigned acc = 0;
      for (int i = 0; i < kNp; ++i)
        if (c[i]) acc ^= ext[j + i];
      w[j] = (int)acc;
    }
  }
};

// ---------------------------------------------------------------- device side
__device__ __constant__ double kFnorm = 4.656612870908988e-10;

template <bool kGauss>
__global__ void __launch_bounds__(128) mseries_draw_kernel(int* state, int nplanes, double* out,
                                                           int lx, int ly, long nvol, int nin,
                                                           int nex) {
  __shared__ int ring[4][kNp];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int zt = blockIdx.x * 4 + warp;
  if (zt >= nplanes) return;                 // whole warps only
  int* st = state + (size_t)zt * kStride;
  int* r = ring[warp];
  for (int i = lane; i < kNp; i += 32) r[i] = st[i];
  int jr = st[kNp], kr = st[kNp + 1];
  __syncwarp();
  const double sq2r = 1.0 / sqrt(2.0);
  const double pi2 = 2.0 * (4.0 * atan(1.0));
  const int blk = kGauss ? nin : 1;          // numbers consumed per site
  const long total = (long)nex * ly * lx * blk;
  for (long base = 0; base < total; base += 32) {
    const long n = base + lane;
    const bool act = n < total;
    int ij = jr + lane; if (ij >= kNp) ij -= kNp;
    int ik = kr + lane; if (ik >= kNp) ik -= kNp;
    int v = 0;
    if (act) v = r[ij] ^ r[ik];              // r[ik] was written one step earlier
    __syncwarp();
    if (act) r[ij] = v;
    __syncwarp();
    const double x = (double)v * kFnorm;
    // Box-Muller over lane pairs (2k, 2k+1): every block starts at an even n
    const double partner = __shfl_xor_sync(0xffffffffu, x, 1);
    const long sb = n / blk;
    const int i = (int)(n - sb * blk);
    const int x0 = (int)(sb % lx);
    const long rest = sb / lx;
    const int y0 = (int)(rest % ly);
    const int j = (int)(rest / ly);
    const long site = x0 + (long)lx * (y0 + (long)ly * zt);
    double* dst = out + (size_t)nin * (site + nvol * j);
    if (kGauss) {
      const double r1 = (lane & 1) ? partner : x;
      const double r2 = (lane & 1) ? x : partner;
      const double slg = sqrt(-log(1.0 - r1) * 2.0) * sq2r;
      const double ang = pi2 * r2;
      if (act) dst[i] = (lane & 1) ? slg * sin(ang) : slg * cos(ang);
    } else if (act) {
      dst[0] = x;
      for (int q = 1; q < nin; ++q) dst[q] = 0.0;
    }
    const int cnt = (total - base < 32) ? (int)(total - base) : 32;
    jr += cnt; if (jr >= kNp) jr -= kNp;
    kr += cnt; if (kr >= kNp) kr -= kNp;
  }
  __syncwarp();
  for (int i = lane; i < kNp; i += 32) st[i] = r[i];
  if (lane == 0) { st[kNp] = jr; st[kNp + 1] = kr; }
}

}  // namespace

struct b200_rng {
  int L[4];
  int nplanes;
  int* state = nullptr;      // device: nplanes x kStride words
};

namespace {

int rng_fail(int code, const char* msg) {
  b200::set_last_error(code, "%s", msg);
  return code;
}

int seed_planes(b200_rng* g, unsigned long seed) {
  const int lz = g->L[2], lt = g->L[3];
  // The generator of plane zt starts from the delay (seed + 1) Lz Lt + zt,
  // which the reference hands to RandomNumbers_Mseries as an int
  // (randomNumbers_parallel_Mseries.cpp:52-55); past INT_MAX that int is
  // negative and the jump-ahead (delay3, randomNumbers_Mseries.cpp:79-140)
  // indexes its polynomial below zero.  Such seeds are refused.
  const unsigned long long planes = (unsigned long long)lz * (unsigned long long)lt;
  if ((unsigned long long)seed + 1ull > (2147483647ull - (planes - 1ull)) / planes)
    return rng_fail(B200_EINVAL,
                    "seed too large for this lattice: (seed + 1) * Lz * Lt + plane must fit the "
                    "M-series generator's int delay");
  // draws still running on any stream finish before the state is replaced
  const cudaError_t es = cudaDeviceSynchronize();
  if (es != cudaSuccess) return rng_fail(B200_ECUDA, cudaGetErrorString(es));
  std::vector<int> h((size_t)g->nplanes * kStride, 0);
  for (int t = 0; t < lt; ++t)
    for (int z = 0; z < lz; ++z) {
      const int zt = z + lz * t;
      const unsigned long s = (seed + 1) * (unsigned long)lz * (unsigned long)lt + (unsigned long)zt;
      Stream str;
      str.start((int)s);
      for (int k = 0; k < kThermalization; ++k) str.get_word();
      int* d = h.data() + (size_t)zt * kStride;
      for (int i = 0; i < kNp; ++i) d[i] = str.w[i];
      d[kNp] = str.jr;
      d[kNp + 1] = str.kr;
    }
  const cudaError_t e =
      cudaMemcpy(g->state, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return rng_fail(B200_ECUDA, cudaGetErrorString(e));
  return 0;
}

int draw(b200_rng* g, double* v, int nin, int nex, void* stream, bool gauss) {
  if (!g || !v || nin < 1 || nex < 1) return rng_fail(B200_EINVAL, "invalid argument");
  if (gauss && nin % 2 != 0)
    return rng_fail(B200_EINVAL, "gaussian fields need an even number of components per site");
  const long nvol = (long)g->L[0] * g->L[1] * g->L[2] * g->L[3];
  const int grid = (g->nplanes + 3) / 4;
  cudaStream_t st = (cudaStream_t)stream;
  if (gauss)
    mseries_draw_kernel<true><<<grid, 128, 0, st>>>(g->state, g->nplanes, v, g->L[0], g->L[1], nvol,
                                                    nin, nex);
  else
    mseries_draw_kernel<false><<<grid, 128, 0, st>>>(g->state, g->nplanes, v, g->L[0], g->L[1],
                                                     nvol, nin, nex);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rng_fail(B200_ECUDA, cudaGetErrorString(e));
  return 0;
}

}  // namespace

extern "C" {

int b200_rng_create(b200_rng_t** out, const int lattice[4], unsigned long seed) {
  if (!out || !lattice) return rng_fail(B200_EINVAL, "null argument");
  *out = nullptr;
  for (int mu = 0; mu < 4; ++mu)
    if (lattice[mu] < 1) return rng_fail(B200_EINVAL, "lattice extent invalid");
  b200_rng* g = new b200_rng();
  for (int mu = 0; mu < 4; ++mu) g->L[mu] = lattice[mu];
  g->nplanes = lattice[2] * lattice[3];
  if (cudaMalloc(&g->state, (size_t)g->nplanes * kStride * sizeof(int)) != cudaSuccess) {
    delete g;
    return rng_fail(B200_ENOMEM, "cudaMalloc for the generator state failed");
  }
  const int rc = seed_planes(g, seed);
  if (rc) {
    cudaFree(g->state);
    delete g;
    return rc;
  }
  *out = g;
  return 0;
}

int b200_rng_reset(b200_rng_t* g, unsigned long seed) {
  if (!g) return rng_fail(B200_EINVAL, "null generator");
  return seed_planes(g, seed);
}

int b200_rng_gauss_lex(b200_rng_t* g, double* v, int nin, int nex, void* stream) {
  return draw(g, v, nin, nex, stream, true);
}

int b200_rng_uniform_lex(b200_rng_t* g, double* v, int nin, int nex, void* stream) {
  return draw(g, v, nin, nex, stream, false);
}

int b200_rng_destroy(b200_rng_t* g) {
  if (!g) return 0;
  cudaFree(g->state);
  delete g;
  return 0;
}

}  // extern "C"
