// Shared device-side definitions of the B200 domain-wall library.
//
// Field layout in HBM (one even/odd 5D half-lattice spinor), site-major:
//   every 4D site owns one contiguous "column" of col_bytes(prec, Ls) bytes
//   holding its whole fifth dimension: 16-byte chunks (k, s) -> k*Ls + s,
//   s fastest, so the Ls lanes that own the site read one contiguous run of
//   Ls*16 bytes per chunk and a neighbour's column is one bulk (TMA) copy.
//   A chunk holds complex components q = color + 3*spin:
//     f64 : 1 complex  (double2), K = 12 chunks per (site, s)
//     f32 : 2 complex  (float4),  K = 6
//     f16/bf16 : 4 complex (8 halves in uint4), K = 3, values scaled by a
//       per-(site, s) float stored after the site's chunks (padded to 16 B).
// Link layout (one plan, both parities), record (ieo + 2*mu)*Vh + site:
//   f64 : 9 double2 (full 3x3; LINK_F64_18, read by the FP64 hops)
//   f32 : 5 float4  (full 3x3, 18 floats + padding; LINK_F32_18, FP32 hops)
//         or 3 float4 (two rows, third rebuilt; LINK_F32_12, learned network)
//   f16 : 3 uint4   (full 3x3 as 18 halves + padding; LINK_F16_18)
// The hop formats carry the boundary phase and the t projection's factor 2
// (dwf_hop.cuh, LinkLoad::kFolded).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace b200 {

enum Prec { PREC_F64 = 0, PREC_F32 = 1, PREC_F16 = 2, PREC_BF16 = 3 };

constexpr int kMaxLs = 32;

// ---------------------------------------------------------------- storage
template <int P> struct Store;

template <> struct Store<PREC_F64> {
  using R = double;
  using Chunk = double2;
  static constexpr int K = 12;
  static constexpr bool kScaled = false;
  __host__ __device__ static constexpr size_t col_bytes(int ls) { return (size_t)K * ls * 16; }
  // column already in shared memory (or anywhere): chunk (k, s)
  __device__ static void load_col(const void* col, int ls, int s, R* v) {
    const double2* p = reinterpret_cast<const double2*>(col);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double2 c = p[k * ls + s];
      v[2 * k] = c.x;
      v[2 * k + 1] = c.y;
    }
  }
  __device__ static void load(const void* base, size_t vh, int ls, int site, int s, R* v) {
    const double2* p = reinterpret_cast<const double2*>(base) + (size_t)site * K * ls;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double2 c = __ldg(p + k * ls + s);
      v[2 * k] = c.x;
      v[2 * k + 1] = c.y;
    }
  }
  __device__ static void store(void* base, size_t vh, int ls, int site, int s, const R* v) {
    double2* p = reinterpret_cast<double2*>(base) + (size_t)site * K * ls;
#pragma unroll
    for (int k = 0; k < K; ++k) p[k * ls + s] = make_double2(v[2 * k], v[2 * k + 1]);
  }
};

template <> struct Store<PREC_F32> {
  using R = float;
  using Chunk = float4;
  static constexpr int K = 6;
  static constexpr bool kScaled = false;
  __host__ __device__ static constexpr size_t col_bytes(int ls) { return (size_t)K * ls * 16; }
  __device__ static void load_col(const void* col, int ls, int s, R* v) {
    const float4* p = reinterpret_cast<const float4*>(col);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float4 c = p[k * ls + s];
      v[4 * k] = c.x; v[4 * k + 1] = c.y; v[4 * k + 2] = c.z; v[4 * k + 3] = c.w;
    }
  }
  __device__ static void load_col_raw(const void* col, int ls, int s, R* v, float* sc) {
    load_col(col, ls, s, v);
    *sc = 1.f;
  }
  __device__ static void load(const void* base, size_t vh, int ls, int site, int s, R* v) {
    const float4* p = reinterpret_cast<const float4*>(base) + (size_t)site * K * ls;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float4 c = __ldg(p + k * ls + s);
      v[4 * k] = c.x; v[4 * k + 1] = c.y; v[4 * k + 2] = c.z; v[4 * k + 3] = c.w;
    }
  }
  // unscaled components and the slice's scale (1 for this unscaled storage)
  __device__ static void load_raw(const void* base, size_t vh, int ls, int site, int s, R* v, float* sc) {
    load(base, vh, ls, site, s, v);
    *sc = 1.f;
  }
  __device__ static void store(void* base, size_t vh, int ls, int site, int s, const R* v) {
    float4* p = reinterpret_cast<float4*>(base) + (size_t)site * K * ls;
#pragma unroll
    for (int k = 0; k < K; ++k)
      p[k * ls + s] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  }
};

template <typename H> struct HalfOps;
template <> struct HalfOps<__half> {
  __device__ static float2 to2(unsigned int u) {
    __half2 h = *reinterpret_cast<__half2*>(&u);
    return __half22float2(h);
  }
  __device__ static unsigned int from2(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<unsigned int*>(&h);
  }
};
template <> struct HalfOps<__nv_bfloat16> {
  __device__ static float2 to2(unsigned int u) {
    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(h);
  }
  __device__ static unsigned int from2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<unsigned int*>(&h);
  }
};

template <typename H> struct StoreHalf {
  using R = float;
  using Half = H;
  using Chunk = uint4;
  static constexpr int K = 3;
  static constexpr bool kScaled = true;
  // column: K*ls chunks, then ls floats of scales padded to 16 bytes
  __host__ __device__ static constexpr size_t col_bytes(int ls) {
    return (size_t)K * ls * 16 + (((size_t)ls * 4 + 15) / 16) * 16;
  }
  __device__ static void decode(const uint4* p, const float sc, int ls, int s, R* v) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint4 c = p[k * ls + s];
      float2 a = HalfOps<H>::to2(c.x), b = HalfOps<H>::to2(c.y);
      float2 d = HalfOps<H>::to2(c.z), e = HalfOps<H>::to2(c.w);
      v[8 * k + 0] = a.x * sc; v[8 * k + 1] = a.y * sc;
      v[8 * k + 2] = b.x * sc; v[8 * k + 3] = b.y * sc;
      v[8 * k + 4] = d.x * sc; v[8 * k + 5] = d.y * sc;
      v[8 * k + 6] = e.x * sc; v[8 * k + 7] = e.y * sc;
    }
  }
  __device__ static void load_col(const void* col, int ls, int s, R* v) {
    const uint4* p = reinterpret_cast<const uint4*>(col);
    const float sc = reinterpret_cast<const float*>(p + K * ls)[s];
    decode(p, sc, ls, s, v);
  }
  // stored components without their scale, and the scale of slice s
  __device__ static void load_col_raw(const void* col, int ls, int s, R* v, float* sc) {
    const uint4* p = reinterpret_cast<const uint4*>(col);
    *sc = reinterpret_cast<const float*>(p + K * ls)[s];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint4 c = p[k * ls + s];
      float2 a = HalfOps<H>::to2(c.x), b = HalfOps<H>::to2(c.y);
      float2 d = HalfOps<H>::to2(c.z), e = HalfOps<H>::to2(c.w);
      v[8 * k + 0] = a.x; v[8 * k + 1] = a.y; v[8 * k + 2] = b.x; v[8 * k + 3] = b.y;
      v[8 * k + 4] = d.x; v[8 * k + 5] = d.y; v[8 * k + 6] = e.x; v[8 * k + 7] = e.y;
    }
  }
  __device__ static void load(const void* base, size_t vh, int ls, int site, int s, R* v) {
    const unsigned char* colp = reinterpret_cast<const unsigned char*>(base) + (size_t)site * col_bytes(ls);
    const uint4* p = reinterpret_cast<const uint4*>(colp);
    const float sc = __ldg(reinterpret_cast<const float*>(p + K * ls) + s);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint4 c = __ldg(p + k * ls + s);
      float2 a = HalfOps<H>::to2(c.x), b = HalfOps<H>::to2(c.y);
      float2 d = HalfOps<H>::to2(c.z), e = HalfOps<H>::to2(c.w);
      v[8 * k + 0] = a.x * sc; v[8 * k + 1] = a.y * sc;
      v[8 * k + 2] = b.x * sc; v[8 * k + 3] = b.y * sc;
      v[8 * k + 4] = d.x * sc; v[8 * k + 5] = d.y * sc;
      v[8 * k + 6] = e.x * sc; v[8 * k + 7] = e.y * sc;
    }
  }
  // stored components without their scale, and the scale of slice s
  __device__ static void load_raw(const void* base, size_t vh, int ls, int site, int s, R* v, float* sc) {
    const unsigned char* colp = reinterpret_cast<const unsigned char*>(base) + (size_t)site * col_bytes(ls);
    const uint4* p = reinterpret_cast<const uint4*>(colp);
    *sc = __ldg(reinterpret_cast<const float*>(p + K * ls) + s);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint4 c = __ldg(p + k * ls + s);
      float2 a = HalfOps<H>::to2(c.x), b = HalfOps<H>::to2(c.y);
      float2 d = HalfOps<H>::to2(c.z), e = HalfOps<H>::to2(c.w);
      v[8 * k + 0] = a.x; v[8 * k + 1] = a.y; v[8 * k + 2] = b.x; v[8 * k + 3] = b.y;
      v[8 * k + 4] = d.x; v[8 * k + 5] = d.y; v[8 * k + 6] = e.x; v[8 * k + 7] = e.y;
    }
  }
  __device__ static void store(void* base, size_t vh, int ls, int site, int s, const R* v) {
    unsigned char* colp = reinterpret_cast<unsigned char*>(base) + (size_t)site * col_bytes(ls);
    uint4* p = reinterpret_cast<uint4*>(colp);
    float m = 0.f;
#pragma unroll
    for (int i = 0; i < 24; ++i) m = fmaxf(m, fabsf(v[i]));
    const float sc = (m > 0.f) ? m : 1.f;
    const float inv = 1.f / sc;
    reinterpret_cast<float*>(p + K * ls)[s] = sc;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint4 c;
      c.x = HalfOps<H>::from2(v[8 * k + 0] * inv, v[8 * k + 1] * inv);
      c.y = HalfOps<H>::from2(v[8 * k + 2] * inv, v[8 * k + 3] * inv);
      c.z = HalfOps<H>::from2(v[8 * k + 4] * inv, v[8 * k + 5] * inv);
      c.w = HalfOps<H>::from2(v[8 * k + 6] * inv, v[8 * k + 7] * inv);
      p[k * ls + s] = c;
    }
  }
};
template <> struct Store<PREC_F16> : StoreHalf<__half> {};
template <> struct Store<PREC_BF16> : StoreHalf<__nv_bfloat16> {};

// Bytes of one field of Vh sites x Ls in precision p.
inline size_t field_bytes(int p, size_t vh, int ls) {
  switch (p) {
    case PREC_F64: return vh * Store<PREC_F64>::col_bytes(ls);
    case PREC_F32: return vh * Store<PREC_F32>::col_bytes(ls);
    default: return vh * Store<PREC_F16>::col_bytes(ls);
  }
}

// ---------------------------------------------------------------- links
// Link formats: LINK18 = full 3x3 matrix, LINK12 = two rows, third rebuilt.
template <typename R, bool kRecon> struct Su3 {
  R u[18];  // row-major re/im
};

template <typename R>
__device__ __forceinline__ void su3_reconstruct(R* u) {
  // row3 = conj(row1 x row2)
  const R a0r = u[0], a0i = u[1], a1r = u[2], a1i = u[3], a2r = u[4], a2i = u[5];
  const R b0r = u[6], b0i = u[7], b1r = u[8], b1i = u[9], b2r = u[10], b2i = u[11];
  // c0 = a1 b2 - a2 b1
  R c0r = (a1r * b2r - a1i * b2i) - (a2r * b1r - a2i * b1i);
  R c0i = (a1r * b2i + a1i * b2r) - (a2r * b1i + a2i * b1r);
  R c1r = (a2r * b0r - a2i * b0i) - (a0r * b2r - a0i * b2i);
  R c1i = (a2r * b0i + a2i * b0r) - (a0r * b2i + a0i * b2r);
  R c2r = (a0r * b1r - a0i * b1i) - (a1r * b0r - a1i * b0i);
  R c2i = (a0r * b1i + a0i * b1r) - (a1r * b0i + a1i * b0r);
  u[12] = c0r; u[13] = -c0i; u[14] = c1r; u[15] = -c1i; u[16] = c2r; u[17] = -c2i;
}

}  // namespace b200
