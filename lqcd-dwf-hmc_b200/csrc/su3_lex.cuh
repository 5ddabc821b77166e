// Small SU(3) / lexical-lattice helpers shared by the link-field kernels
// (stout smearing, gauge force and action, link update): complex numbers,
// 3x3 complex matrices in the reference Field_G layout
// ri + 2*(col + 3*row) + 18*(site + Nvol*mu), and periodic lexical shifts.
#pragma once

#include <cuda_runtime.h>

namespace b200 {

struct Cx {
  double r, i;
};
__device__ __forceinline__ Cx cx(double r, double i) { return Cx{r, i}; }
__device__ __forceinline__ Cx operator+(Cx a, Cx b) { return cx(a.r + b.r, a.i + b.i); }
__device__ __forceinline__ Cx operator-(Cx a, Cx b) { return cx(a.r - b.r, a.i - b.i); }
__device__ __forceinline__ Cx operator*(Cx a, Cx b) { return cx(a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r); }
__device__ __forceinline__ Cx operator*(double s, Cx a) { return cx(s * a.r, s * a.i); }

struct M3 {
  Cx m[9];   // row-major
};

__device__ __forceinline__ M3 load3(const double* base, size_t idx) {
  M3 a;
  const double2* p = reinterpret_cast<const double2*>(base + 18 * idx);
#pragma unroll
  for (int k = 0; k < 9; ++k) { double2 v = p[k]; a.m[k] = cx(v.x, v.y); }
  return a;
}
__device__ __forceinline__ void store3(double* base, size_t idx, const M3& a) {
  double2* p = reinterpret_cast<double2*>(base + 18 * idx);
#pragma unroll
  for (int k = 0; k < 9; ++k) p[k] = make_double2(a.m[k].r, a.m[k].i);
}
__device__ __forceinline__ M3 zero3() {
  M3 a;
#pragma unroll
  for (int k = 0; k < 9; ++k) a.m[k] = cx(0, 0);
  return a;
}
__device__ __forceinline__ M3 unit3() {
  M3 a = zero3();
  a.m[0] = a.m[4] = a.m[8] = cx(1, 0);
  return a;
}
// A B, A B^+, A^+ B, A^+ B^+
__device__ __forceinline__ M3 mul_nn(const M3& a, const M3& b) {
  M3 c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Cx s = cx(0, 0);
#pragma unroll
      for (int k = 0; k < 3; ++k) s = s + a.m[3 * i + k] * b.m[3 * k + j];
      c.m[3 * i + j] = s;
    }
  return c;
}
__device__ __forceinline__ Cx conj(Cx a) { return cx(a.r, -a.i); }
__device__ __forceinline__ M3 mul_nd(const M3& a, const M3& b) {
  M3 c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Cx s = cx(0, 0);
#pragma unroll
      for (int k = 0; k < 3; ++k) s = s + a.m[3 * i + k] * conj(b.m[3 * j + k]);
      c.m[3 * i + j] = s;
    }
  return c;
}
__device__ __forceinline__ M3 mul_dn(const M3& a, const M3& b) {
  M3 c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Cx s = cx(0, 0);
#pragma unroll
      for (int k = 0; k < 3; ++k) s = s + conj(a.m[3 * k + i]) * b.m[3 * k + j];
      c.m[3 * i + j] = s;
    }
  return c;
}
__device__ __forceinline__ M3 mul_dd(const M3& a, const M3& b) {
  M3 c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Cx s = cx(0, 0);
#pragma unroll
      for (int k = 0; k < 3; ++k) s = s + conj(a.m[3 * k + i]) * conj(b.m[3 * j + k]);
      c.m[3 * i + j] = s;
    }
  return c;
}
__device__ __forceinline__ void add_to(M3& a, const M3& b, double s = 1.0) {
#pragma unroll
  for (int k = 0; k < 9; ++k) a.m[k] = a.m[k] + s * b.m[k];
}
// traceless anti-Hermitian part (Mat_SU_N::at, src/lib/Tools/mat_SU_N.h:375-398)
__device__ __forceinline__ void at3(M3& a) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i + 1; j < 3; ++j) {
      const double re = a.m[3 * i + j].r - a.m[3 * j + i].r;
      const double im = a.m[3 * i + j].i + a.m[3 * j + i].i;
      a.m[3 * i + j] = cx(0.5 * re, 0.5 * im);
      a.m[3 * j + i] = cx(-0.5 * re, 0.5 * im);
    }
  const double tr = (a.m[0].i + a.m[4].i + a.m[8].i) / 3.0;
  a.m[0] = cx(0.0, a.m[0].i - tr);
  a.m[4] = cx(0.0, a.m[4].i - tr);
  a.m[8] = cx(0.0, a.m[8].i - tr);
}
__device__ __forceinline__ double norm2_3(const M3& a) {
  double t = 0;
#pragma unroll
  for (int k = 0; k < 9; ++k) t += a.m[k].r * a.m[k].r + a.m[k].i * a.m[k].i;
  return t;
}

struct LexGeom {
  int n[4];
  size_t vol;
  __device__ size_t shift(size_t site, int mu, int dir) const {   // site + dir*mu (periodic)
    int c[4];
    size_t s = site;
    c[0] = (int)(s % n[0]); s /= n[0];
    c[1] = (int)(s % n[1]); s /= n[1];
    c[2] = (int)(s % n[2]); s /= n[2];
    c[3] = (int)s;
    c[mu] = (c[mu] + dir + n[mu]) % n[mu];
    return c[0] + (size_t)n[0] * (c[1] + (size_t)n[1] * (c[2] + (size_t)n[2] * c[3]));
  }
};

}  // namespace b200
