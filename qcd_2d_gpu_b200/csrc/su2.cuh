// SU(2) link algebra on unit quaternions U = w + i (x, y, z) . sigma.
//
// The four products keep the term order of the reference's su2_product,
// su2_product_tc (A B^dagger), su2_product_tc1 (A^dagger B) and
// su2_product_tc2 (A^dagger B^dagger) (functions/su2.h:50-73): with the
// same expression tree nvcc makes the same FMA contractions, so the FP64
// path reproduces the reference bit for bit.
#pragma once
#include <cuda_runtime.h>

namespace qcd {

template <class R>
struct Quat {
  R w, x, y, z;
};

template <class R>
__device__ __forceinline__ Quat<R> q_zero() {
  return Quat<R>{R(0), R(0), R(0), R(0)};
}

template <class R>
__device__ __forceinline__ Quat<R> q_one() {
  return Quat<R>{R(1), R(0), R(0), R(0)};
}

// A + B, component by component (su2.h:77-80)
template <class R>
__device__ __forceinline__ Quat<R> q_add(const Quat<R>& a, const Quat<R>& b) {
  return Quat<R>{a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z};
}

// A B  (su2.h:50-55)
template <class R>
__device__ __forceinline__ Quat<R> q_mul(const Quat<R>& a, const Quat<R>& b) {
  Quat<R> c;
  c.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = a.x * b.w + a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = a.y * b.w + a.z * b.x + a.w * b.y - a.x * b.z;
  c.z = a.z * b.w - a.y * b.x + a.w * b.z + a.x * b.y;
  return c;
}

// A B^dagger  (su2.h:56-61)
template <class R>
__device__ __forceinline__ Quat<R> q_mul_bd(const Quat<R>& a, const Quat<R>& b) {
  Quat<R> c;
  c.w = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = a.x * b.w - a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = a.y * b.w - a.z * b.x - a.w * b.y + a.x * b.z;
  c.z = a.z * b.w + a.y * b.x - a.w * b.z - a.x * b.y;
  return c;
}

// A^dagger B  (su2.h:62-67)
template <class R>
__device__ __forceinline__ Quat<R> q_mul_ad(const Quat<R>& a, const Quat<R>& b) {
  Quat<R> c;
  c.w = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = -a.x * b.w + a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = -a.y * b.w - a.z * b.x + a.w * b.y + a.x * b.z;
  c.z = -a.z * b.w + a.y * b.x + a.w * b.z - a.x * b.y;
  return c;
}

// A^dagger B^dagger  (su2.h:68-73)
template <class R>
__device__ __forceinline__ Quat<R> q_mul_adbd(const Quat<R>& a, const Quat<R>& b) {
  Quat<R> c;
  c.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = -a.x * b.w - a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = -a.y * b.w + a.z * b.x - a.w * b.y - a.x * b.z;
  c.z = -a.z * b.w - a.y * b.x - a.w * b.z + a.x * b.y;
  return c;
}

// |A|^2 = det A  (su2.h:1-3)
template <class R>
__device__ __forceinline__ R q_det(const Quat<R>& a) {
  return a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z;
}

// Re 1/2 tr(A B)  (su2.h:74-76)
template <class R>
__device__ __forceinline__ R q_retr_mul(const Quat<R>& a, const Quat<R>& b) {
  return a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
}

// A / |A| with one reciprocal square root (su2.h:4-8)
__device__ __forceinline__ Quat<double> q_normalize(const Quat<double>& a) {
  double inv = rsqrt(q_det(a));
  return Quat<double>{a.w * inv, a.x * inv, a.y * inv, a.z * inv};
}

// A / |A| and |A| (su2.h:16-21)
__device__ __forceinline__ Quat<double> q_normalize_norm(const Quat<double>& a, double* norm) {
  double det = q_det(a), inv = rsqrt(det);
  *norm = det * inv;
  return Quat<double>{a.w * inv, a.x * inv, a.y * inv, a.z * inv};
}

}  // namespace qcd
