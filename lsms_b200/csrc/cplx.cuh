// Complex FP64 helpers of the elimination and sweep kernels (double2 = re, im).
#pragma once

#include <cuda_runtime.h>

namespace b200 {
namespace cx {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // c + a b
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ double2 crecip(double2 a) {
  // 1/a with scaling against overflow of |a|^2
  const double s = fmax(fabs(a.x), fabs(a.y));
  const double ar = a.x / s, ai = a.y / s;
  const double d = ar * ar + ai * ai;
  return make_double2(ar / (d * s), -ai / (d * s));
}
// Loads and stores of the factor storage (FP64 or FP32), arithmetic in FP64.
__device__ __forceinline__ double2 ldc(const double2 *p) { return *p; }
__device__ __forceinline__ double2 ldc(const float2 *p) {
  const float2 v = *p;
  return make_double2(v.x, v.y);
}
__device__ __forceinline__ void stc(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void stc(float2 *p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

// FP32 complex multiply-add (c + a b).
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  c.x = fmaf(a.x, b.x, c.x);
  c.x = fmaf(-a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y);
  c.y = fmaf(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Conversions between the storage type and the arithmetic type V (double2 or float2).
template <typename V> __device__ __forceinline__ V to_v(double2 a);
template <> __device__ __forceinline__ double2 to_v<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 to_v<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <typename V> __device__ __forceinline__ V to_v(float2 a);
template <> __device__ __forceinline__ double2 to_v<double2>(float2 a) { return make_double2(a.x, a.y); }
template <> __device__ __forceinline__ float2 to_v<float2>(float2 a) { return a; }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
template <typename V> __device__ __forceinline__ V vzero();
template <> __device__ __forceinline__ double2 vzero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 vzero<float2>() { return make_float2(0.f, 0.f); }

// Refinement round skip flag (set on the device by the convergence check, read by later launches).
__device__ __forceinline__ bool converged(const int *conv) {
  return conv != nullptr && *reinterpret_cast<volatile const int *>(conv) != 0;
}

}  // namespace cx
}  // namespace b200
