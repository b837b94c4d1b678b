// dmb_device.cuh -- device-side helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#define DMB_INV_FOUR_PI 0.07957747154594767  // 1/(4*pi) rounded to binary64

// ---------------------------------------------------------------------------
// complex arithmetic on double2 / float2 (re = x, im = y)
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// a / b for complex b (Smith's algorithm)
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
__host__ __device__ __forceinline__ float2 caddf(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cdivf(float2 a, float2 b) {
  if (fabsf(b.x) >= fabsf(b.y)) {
    float r = b.y / b.x, d = b.x + b.y * r;
    return make_float2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    float r = b.x / b.y, d = b.x * r + b.y;
    return make_float2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}

// float2 overloads so templates can use one spelling for both precisions
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cdiv(float2 a, float2 b) { return cdivf(a, b); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
// a += b * c
__device__ __forceinline__ void cfma(double2 &a, double2 b, double2 c) {
  a.x = fma(b.x, c.x, a.x);
  a.x = fma(-b.y, c.y, a.x);
  a.y = fma(b.x, c.y, a.y);
  a.y = fma(b.y, c.x, a.y);
}
__device__ __forceinline__ void cfma(float2 &a, float2 b, float2 c) {
  a.x = fmaf(b.x, c.x, a.x);
  a.x = fmaf(-b.y, c.y, a.x);
  a.y = fmaf(b.x, c.y, a.y);
  a.y = fmaf(b.y, c.x, a.y);
}
template <class C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }
template <class C> __device__ __forceinline__ C cone();
template <> __device__ __forceinline__ double2 cone<double2>() { return make_double2(1.0, 0.0); }
template <> __device__ __forceinline__ float2 cone<float2>() { return make_float2(1.f, 0.f); }
__device__ __forceinline__ double cabsv(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ float cabsv(float2 a) { return hypotf(a.x, a.y); }

// storage conversion
template <class T> struct CplxOf;
template <> struct CplxOf<double> { typedef double2 type; };
template <> struct CplxOf<float> { typedef float2 type; };

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }
__device__ __forceinline__ void store_c(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void store_c(float2 *p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

// ---------------------------------------------------------------------------
// warp / block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double2 warp_sum2(double2 v) {
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
