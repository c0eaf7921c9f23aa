// Complex arithmetic on CUDA vector types for the two storage precisions:
// double2 (plain complex128 path) and float2 (mixed complex64 path).
#pragma once
#include <cuda_runtime.h>

template <typename R> struct cvec;
template <> struct cvec<double> { using type = double2; };
template <> struct cvec<float> { using type = float2; };

__host__ __device__ __forceinline__ double2 mk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ float2 mk(float r, float i) { return make_float2(r, i); }

template <typename C> __host__ __device__ __forceinline__ C czero();
template <> __host__ __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __host__ __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }

__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }

__host__ __device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ double abs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ float abs2(float2 a) { return a.x * a.x + a.y * a.y; }

// acc += a * b   (fused)
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x); acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y); acc.y = fmaf(a.y, b.x, acc.y);
}
// acc += a * conj(b)
__device__ __forceinline__ void cfma_conj(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.y, b.x, acc.y); acc.y = fma(-a.x, b.y, acc.y);
}
__device__ __forceinline__ void cfma_conj(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x); acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.y, b.x, acc.y); acc.y = fmaf(-a.x, b.y, acc.y);
}

__host__ __device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__host__ __device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
template <typename C> __host__ __device__ __forceinline__ C from_d2(double2 a);
template <> __host__ __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <> __host__ __device__ __forceinline__ float2 from_d2<float2>(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}
