// Minimal complex arithmetic on float2 / double2 for the link kernels.
#pragma once
#include <cuda_runtime.h>

namespace u1b {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
// conj(a) * conj(b) = conj(a*b)
__device__ __forceinline__ float2 cconjmul(float2 a, float2 b) {
  float2 m = cmul(a, b);
  return make_float2(m.x, -m.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// Im(a * b)
__device__ __forceinline__ float cim_mul(float2 a, float2 b) { return fmaf(a.x, b.y, a.y * b.x); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// wa*a + wb*b with an explicit fused multiply-add, so every kernel that
// forms a staple rounds it identically (the library is built with
// -fmad=false: no compiler-chosen contractions).
__device__ __forceinline__ float2 cweigh(float2 a, float wa, float2 b, float wb) {
  return make_float2(fmaf(a.x, wa, b.x * wb), fmaf(a.y, wa, b.y * wb));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// Re(a * b)
__device__ __forceinline__ float cre_mul(float2 a, float2 b) { return fmaf(a.x, b.x, -a.y * b.y); }

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

}  // namespace u1b
