// Device helpers shared by the register-streaming H*x kernels (spmv_lane.cu,
// spmv_pen.cu): 16-byte loads of block rows and vector segments, complex
// multiply-adds, and explicitly rounded products for epilogues that several
// launch shapes must round identically.
#pragma once

namespace tbgpu {
namespace lanemath {

template <typename V> struct RealOf;
template <> struct RealOf<double2> { using T = double; };
template <> struct RealOf<float2> { using T = float; };

// two consecutive block rows (20 elements) by 16-byte read-only loads;
// the pair starts on a 16-byte boundary (rows of 10 doubles are 80 bytes,
// a pair of float rows 80 bytes)
__device__ __forceinline__ void load_rows2(const double *__restrict__ p, double (&r)[20]) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
  for (int k = 0; k < 10; k++) {
    const double2 v = __ldg(q + k);
    r[2 * k] = v.x;
    r[2 * k + 1] = v.y;
  }
}
__device__ __forceinline__ void load_rows2(const float *__restrict__ p, float (&r)[20]) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const float4 v = __ldg(q + k);
    r[4 * k] = v.x;
    r[4 * k + 1] = v.y;
    r[4 * k + 2] = v.z;
    r[4 * k + 3] = v.w;
  }
}
// one spin's x segment (10 complex), 16-byte aligned
__device__ __forceinline__ void load_seg(const double2 *__restrict__ p, double2 (&v)[10]) {
#pragma unroll
  for (int k = 0; k < 10; k++) v[k] = __ldg(p + k);
}
__device__ __forceinline__ void load_seg(const float2 *__restrict__ p, float2 (&v)[10]) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const float4 t = __ldg(q + k);
    v[2 * k] = make_float2(t.x, t.y);
    v[2 * k + 1] = make_float2(t.z, t.w);
  }
}
// two consecutive complex entries (the first on a 16-byte boundary)
__device__ __forceinline__ void load_pair(const double2 *__restrict__ p, double2 &a, double2 &b) {
  a = __ldg(p);
  b = __ldg(p + 1);
}
__device__ __forceinline__ void load_pair(const float2 *__restrict__ p, float2 &a, float2 &b) {
  const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
  a = make_float2(t.x, t.y);
  b = make_float2(t.z, t.w);
}

template <typename T, typename V>
__device__ __forceinline__ void cfma(V &acc, T h, V x) {
  acc.x = fma(h, x.x, acc.x);
  acc.y = fma(h, x.y, acc.y);
}
// acc += (i * lam) * x
template <typename T, typename V>
__device__ __forceinline__ void cfma_im(V &acc, T lam, V x) {
  acc.x = fma(-lam, x.y, acc.x);
  acc.y = fma(lam, x.x, acc.y);
}

// products that are never contracted into an FMA, so that every launch
// shape rounds the epilogue the same way
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }


}  // namespace lanemath
}  // namespace tbgpu
