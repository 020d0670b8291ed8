// elem.cuh -- storage element types of the wavefield sets: FP32, or 16-bit
// (IEEE half, bfloat16) with one power-of-two scale per component.  All
// arithmetic is FP32: values are widened on load and rounded to nearest on
// store.  A stored 16-bit number s of component c stands for s * 2^k[c];
// because the scale is a power of two, scaling is exact and folds into the
// stencil's 1/h factor and the RK coefficients.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace cgfd {

enum { ELEM_F32 = 0, ELEM_F16 = 1, ELEM_BF16 = 2 };

template <typename T> struct Elem;

template <> struct Elem<float> {
  static constexpr int kind = ELEM_F32;
  __device__ __forceinline__ static float ld(const float *p) { return *p; }
  __device__ __forceinline__ static void st(float *p, float v) { *p = v; }
  __device__ __forceinline__ static float2 ld2(const float *p) {
    return *reinterpret_cast<const float2 *>(p);
  }
  __device__ __forceinline__ static void st2(float *p, float2 v) {
    *reinterpret_cast<float2 *>(p) = v;
  }
};

template <> struct Elem<__half> {
  static constexpr int kind = ELEM_F16;
  __device__ __forceinline__ static float ld(const __half *p) { return __half2float(*p); }
  __device__ __forceinline__ static void st(__half *p, float v) { *p = __float2half_rn(v); }
  __device__ __forceinline__ static float2 ld2(const __half *p) {
    return __half22float2(*reinterpret_cast<const __half2 *>(p));
  }
  __device__ __forceinline__ static void st2(__half *p, float2 v) {
    *reinterpret_cast<__half2 *>(p) = __float22half2_rn(v);
  }
};

template <> struct Elem<__nv_bfloat16> {
  static constexpr int kind = ELEM_BF16;
  __device__ __forceinline__ static float ld(const __nv_bfloat16 *p) {
    return __bfloat162float(*p);
  }
  __device__ __forceinline__ static void st(__nv_bfloat16 *p, float v) {
    *p = __float2bfloat16_rn(v);
  }
  __device__ __forceinline__ static float2 ld2(const __nv_bfloat16 *p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
  }
  __device__ __forceinline__ static void st2(__nv_bfloat16 *p, float2 v) {
    *reinterpret_cast<__nv_bfloat162 *>(p) = __float22bfloat162_rn(v);
  }
};

inline size_t elem_size(int kind) { return kind == ELEM_F32 ? 4 : 2; }

}  // namespace cgfd
