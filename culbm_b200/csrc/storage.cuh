// Population storage formats and the load/store conversions between the
// storage type S in HBM and the arithmetic type R in registers.
//
//   S = float          FP32 storage, FP32 arithmetic (the reference's format)
//   S = double         FP64 storage and arithmetic (the GPU oracle)
//   S = __half         FP16 storage of the shifted population f_i - w_i, scaled
//                      by 2^15 so that small deviations stay in the normal
//                      range; FP32 arithmetic.  The scale is a power of two,
//                      so only the half rounding (nearest-even) loses bits.
//   S = __nv_bfloat16  BF16 storage of f_i - w_i (float exponent range, no
//                      scale); FP32 arithmetic, nearest-even rounding.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace culbm {

constexpr float kHalfScale = 32768.0f;          // 2^15
constexpr float kHalfInvScale = 1.0f / 32768.0f;

template <typename S, typename R> struct Cvt;

// ld_cs / st_cs: streaming ("evict first") variants for data touched once per
// pass, so that it does not push L2-resident tile data out.
template <> struct Cvt<float, float> {
    static __device__ __forceinline__ float ld(const float* p) { return *p; }
    static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
    static __device__ __forceinline__ float ld_cs(const float* p) { return __ldcs(p); }
    static __device__ __forceinline__ void st_cs(float* p, float v) { __stcs(p, v); }
};

template <> struct Cvt<double, double> {
    static __device__ __forceinline__ double ld(const double* p) { return *p; }
    static __device__ __forceinline__ void st(double* p, double v) { *p = v; }
    static __device__ __forceinline__ double ld_cs(const double* p) { return __ldcs(p); }
    static __device__ __forceinline__ void st_cs(double* p, double v) { __stcs(p, v); }
};

template <> struct Cvt<__half, float> {
    static __device__ __forceinline__ float ld(const __half* p)
    {
        return __fmul_rn(__half2float(*p), kHalfInvScale);
    }
    static __device__ __forceinline__ void st(__half* p, float v)
    {
        *p = __float2half_rn(__fmul_rn(v, kHalfScale));
    }
    static __device__ __forceinline__ float ld_cs(const __half* p)
    {
        return __fmul_rn(__half2float(__ldcs(p)), kHalfInvScale);
    }
    static __device__ __forceinline__ void st_cs(__half* p, float v)
    {
        __stcs(p, __float2half_rn(__fmul_rn(v, kHalfScale)));
    }
};

template <> struct Cvt<__nv_bfloat16, float> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
    static __device__ __forceinline__ float ld_cs(const __nv_bfloat16* p) { return __bfloat162float(__ldcs(p)); }
    static __device__ __forceinline__ void st_cs(__nv_bfloat16* p, float v) { __stcs(p, __float2bfloat16_rn(v)); }
};

// Arithmetic type used with each storage type.
template <typename S> struct ArithOf { using type = float; };
template <> struct ArithOf<double> { using type = double; };

}  // namespace culbm
