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
//   S = Half16SR, BF16SR  the same two 16-bit layouts written with
//                      stochastic rounding (see below).
#pragma once

#include <cstdint>
#include <type_traits>

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

// 16-bit storage with stochastic rounding: the same bit layouts as __half
// (scaled by 2^15) and __nv_bfloat16, but every store rounds up or down with
// probability given by the discarded fraction, driven by a counter-based hash
// of (cell, direction, time step).  The hash inputs name the value, not the
// address it is written to, so every copy of a population (streaming target,
// clamp slots, tile buffers) gets the same bits and all streaming policies
// stay bitwise equal to each other.  Deterministic for a given run.
struct Half16SR {
    unsigned short bits;
};
struct BF16SR {
    unsigned short bits;
};

template <typename S> struct IsSR { static constexpr bool value = false; };
template <> struct IsSR<Half16SR> { static constexpr bool value = true; };
template <> struct IsSR<BF16SR> { static constexpr bool value = true; };

// Per-step seed, per-cell hash (one per cell and step) and per-direction
// random bits.  Integer mixing in the style of the murmur3 finaliser; the
// per-direction bits are a multiplicative hash whose high bits are used.
__host__ __device__ __forceinline__ uint32_t step_seed(uint32_t t)
{
    uint32_t h = t * 0x9E3779B1u + 0x7F4A7C15u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ uint32_t cell_hash(uint32_t cell, uint32_t seed)
{
    uint32_t h = cell * 0x27D4EB2Fu ^ seed;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// Random bits of direction d: the cell hash times an odd multiplier of its
// own per direction (one multiply; the high bits are used).
__host__ __device__ constexpr uint32_t dir_multiplier(uint32_t d)
{
    return (0x2C1B3C6Du ^ (d * 0x9E3779B9u)) | 1u;
}

__device__ __forceinline__ uint32_t dir_bits(uint32_t hcell, uint32_t d)
{
    return hcell * dir_multiplier(d);
}

template <> struct Cvt<Half16SR, float> {
    static __device__ __forceinline__ float ld(const Half16SR* p)
    {
        return __fmul_rn(__half2float(__ushort_as_half(p->bits)), kHalfInvScale);
    }
    static __device__ __forceinline__ float ld_cs(const Half16SR* p)
    {
        return __fmul_rn(__half2float(__ushort_as_half(__ldcs(&p->bits))), kHalfInvScale);
    }
    // nearest-even (used only for exact values such as the rest state)
    static __device__ __forceinline__ void st(Half16SR* p, float v)
    {
        p->bits = __half_as_ushort(__float2half_rn(__fmul_rn(v, kHalfScale)));
    }
    // stochastic: add 13 random bits (the high bits of rnd) below the half's
    // last mantissa bit, truncate
    static __device__ __forceinline__ unsigned short enc(float v, uint32_t rnd)
    {
        const uint32_t u = __float_as_uint(__fmul_rn(v, kHalfScale)) + (rnd >> 19);
        return __half_as_ushort(__float2half_rz(__uint_as_float(u)));
    }
    static __device__ __forceinline__ void st_sr(Half16SR* p, float v, uint32_t rnd) { p->bits = enc(v, rnd); }
    static __device__ __forceinline__ void st_sr_cs(Half16SR* p, float v, uint32_t rnd) { __stcs(&p->bits, enc(v, rnd)); }
};

template <> struct Cvt<BF16SR, float> {
    static __device__ __forceinline__ float ld(const BF16SR* p) { return __uint_as_float(uint32_t(p->bits) << 16); }
    static __device__ __forceinline__ float ld_cs(const BF16SR* p)
    {
        return __uint_as_float(uint32_t(__ldcs(&p->bits)) << 16);
    }
    static __device__ __forceinline__ void st(BF16SR* p, float v)
    {
        p->bits = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
    static __device__ __forceinline__ unsigned short enc(float v, uint32_t rnd)
    {
        return static_cast<unsigned short>((__float_as_uint(v) + (rnd >> 16)) >> 16);
    }
    static __device__ __forceinline__ void st_sr(BF16SR* p, float v, uint32_t rnd) { p->bits = enc(v, rnd); }
    static __device__ __forceinline__ void st_sr_cs(BF16SR* p, float v, uint32_t rnd) { __stcs(&p->bits, enc(v, rnd)); }
};

// Raw load for consumers that are linear in the populations: the stored
// value without the format's power-of-two scale; f = RawScale<S>::value * raw.
template <typename S> struct RawScale { static constexpr float value = 1.0f; };
template <> struct RawScale<__half> { static constexpr float value = kHalfInvScale; };
template <> struct RawScale<Half16SR> { static constexpr float value = kHalfInvScale; };

template <typename S, typename R>
__device__ __forceinline__ R ld_raw(const S* p)
{
    if constexpr (std::is_same<S, __half>::value)
        return __half2float(*p);
    else if constexpr (std::is_same<S, Half16SR>::value)
        return __half2float(__ushort_as_half(p->bits));
    else
        return Cvt<S, R>::ld(p);
}

// Store of population d of the cell whose cell_hash for this step is hcell:
// stochastic rounding for the SR formats, the format's plain conversion
// otherwise (hcell then goes unused and its computation is dropped).
template <typename S, typename R>
__device__ __forceinline__ void put(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (IsSR<S>::value)
        Cvt<S, R>::st_sr(p, v, dir_bits(hcell, d));
    else
        Cvt<S, R>::st(p, v);
}

// The 16-bit population formats.
template <typename S> struct Is16 { static constexpr bool value = sizeof(S) == 2; };

// The power-of-two exponent E of a format's raw scale (raw = 2^E * f; 15 for
// the scaled half formats, 0 otherwise).
template <typename S> struct ScaleExp { static constexpr int value = 0; };
template <> struct ScaleExp<__half> { static constexpr int value = 15; };
template <> struct ScaleExp<Half16SR> { static constexpr int value = 15; };

// put() of a raw value v = 2^E * f: the same bits as put(p, f, ...), without
// the scaling multiply.
template <typename S, typename R>
__device__ __forceinline__ void put_raw(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (std::is_same<S, __half>::value) {
        *p = __float2half_rn(v);
    } else if constexpr (std::is_same<S, Half16SR>::value) {
        const uint32_t u = __float_as_uint(v) + (dir_bits(hcell, d) >> 19);
        p->bits = __half_as_ushort(__float2half_rz(__uint_as_float(u)));
    } else {
        put(p, v, hcell, d);
    }
}

template <typename S, typename R>
__device__ __forceinline__ void put_cs(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (IsSR<S>::value)
        Cvt<S, R>::st_sr_cs(p, v, dir_bits(hcell, d));
    else
        Cvt<S, R>::st_cs(p, v);
}

// Arithmetic type used with each storage type.
template <typename S> struct ArithOf { using type = float; };
template <> struct ArithOf<double> { using type = double; };

}  // namespace culbm
