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
// probability given by the discarded fraction.  The rounding is sm_100a's
// cvt.rs conversion (PTX ISA, "cvt" with the .rs rounding modifier): a
// random integer R is added to the discarded part of the value's magnitude,
// measured in units of 2^-13 (f16) or 2^-16 (bf16) of the destination's
// last place, and the magnitude rounds up when the sum carries.  Its random
// bits come from a counter-based hash of (cell, direction, time step).  The
// hash inputs name the value, not the address it is written to, so every
// copy of a population (streaming target, clamp slots, tile buffers) gets
// the same bits and all streaming policies stay bitwise equal to each other.
// Deterministic for a given run.
struct Half16SR {
    unsigned short bits;
};
struct BF16SR {
    unsigned short bits;
};

template <typename S> struct IsSR { static constexpr bool value = false; };
template <> struct IsSR<Half16SR> { static constexpr bool value = true; };
template <> struct IsSR<BF16SR> { static constexpr bool value = true; };

// Per-step seed and per-cell hash (one per cell and step): integer mixing
// in the style of the murmur3 finaliser.
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

// Random integer of direction d: bits 16-31 of the cell hash times an odd
// multiplier of the direction (mod 2^32); f16 uses its low 13 bits, bf16 all
// 16.  Directions are converted in pairs, pair k < 13 holding direction k in
// the low 16 bits and direction 26 - k in the high 16 bits (pair 13: the
// centre, low bits), so a pair's rbits word carries the integer of its low
// direction in bits 0-15 and that of its high direction in bits 16-31.
__host__ __device__ constexpr int sr_pair(int d) { return d <= 13 ? d : 26 - d; }
__host__ __device__ constexpr bool sr_high(int d) { return d > 13; }
__host__ __device__ constexpr uint32_t dir_multiplier(int d)
{
    return (0x2C1B3C6Du ^ (static_cast<uint32_t>(d) * 0x9E3779B9u)) | 1u;
}

// rbits word of direction d alone (its integer in the half that d occupies).
__device__ __forceinline__ uint32_t sr_word_dir(uint32_t hcell, int d)
{
    const uint32_t w = hcell * dir_multiplier(d);
    return sr_high(d) ? w : w >> 16;
}

// rbits word of pair k < 13 (directions k and 26 - k).
__device__ __forceinline__ uint32_t sr_word_pair(uint32_t hcell, int k)
{
    return __byte_perm(hcell * dir_multiplier(k), hcell * dir_multiplier(26 - k), 0x7632);
}

// Two FP32 values converted to one word of two 16-bit storage values, `hi`
// in bits 16-31 and `lo` in bits 0-15, in the format's raw domain (the half
// formats' 2^15 scale already applied).  Nearest-even for __half and
// __nv_bfloat16.  For the stochastic formats, `rbits` bits 0-12 (f16) or
// 0-15 (bf16) are the random integer of `lo`, bits 16-28 or 16-31 that of
// `hi`.  Each half is converted on its own: packing a value with any other
// value gives it the same bits.
template <typename S> struct Pack2;
template <> struct Pack2<__half> {
    static __device__ __forceinline__ uint32_t cvt(float hi, float lo, uint32_t)
    {
        uint32_t d;
        asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
        return d;
    }
};
template <> struct Pack2<__nv_bfloat16> {
    static __device__ __forceinline__ uint32_t cvt(float hi, float lo, uint32_t)
    {
        uint32_t d;
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
        return d;
    }
};
template <> struct Pack2<Half16SR> {
    static __device__ __forceinline__ uint32_t cvt(float hi, float lo, uint32_t rbits)
    {
        uint32_t d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
        return d;
    }
};
template <> struct Pack2<BF16SR> {
    static __device__ __forceinline__ uint32_t cvt(float hi, float lo, uint32_t rbits)
    {
        uint32_t d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
        return d;
    }
};

// The 16-bit pattern of direction d of a cell whose cell_hash for this step
// is hcell, from its raw value v (2^15 f for the half formats, f for bf16).
template <typename S>
__device__ __forceinline__ unsigned short enc16_raw(float v, uint32_t hcell, int d)
{
    const uint32_t r = IsSR<S>::value ? sr_word_dir(hcell, d) : 0u;
    if (sr_high(d)) return static_cast<unsigned short>(Pack2<S>::cvt(v, 0.0f, r) >> 16);
    return static_cast<unsigned short>(Pack2<S>::cvt(0.0f, v, r));
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

// ld_raw with the evict-first hint (ld.global.cs).
template <typename S, typename R>
__device__ __forceinline__ R ld_raw_cs(const S* p)
{
    if constexpr (std::is_same<S, __half>::value || std::is_same<S, Half16SR>::value)
        return __half2float(__ushort_as_half(__ldcs(reinterpret_cast<const unsigned short*>(p))));
    else
        return Cvt<S, R>::ld_cs(p);
}

// ld_raw from global memory with a 256-byte L2 fetch granularity
// (ld.global.L2::256B): the step kernels read every population plane as a
// stream, and on B200 the larger L2 fetch made the FP32 in-place and pull
// steps 1.3 % and 0.9 % faster.  Global addresses only (never shared memory).
template <typename S, typename R>
__device__ __forceinline__ R ld_stream_raw(const S* p)
{
    if constexpr (std::is_same<S, float>::value) {
        float v;
        asm volatile("ld.global.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
        return v;
    } else if constexpr (std::is_same<S, double>::value) {
        double v;
        asm volatile("ld.global.L2::256B.f64 %0, [%1];" : "=d"(v) : "l"(p));
        return v;
    } else {
        unsigned short b;
        asm volatile("ld.global.L2::256B.u16 %0, [%1];" : "=h"(b) : "l"(p));
        if constexpr (std::is_same<S, __half>::value || std::is_same<S, Half16SR>::value)
            return __half2float(__ushort_as_half(b));
        else
            return __uint_as_float(static_cast<uint32_t>(b) << 16);
    }
}

// Raw 16-bit store (the pattern enc16_raw gives).
template <typename S>
__device__ __forceinline__ void st16(S* p, unsigned short bits)
{
    *reinterpret_cast<unsigned short*>(p) = bits;
}
template <typename S>
__device__ __forceinline__ void st16_cs(S* p, unsigned short bits)
{
    __stcs(reinterpret_cast<unsigned short*>(p), bits);
}

// The 16-bit population formats.
template <typename S> struct Is16 { static constexpr bool value = sizeof(S) == 2; };

// The power-of-two exponent E of a format's raw scale (raw = 2^E * f; 15 for
// the scaled half formats, 0 otherwise).
template <typename S> struct ScaleExp { static constexpr int value = 0; };
template <> struct ScaleExp<__half> { static constexpr int value = 15; };
template <> struct ScaleExp<Half16SR> { static constexpr int value = 15; };

// Store of population d (value v) of the cell whose cell_hash for this step
// is hcell: the format's rounding (stochastic for the SR formats; hcell then
// feeds the random bits, otherwise it goes unused and its computation is
// dropped).
template <typename S, typename R>
__device__ __forceinline__ void put(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (Is16<S>::value)
        st16(p, enc16_raw<S>(ScaleExp<S>::value ? __fmul_rn(v, kHalfScale) : v, hcell, d));
    else
        Cvt<S, R>::st(p, v);
}

// put() of a raw value v = 2^E * f: the same bits as put(p, f, ...), without
// the scaling multiply.
template <typename S, typename R>
__device__ __forceinline__ void put_raw(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (Is16<S>::value)
        st16(p, enc16_raw<S>(v, hcell, d));
    else
        Cvt<S, R>::st(p, v);
}

// put() with the evict-first hint.
template <typename S, typename R>
__device__ __forceinline__ void put_cs(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (Is16<S>::value)
        st16_cs(p, enc16_raw<S>(ScaleExp<S>::value ? __fmul_rn(v, kHalfScale) : v, hcell, d));
    else
        Cvt<S, R>::st_cs(p, v);
}

// put_raw() with the evict-first hint when CS.
template <bool CS, typename S, typename R>
__device__ __forceinline__ void put_raw_h(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (!CS)
        put_raw(p, v, hcell, d);
    else if constexpr (Is16<S>::value)
        st16_cs(p, enc16_raw<S>(v, hcell, d));
    else
        Cvt<S, R>::st_cs(p, v);
}

// Stores the 27 raw values f of one cell, direction d at addr(d), with the
// bits of put_raw (evict-first stores when CS).  The 16-bit formats convert
// the directions in pairs (d, 26 - d) with one packed conversion per pair.
template <typename S, bool CS = false, typename R, class A>
__device__ __forceinline__ void put27_raw(const R* f, uint32_t hcell, A&& addr)
{
    if constexpr (Is16<S>::value) {
        auto st = [](S* p, unsigned short b) {
            if constexpr (CS)
                st16_cs(p, b);
            else
                st16(p, b);
        };
#pragma unroll
        for (int k = 0; k < 13; ++k) {
            const uint32_t w = Pack2<S>::cvt(f[26 - k], f[k], IsSR<S>::value ? sr_word_pair(hcell, k) : 0u);
            st(addr(k), static_cast<unsigned short>(w));
            st(addr(26 - k), static_cast<unsigned short>(w >> 16));
        }
        st(addr(13), enc16_raw<S>(f[13], hcell, 13));
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) put_raw_h<CS>(addr(d), f[d], hcell, d);
    }
}

// put27_raw for the directions d with keep(d) only (the others are not
// stored); the 16-bit formats still convert in pairs.
template <typename S, typename R, class A, class K>
__device__ __forceinline__ void put27_raw_if(const R* f, uint32_t hcell, A&& addr, K&& keep)
{
    if constexpr (Is16<S>::value) {
#pragma unroll
        for (int k = 0; k < 13; ++k) {
            const uint32_t w = Pack2<S>::cvt(f[26 - k], f[k], IsSR<S>::value ? sr_word_pair(hcell, k) : 0u);
            if (keep(k)) st16(addr(k), static_cast<unsigned short>(w));
            if (keep(26 - k)) st16(addr(26 - k), static_cast<unsigned short>(w >> 16));
        }
        if (keep(13)) st16(addr(13), enc16_raw<S>(f[13], hcell, 13));
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            if (keep(d)) put_raw(addr(d), f[d], hcell, d);
    }
}

// Arithmetic type used with each storage type.
template <typename S> struct ArithOf { using type = float; };
template <> struct ArithOf<double> { using type = double; };

}  // namespace culbm
