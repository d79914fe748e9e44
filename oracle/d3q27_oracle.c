/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement of the reference's single-device D3Q27 BGK hot path
 * (cuLBM, src/simulator/single_dev_expt/kernel.cu StaticD3Q27PullKernel and
 * StaticD3Q27PullDumpKernel over the lbm_core routines of
 * src/lbm_core/device_function.hpp).  It is the checker for the CUDA kernels
 * of culbm_b200: only the tests, the smoke check and bench.py's CPU-baseline
 * leg may load it.  The product never links or calls it.
 *
 * Built with -ffp-contract=off (see oracle/Makefile) so that a*b+c stays two
 * roundings and only the reference's explicit fma calls are fused.  With that,
 * the FP32 instance rounds exactly like the reference routines compiled for
 * the host; the test suite pins this against those routines (oracle/_ref) and
 * against the committed golden fixtures.
 */
#include <math.h>
#include <stdint.h>

/* Flag bits, src/simulator/single_dev_expt/local_config.hpp:12-22. */
#define ORC_LOAD        (1u << 0)
#define ORC_EQU         (1u << 1)
#define ORC_COLLIDE     (1u << 2)
#define ORC_BOUNCE_BACK (1u << 3)
#define ORC_STORE       (1u << 4)
#define ORC_DUMP_RHO    (1u << 27)
#define ORC_DUMP_VX     (1u << 28)
#define ORC_DUMP_VY     (1u << 29)
#define ORC_DUMP_VZ     (1u << 30)
#define ORC_CORRECT     (1u << 31)

#define REAL float
#define SFX f32
#define FMA fmaf
#include "d3q27_oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

#define REAL double
#define SFX f64
#define FMA fma
#include "d3q27_oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

/* Blocking geometry of the reference's temporal blocking.
 * Restates blocking_core::validBlkAxisConfig / calcBlkNum / calcValidPrev,
 * src/blocking_core/blocking_alogrithm.hpp:7-41 (unsigned arithmetic as the
 * simulator instantiates them with std::uint32_t). */
int orc_valid_blk_axis(uint32_t dom, uint32_t blk, uint32_t iter)
{
    if (blk < dom && blk + 1 <= iter) return 0;
    if (2 * (blk + 1 - iter) < dom && blk + 2 <= iter) return 0;
    return 1;
}

uint32_t orc_blk_num(uint32_t dom, uint32_t blk, uint32_t iter)
{
    if (dom <= blk) return 1;
    if (dom <= 2 * (blk + 1 - iter)) return 2;
    const uint32_t num = dom - 2 * (blk + 1 - iter);
    const uint32_t den = blk + 2 - 2 * iter;
    return 2 + (num + den - 1) / den;
}

int32_t orc_valid_prev(int32_t idx, int32_t blk, int32_t num, int32_t iter, int32_t dom)
{
    if (idx == num) return dom;
    if (idx == 0) return 0;
    return (blk + 1 - iter) + (idx - 1) * (blk + 2 - 2 * iter);
}

/* ---------------------------------------------------------------------------
 * 16-bit population storage (no reference counterpart): the stored value is
 * the shifted population f_i - w_i as IEEE half scaled by 2^15 (kind 0, 2)
 * or as bfloat16 (kind 1, 3); arithmetic in FP32.  Kinds 0/1 round to nearest
 * even, kinds 2/3 round stochastically with random bits from a counter-based
 * hash of (cell, direction, time step).  A step is: widen src to FP32, one FP32
 * pull step, narrow every cell back.  Widening and narrowing a stored value
 * gives it back exactly, so cells without STORE keep their old bits.
 * ------------------------------------------------------------------------- */
#include <stdlib.h>
#include <string.h>

static uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

uint32_t orc_step_seed(uint32_t t)
{
    uint32_t h = t * 0x9E3779B1u + 0x7F4A7C15u;
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}

/* Per-cell hash of the step seeded by `seed` (murmur3-style finaliser). */
static uint32_t orc_cell_hash(uint32_t cell, uint32_t seed)
{
    uint32_t h = cell * 0x27D4EB2Fu ^ seed;
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}

/* The random integer of population d of `cell` at the step seeded by `seed`:
 * bits 16-31 of the cell hash times an odd multiplier of d (mod 2^32); f16
 * uses its low 13 bits, bf16 all 16. */
uint32_t orc_sr_bits(uint32_t cell, uint32_t d, uint32_t seed)
{
    const uint32_t m = (0x2C1B3C6Du ^ (d * 0x9E3779B9u)) | 1u;
    return (orc_cell_hash(cell, seed) * m) >> 16;
}

/* Stochastic rounding of an FP32 value to IEEE half (PTX cvt.rs.f16x2.f32,
 * one half; no saturation): with q = |v| / ulp, ulp the half's last place at
 * |v| (2^-24 below the normal range), the magnitude is floor(q), plus one when
 * floor(frac(q) * 2^13) + r13 >= 2^13.  NaN gives 0x7FFF; a result at or above
 * 2^16 is infinite. */
uint16_t orc_round_f16_sr(float v, uint32_t r13)
{
    const uint32_t u = f2u(v);
    const uint16_t sign = (uint16_t)((u >> 16) & 0x8000u);
    const uint32_t mag = u & 0x7FFFFFFFu;
    r13 &= 0x1FFFu;
    if (mag > 0x7F800000u) return 0x7FFF;
    if (mag == 0x7F800000u) return sign | 0x7C00;
    const int E = (int)(mag >> 23);
    if (E == 0) return sign;                       /* below 2^-126: frac(q) * 2^13 < 1 */
    const uint32_t sig = (mag & 0x7FFFFFu) | 0x800000u;
    const int e = E - 127;
    uint32_t m, frac;
    if (e >= -14) {                                /* normal half: 13 discarded bits */
        m = sig >> 13;
        frac = sig & 0x1FFFu;
    } else {                                       /* subnormal half: units of 2^-24 */
        const int sh = 126 - E;
        m = sh < 32 ? sig >> sh : 0u;
        frac = (sh - 13) < 32 ? (sig >> (sh - 13)) & 0x1FFFu : 0u;
    }
    if (frac + r13 >= 0x2000u) m += 1;
    if (e < -14) return sign | (uint16_t)m;        /* m = 1024 is the smallest normal */
    if (e > 15) return sign | 0x7C00;
    uint32_t h = ((uint32_t)(e + 15) << 10) + (m - 1024u);
    if (h > 0x7C00u) h = 0x7C00u;
    return sign | (uint16_t)h;
}

/* Stochastic rounding of an FP32 value to bfloat16 (PTX cvt.rs.bf16x2.f32, one
 * half; no saturation): r16 added to the 16 discarded bits of the magnitude,
 * then truncated.  NaN gives 0x7FFF. */
uint16_t orc_round_bf16_sr(float v, uint32_t r16)
{
    const uint32_t u = f2u(v);
    const uint32_t mag = u & 0x7FFFFFFFu;
    const uint16_t sign = (uint16_t)((u >> 16) & 0x8000u);
    if (mag > 0x7F800000u) return 0x7FFF;
    if (mag == 0x7F800000u) return sign | 0x7F80;
    return sign | (uint16_t)((mag + (r16 & 0xFFFFu)) >> 16);
}

static float h16_decode(uint16_t h)
{
    _Float16 v;
    memcpy(&v, &h, 2);
    return (float)v * (1.0f / 32768.0f);
}

static uint16_t h16_encode_rn(float v)
{
    _Float16 h = (_Float16)(v * 32768.0f);   /* nearest-even */
    uint16_t b;
    memcpy(&b, &h, 2);
    return b;
}

static float b16_decode(uint16_t b) { return u2f((uint32_t)b << 16); }

static uint16_t b16_encode_rn(float v)
{
    const uint32_t u = f2u(v);
    return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

static float s16_decode(int kind, uint16_t b) { return (kind & 1) ? b16_decode(b) : h16_decode(b); }

static uint16_t s16_encode(int kind, float v, uint32_t cell, uint32_t d, uint32_t seed)
{
    switch (kind) {
        case 0: return h16_encode_rn(v);
        case 1: return b16_encode_rn(v);
        case 2: return orc_round_f16_sr(v * 32768.0f, orc_sr_bits(cell, d, seed));
        default: return orc_round_bf16_sr(v, orc_sr_bits(cell, d, seed));
    }
}

/* ---- compact FP32 update used with 16-bit storage ------------------------
 * The 16-bit formats keep about three significant digits, so culbm_b200 does
 * the cell arithmetic of those formats in a shorter form (fused multiply-adds,
 * pair symmetry c_{26-d} = -c_d) instead of the reference's operation order.
 * This is that form, operation for operation (compiled without contraction,
 * explicit fmaf):
 *   dr = f_13 + sum_{d<13} (f_d + f_{26-d}),  rho = 1 + dr,
 *   j = sum_{d<13} c_d (f_d - f_{26-d}),
 *   w feq_d = A_k (P + 3 c_d.u) + C_k,  P = 9/2 (c_d.u)^2 - 3/2 |u|^2,
 *   A_k = w W_k rho, C_k = w W_k dr,  f_d <- (1 - w) f_d + w feq_d. */
static float cdot_fast(int d, float ux, float uy, float uz)
{
    const int cx = d % 3 - 1, cy = (d / 3) % 3 - 1, cz = d / 9 - 1;
    float v = cx == 1 ? ux : cx == -1 ? -ux : 0.0f;
    if (cy != 0) v = cx == 0 ? (cy == 1 ? uy : -uy) : (cy == 1 ? v + uy : v - uy);
    if (cz != 0) v = (cx == 0 && cy == 0) ? (cz == 1 ? uz : -uz) : (cz == 1 ? v + uz : v - uz);
    return v;
}

static void fast_class_terms(float w, float rho, float dr, float *Ak, float *Ck)
{
    const float W[4] = {8.0f / 27.0f, 2.0f / 27.0f, 1.0f / 54.0f, 1.0f / 216.0f};
    for (int k = 0; k < 4; ++k) {
        const float b = w * W[k];
        Ak[k] = b * rho;
        Ck[k] = b * dr;
    }
}

static void fast_relax(int relax, float om, float ux, float uy, float uz, const float *Ak, const float *Ck, float *f)
{
    const float uu = fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    const float base = -1.5f * uu;
    for (int d = 0; d < 13; ++d) {
        const int e = 26 - d;
        const int k = (d % 3 != 1) + ((d / 3) % 3 != 1) + (d / 9 != 1);
        const float cu = cdot_fast(d, ux, uy, uz);
        const float P = fmaf(4.5f * cu, cu, base);
        const float ed = fmaf(Ak[k], fmaf(3.0f, cu, P), Ck[k]);
        const float ee = fmaf(Ak[k], fmaf(-3.0f, cu, P), Ck[k]);
        f[d] = relax ? fmaf(om, f[d], ed) : ed;
        f[e] = relax ? fmaf(om, f[e], ee) : ee;
    }
    const float e13 = fmaf(Ak[0], base, Ck[0]);
    f[13] = relax ? fmaf(om, f[13], e13) : e13;
}

void orc_cell_fast_f32(uint32_t flag, float w, float rho_in, float vx_in, float vy_in, float vz_in, float *f)
{
    float Ak[4], Ck[4];
    if (flag & ORC_EQU) {
        fast_class_terms(1.0f, rho_in, rho_in - 1.0f, Ak, Ck);
        fast_relax(0, 0.0f, vx_in, vy_in, vz_in, Ak, Ck, f);
    }
    if (flag & ORC_BOUNCE_BACK)
        for (int d = 0; d < 13; ++d) {
            const float t = f[d];
            f[d] = f[26 - d];
            f[26 - d] = t;
        }
    if (!(flag & ORC_COLLIDE)) return;
    float r = f[13], jx = 0.0f, jy = 0.0f, jz = 0.0f;
    int hx = 0, hy = 0, hz = 0;
    for (int d = 0; d < 13; ++d) {
        const int cx = d % 3 - 1, cy = (d / 3) % 3 - 1, cz = d / 9 - 1;
        const float sp = f[d] + f[26 - d], tm = f[d] - f[26 - d];
        r = r + sp;
        if (cx) { jx = hx ? (cx == 1 ? jx + tm : jx - tm) : (cx == 1 ? tm : -tm); hx = 1; }
        if (cy) { jy = hy ? (cy == 1 ? jy + tm : jy - tm) : (cy == 1 ? tm : -tm); hy = 1; }
        if (cz) { jz = hz ? (cz == 1 ? jz + tm : jz - tm) : (cz == 1 ? tm : -tm); hz = 1; }
    }
    const float dr = r, rho = 1.0f + dr, inv = 1.0f / rho;
    const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
    fast_class_terms(w, rho, dr, Ak, Ck);
    fast_relax(1, 1.0f - w, ux, uy, uz, Ak, Ck, f);
}

/* The FP32 pull step of orc_step_f32 with the compact cell update. */
void orc_step_fast_f32(int64_t nx, int64_t ny, int64_t nz, const uint32_t *flag, const float *rho, const float *vx,
                       const float *vy, const float *vz, float inv_tau, const float *src, float *dst)
{
    const int64_t n = nx * ny * nz;
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t i = (ny * z + y) * nx + x;
                const uint32_t fl = flag[i];
                float f[27];
                for (int d = 0; d < 27; ++d) f[d] = 0;
                if (fl & ORC_LOAD) orc_pull_f32(nx, ny, nz, x, y, z, src, f);
                orc_cell_fast_f32(fl, inv_tau, rho[i], vx[i], vy[i], vz[i], f);
                if (fl & ORC_STORE)
                    for (int d = 0; d < 27; ++d) dst[d * n + i] = f[d];
            }
}

/* One step with 16-bit storage; `t` is the index of the step being taken
 * (0 for the first step after loading), which seeds stochastic rounding. */
void orc_step_s16(int kind, int64_t nx, int64_t ny, int64_t nz, const uint32_t *flag,
                  const float *rho, const float *vx, const float *vy, const float *vz,
                  float inv_tau, const uint16_t *src, uint16_t *dst, uint32_t t)
{
    const int64_t n = nx * ny * nz;
    float *a = (float *)malloc(sizeof(float) * 27 * n);
    float *b = (float *)malloc(sizeof(float) * 27 * n);
    for (int64_t k = 0; k < 27 * n; ++k) {
        a[k] = s16_decode(kind, src[k]);
        b[k] = s16_decode(kind, dst[k]);
    }
    orc_step_fast_f32(nx, ny, nz, flag, rho, vx, vy, vz, inv_tau, a, b);
    const uint32_t seed = orc_step_seed(t);
    for (int64_t d = 0; d < 27; ++d)
        for (int64_t i = 0; i < n; ++i) {
            if (flag[i] & ORC_STORE)
                dst[d * n + i] = s16_encode(kind, b[d * n + i], (uint32_t)i, (uint32_t)d, seed);
        }
    free(a);
    free(b);
}

/* Widen a 16-bit state to FP32 (for comparisons). */
void orc_decode_s16(int kind, int64_t count, const uint16_t *src, float *out)
{
    for (int64_t k = 0; k < count; ++k) out[k] = s16_decode(kind, src[k]);
}

/* Narrow an FP32 state (rest state, imports) with nearest-even or the
 * stochastic rule keyed on (cell, direction, seed of step t). */
void orc_encode_s16(int kind, int64_t n, const float *src, uint16_t *out, uint32_t t)
{
    const uint32_t seed = orc_step_seed(t);
    for (int64_t d = 0; d < 27; ++d)
        for (int64_t i = 0; i < n; ++i)
            out[d * n + i] = s16_encode(kind, src[d * n + i], (uint32_t)i, (uint32_t)d, seed);
}

/* Element-wise stochastic rounding of n FP32 values with their random
 * integers r[k]: IEEE half (kind 0, orc_round_f16_sr) or bfloat16 (kind 1,
 * orc_round_bf16_sr). */
void orc_round16_sr_n(int kind, int64_t n, const float *v, const uint32_t *r, uint16_t *out)
{
    for (int64_t k = 0; k < n; ++k)
        out[k] = kind ? orc_round_bf16_sr(v[k], r[k]) : orc_round_f16_sr(v[k], r[k]);
}
