// D3Q27 lattice constants and the per-cell BGK arithmetic shared by every
// kernel of the library (pull, in-place, L2-tile, FP64).
//
// Direction numbering follows the reference's VelSet3D<27>
// (src/basic/velocity_set.hpp:189-255): d = (cx+1) + 3*(cy+1) + 9*(cz+1),
// centre 13, opposite 26-d.  Populations are stored shifted, f_i - w_i, so
// rho = 1 + sum(f).
//
// All arithmetic goes through explicit round-to-nearest intrinsics.  nvcc
// never contracts them, so a*b + c stays two roundings exactly as in the
// reference's routines compiled for the host with contraction disabled, and
// only the reference's own fma() calls are fused.  Every kernel therefore
// produces the same bits for the same cell, which is what makes the blocked
// and in-place policies bitwise equal to the plain pull step.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace culbm {

// Flag bits of the init-state flag.dat word,
// reference src/simulator/single_dev_expt/local_config.hpp:12-22.
constexpr uint32_t FLAG_LOAD = 1u << 0;
constexpr uint32_t FLAG_EQU = 1u << 1;
constexpr uint32_t FLAG_COLLIDE = 1u << 2;
constexpr uint32_t FLAG_BOUNCE_BACK = 1u << 3;
constexpr uint32_t FLAG_STORE = 1u << 4;
constexpr uint32_t FLAG_DUMP_RHO = 1u << 27;
constexpr uint32_t FLAG_DUMP_VX = 1u << 28;
constexpr uint32_t FLAG_DUMP_VY = 1u << 29;
constexpr uint32_t FLAG_DUMP_VZ = 1u << 30;
constexpr uint32_t FLAG_CORRECT = 1u << 31;

// Device-side compact operation byte: the five step bits keep their
// positions; bit 5 marks a cell on the domain boundary (some neighbour is
// outside), bit 6 marks a cell with at least one DUMP bit.
constexpr uint8_t OP_LOAD = 1u << 0;
constexpr uint8_t OP_EQU = 1u << 1;
constexpr uint8_t OP_COLLIDE = 1u << 2;
constexpr uint8_t OP_BB = 1u << 3;
constexpr uint8_t OP_STORE = 1u << 4;
constexpr uint8_t OP_EDGE = 1u << 5;
constexpr uint8_t OP_SOFT = 1u << 6;   // soft-obstacle cell (adjoint model only)

constexpr int Q = 27;

__host__ __device__ constexpr int cx_of(int d) { return d % 3 - 1; }
__host__ __device__ constexpr int cy_of(int d) { return (d / 3) % 3 - 1; }
__host__ __device__ constexpr int cz_of(int d) { return d / 9 - 1; }
__host__ __device__ constexpr int opp_of(int d) { return 26 - d; }

// Compile-time loop over the 27 directions: f(std::integral_constant<int, d>).
template <int D_ = 0, class F>
__device__ __forceinline__ void for_dirs(F&& f)
{
    if constexpr (D_ < 27) {
        f(std::integral_constant<int, D_>{});
        for_dirs<D_ + 1>(f);
    }
}

// Lattice weights w_d (8/27 centre, 2/27 face, 1/54 edge, 1/216 corner).
template <typename R>
__host__ __device__ constexpr R weight(int d)
{
    const int k = (cx_of(d) != 0) + (cy_of(d) != 0) + (cz_of(d) != 0);
    return k == 0 ? R(8) / R(27) : k == 1 ? R(2) / R(27) : k == 2 ? R(1) / R(54) : R(1) / R(216);
}

// Round-to-nearest arithmetic with contraction ruled out.
template <typename R> struct Rn;
template <> struct Rn<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
};
template <> struct Rn<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

// Exact power-of-two factors 2^E and 2^-E.
template <typename R, int E>
__host__ __device__ constexpr R pow2()
{
    R v = R(1);
    for (int k = 0; k < (E > 0 ? E : -E); ++k) v = E > 0 ? v * R(2) : v / R(2);
    return v;
}

// rho = 1 + sum f in the reference's pairing, u = (sum c f) * (1/rho).
// Same operation order as bgk::detail::calcRhoU<27>,
// reference src/lbm_core/device_function.hpp:439-463.
// With E > 0, f holds raw values 2^E * f: every sum is the exact 2^E
// multiple of the unscaled one, so rho and u come out with the same bits.
template <typename R, int E = 0>
__device__ __forceinline__ void moments(const R* f, R& rho, R& ux, R& uy, R& uz)
{
    using A = Rn<R>;
    R s = A::add(pow2<R, E>(), f[0]);
#pragma unroll
    for (int k = 1; k < 27; k += 2) s = A::add(s, A::add(f[k], f[k + 1]));
    rho = E ? A::mul(s, pow2<R, -E>()) : s;
    const R inv = A::div(R(1), rho);
    // x: pairs (3k+2, 3k); y: (9s+6+j, 9s+j); z: (18+j, j).
    R x = A::sub(f[2], f[0]);
#pragma unroll
    for (int k = 1; k < 9; ++k) x = A::add(x, A::sub(f[3 * k + 2], f[3 * k]));
    R y = A::sub(f[6], f[0]);
#pragma unroll
    for (int k = 1; k < 9; ++k) {
        const int lo = 9 * (k / 3) + (k % 3);
        y = A::add(y, A::sub(f[lo + 6], f[lo]));
    }
    R z = A::sub(f[18], f[0]);
#pragma unroll
    for (int k = 1; k < 9; ++k) z = A::add(z, A::sub(f[18 + k], f[k]));
    if (E) {
        x = A::mul(x, pow2<R, -E>());
        y = A::mul(y, pow2<R, -E>());
        z = A::mul(z, pow2<R, -E>());
    }
    ux = A::mul(x, inv);
    uy = A::mul(y, inv);
    uz = A::mul(z, inv);
}

// Shared intermediate terms of the shifted equilibrium.
template <typename R>
struct EquTerms {
    R c3, h;
    R v[13];   // 3u projected on the 13 direction classes (see vsel)
    R rw[4], rm[4];
};

// Which projection and which weight class each direction uses, and whether
// it enters with + or - sign, transcribed from the 27 expressions of
// bgk::detail::calcEqu<27> (device_function.hpp:336-397).
// v index: 0..2 = 3ux,3uy,3uz; 3..12 = v0..v9 of the reference.
// weight class: 0 centre, 1 face (rhos), 2 edge (rhoe), 3 corner (rhoc).
__host__ __device__ constexpr int equ_vsel(int d)
{
    constexpr int t[27] = {9, 5, 12, 4, 2, 7, 11, 8, 10,
                           3, 1, 6, 0, 0, 0, 6, 1, 3,
                           10, 8, 11, 7, 2, 4, 12, 5, 9};
    return t[d];
}
__host__ __device__ constexpr bool equ_plus(int d)
{
    constexpr bool t[27] = {false, false, false, false, false, true, false, true, true,
                            false, false, true, false, false, true, false, true, true,
                            false, false, true, false, true, true, true, true, true};
    return t[d];
}
__host__ __device__ constexpr int equ_wcls(int d)
{
    const int k = (cx_of(d) != 0) + (cy_of(d) != 0) + (cz_of(d) != 0);
    return k;   // 0 centre, 1 face, 2 edge, 3 corner
}

// With E > 0 the weighted terms rw, rm carry the factor 2^E (exactly), so
// every equilibrium built from them is the raw value 2^E * feq.
template <typename R, int E = 0>
__device__ __forceinline__ void equ_terms(R rho, R ux, R uy, R uz, EquTerms<R>& t)
{
    using A = Rn<R>;
    const R WS = R(2) / R(27) * pow2<R, E>(), WE = R(1) / R(54) * pow2<R, E>(), WC = R(1) / R(216) * pow2<R, E>();
    const R rhom1 = A::sub(rho, R(1));
    t.c3 = A::mul(R(-3), A::add(A::add(A::mul(ux, ux), A::mul(uy, uy)), A::mul(uz, uz)));
    t.h = R(0.5);
    const R vx = A::mul(ux, R(3)), vy = A::mul(uy, R(3)), vz = A::mul(uz, R(3));
    t.v[0] = vx;
    t.v[1] = vy;
    t.v[2] = vz;
    t.v[3] = A::add(vx, vy);                    // v0
    t.v[4] = A::add(vx, vz);                    // v1
    t.v[5] = A::add(vy, vz);                    // v2
    t.v[6] = A::sub(vx, vy);                    // v3
    t.v[7] = A::sub(vx, vz);                    // v4
    t.v[8] = A::sub(vy, vz);                    // v5
    t.v[9] = A::add(A::add(vx, vy), vz);        // v6
    t.v[10] = A::sub(A::add(vx, vy), vz);       // v7
    t.v[11] = A::add(A::sub(vx, vy), vz);       // v8
    t.v[12] = A::add(A::sub(vy, vx), vz);       // v9
    t.rw[0] = E ? A::mul(rho, pow2<R, E>()) : rho;   // centre uses rho directly
    t.rw[1] = A::mul(WS, rho);
    t.rw[2] = A::mul(WE, rho);
    t.rw[3] = A::mul(WC, rho);
    t.rm[0] = E ? A::mul(rhom1, pow2<R, E>()) : rhom1;
    t.rm[1] = A::mul(WS, rhom1);
    t.rm[2] = A::mul(WE, rhom1);
    t.rm[3] = A::mul(WC, rhom1);
}

// feq_d - w_d for a non-centre direction: fma(rw, fma(1/2, fma(v, v, c3), +-v), rm).
template <typename R>
__device__ __forceinline__ R equ_dir(const EquTerms<R>& t, int d)
{
    using A = Rn<R>;
    const R v = t.v[equ_vsel(d)];
    const R sv = equ_plus(d) ? v : -v;
    const int w = equ_wcls(d);
    return A::fma(t.rw[w], A::fma(t.h, A::fma(v, v, t.c3), sv), t.rm[w]);
}

// Shifted equilibrium into f, bgk::detail::calcEqu<27> (device_function.hpp:305-398);
// raw values 2^E * feq with E > 0.
template <typename R, int E = 0>
__device__ __forceinline__ void equilibrium(R rho, R ux, R uy, R uz, R* f)
{
    using A = Rn<R>;
    EquTerms<R> t;
    equ_terms<R, E>(rho, ux, uy, uz, t);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (d == 13)
            f[d] = A::mul(R(8) / R(27), A::fma(t.rw[0], A::mul(t.h, t.c3), t.rm[0]));
        else
            f[d] = equ_dir(t, d);
    }
}

// Shifted equilibrium of direction d (centre included) from the terms.
template <typename R>
__device__ __forceinline__ R equ_any(const EquTerms<R>& t, int d)
{
    using A = Rn<R>;
    if (d == 13) return A::mul(R(8) / R(27), A::fma(t.rw[0], A::mul(t.h, t.c3), t.rm[0]));
    return equ_dir(t, d);
}

// One relaxed population invTau*feq_d + (1-invTau)*f_d, with the centre term
// associated as the reference does: (invTau*W0)*fma(rho, c3/2, rho-1).
template <typename R>
__device__ __forceinline__ R bgk_relax(const EquTerms<R>& t, R inv_tau, R om, int d, R fd)
{
    using A = Rn<R>;
    R e;
    if (d == 13)
        e = A::mul(A::mul(inv_tau, R(8) / R(27)), A::fma(t.rw[0], A::mul(t.h, t.c3), t.rm[0]));
    else
        e = A::mul(inv_tau, equ_dir(t, d));
    return A::add(e, A::mul(om, fd));
}

// BGK relaxation on shifted populations, bgk::detail::collision2<27>
// (device_function.hpp:676-754): f <- invTau*feq + (1-invTau)*f; on raw
// values 2^E * f with E > 0 (same bits after unscaling).
template <typename R, int E = 0>
__device__ __forceinline__ void collide(R inv_tau, R* f)
{
    using A = Rn<R>;
    R rho, ux, uy, uz;
    moments<R, E>(f, rho, ux, uy, uz);
    EquTerms<R> t;
    equ_terms<R, E>(rho, ux, uy, uz, t);
    const R om = A::sub(R(1), inv_tau);
#pragma unroll
    for (int d = 0; d < 27; ++d) f[d] = bgk_relax(t, inv_tau, om, d, f[d]);
}

// Boundary and collision sequence of one cell after its populations were
// loaded: EQU overwrite, full-way bounce-back swap d <-> 26-d, BGK.
// Reference src/simulator/single_dev_expt/kernel.cu:2571-2600.
// With E > 0, f holds raw values 2^E * f in and out.
template <typename R, int E = 0>
__device__ __forceinline__ void cell_update(uint8_t op, R inv_tau, const float* __restrict__ rho,
                                            const float* __restrict__ vx, const float* __restrict__ vy,
                                            const float* __restrict__ vz, int64_t i, R* f)
{
    if (op & OP_EQU) {
        equilibrium<R, E>(R(rho[i]), R(vx[i]), R(vy[i]), R(vz[i]), f);
    }
    if (op & OP_BB) {
#pragma unroll
        for (int d = 0; d < 13; ++d) {
            const R tmp = f[d];
            f[d] = f[26 - d];
            f[26 - d] = tmp;
        }
    }
    if (op & OP_COLLIDE) {
        collide<R, E>(inv_tau, f);
    }
}

// ---------------------------------------------------------------------------
// Compact BGK update for 16-bit population storage.  The FP16/BF16 formats
// store f with about 3 significant digits, so the FP32 cell arithmetic needs
// no bitwise match with the reference's operation order; this form uses
// fused multiply-adds and the pair symmetry c_{26-d} = -c_d to do the same
// update in about 200 instead of 290 instructions.  Every operation is an
// explicit round-to-nearest intrinsic in a fixed order, so the C oracle
// (orc_cell_fast_f32) reproduces it bit for bit.  f holds raw values 2^E * f
// in and out; the result equals 2^E times the E = 0 result exactly.
//   dr = f_13 + sum_{d<13} (f_d + f_{26-d}),  rho = 1 + dr,
//   j = sum_{d<13} c_d (f_d - f_{26-d}),
//   w feq_d = A_k (P + 3 c_d.u) + C_k,  P = 9/2 (c_d.u)^2 - 3/2 |u|^2,
//   A_k = w W_k 2^E rho, C_k = w W_k 2^E dr,  f_d <- (1 - w) f_d + w feq_d
// (k the weight class of d; w = 1 gives the equilibrium itself).  Keeping
// rho - 1 = dr apart, as the reference does, avoids cancelling the 1.

// c_d . u in a fixed order: x, then y, then z; the first non-zero term is
// taken as is (exact negation), the others added or subtracted.
template <int D>
__device__ __forceinline__ float cdot_fast(float ux, float uy, float uz)
{
    using A = Rn<float>;
    constexpr int cx = cx_of(D), cy = cy_of(D), cz = cz_of(D);
    float v = cx == 1 ? ux : cx == -1 ? -ux : 0.0f;
    if constexpr (cy != 0) v = cx == 0 ? (cy == 1 ? uy : -uy) : (cy == 1 ? A::add(v, uy) : A::sub(v, uy));
    if constexpr (cz != 0)
        v = (cx == 0 && cy == 0) ? (cz == 1 ? uz : -uz) : (cz == 1 ? A::add(v, uz) : A::sub(v, uz));
    return v;
}

// Weight-class constants A_k = w W_k 2^E rho and C_k = w W_k 2^E dr.
template <int E>
__device__ __forceinline__ void fast_class_terms(float w, float rho, float dr, float* Ak, float* Ck)
{
    using A = Rn<float>;
    const float W[4] = {8.0f / 27.0f, 2.0f / 27.0f, 1.0f / 54.0f, 1.0f / 216.0f};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float b = A::mul(A::mul(w, W[k]), pow2<float, E>());
        Ak[k] = A::mul(b, rho);
        Ck[k] = A::mul(b, dr);
    }
}

// f_d <- om f_d + (A_k (P +- 3 c.u) + C_k) for every direction (om = 0 and
// w = 1 give the equilibrium).
template <bool RELAX>
__device__ __forceinline__ void fast_relax(float om, float ux, float uy, float uz, const float* Ak, const float* Ck,
                                          float* f)
{
    using A = Rn<float>;
    const float uu = A::fma(ux, ux, A::fma(uy, uy, A::mul(uz, uz)));
    const float base = A::mul(-1.5f, uu);
    for_dirs([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        if constexpr (d < 13) {
            constexpr int e = 26 - d;
            constexpr int k = (cx_of(d) != 0) + (cy_of(d) != 0) + (cz_of(d) != 0);
            const float cu = cdot_fast<d>(ux, uy, uz);
            const float P = A::fma(A::mul(4.5f, cu), cu, base);
            const float ed = A::fma(Ak[k], A::fma(3.0f, cu, P), Ck[k]);
            const float ee = A::fma(Ak[k], A::fma(-3.0f, cu, P), Ck[k]);
            f[d] = RELAX ? A::fma(om, f[d], ed) : ed;
            f[e] = RELAX ? A::fma(om, f[e], ee) : ee;
        }
    });
    const float e13 = A::fma(Ak[0], base, Ck[0]);
    f[13] = RELAX ? A::fma(om, f[13], e13) : e13;
}

template <int E>
__device__ __forceinline__ void collide_fast(float w, float* f)
{
    using A = Rn<float>;
    float r = f[13];
    float jx = 0.0f, jy = 0.0f, jz = 0.0f;
    bool hx = false, hy = false, hz = false;
#pragma unroll
    for (int d = 0; d < 13; ++d) {
        const float sp = A::add(f[d], f[26 - d]);
        const float tm = A::sub(f[d], f[26 - d]);
        r = A::add(r, sp);
        if (cx_of(d) != 0) {
            jx = hx ? (cx_of(d) == 1 ? A::add(jx, tm) : A::sub(jx, tm)) : (cx_of(d) == 1 ? tm : -tm);
            hx = true;
        }
        if (cy_of(d) != 0) {
            jy = hy ? (cy_of(d) == 1 ? A::add(jy, tm) : A::sub(jy, tm)) : (cy_of(d) == 1 ? tm : -tm);
            hy = true;
        }
        if (cz_of(d) != 0) {
            jz = hz ? (cz_of(d) == 1 ? A::add(jz, tm) : A::sub(jz, tm)) : (cz_of(d) == 1 ? tm : -tm);
            hz = true;
        }
    }
    const float dr = A::mul(r, pow2<float, -E>());
    const float rho = A::add(1.0f, dr);
    const float inv = A::div(1.0f, rho);
    const float ux = A::mul(A::mul(jx, pow2<float, -E>()), inv);
    const float uy = A::mul(A::mul(jy, pow2<float, -E>()), inv);
    const float uz = A::mul(A::mul(jz, pow2<float, -E>()), inv);
    float Ak[4], Ck[4];
    fast_class_terms<E>(w, rho, dr, Ak, Ck);
    fast_relax<true>(A::sub(1.0f, w), ux, uy, uz, Ak, Ck, f);
}

template <int E>
__device__ __forceinline__ void equilibrium_fast(float rho, float ux, float uy, float uz, float* f)
{
    float Ak[4], Ck[4];
    fast_class_terms<E>(1.0f, rho, Rn<float>::sub(rho, 1.0f), Ak, Ck);
    fast_relax<false>(0.0f, ux, uy, uz, Ak, Ck, f);
}

template <int E>
__device__ __forceinline__ void cell_update_fast(uint8_t op, float inv_tau, const float* __restrict__ rho,
                                                 const float* __restrict__ vx, const float* __restrict__ vy,
                                                 const float* __restrict__ vz, int64_t i, float* f)
{
    if (op & OP_EQU) equilibrium_fast<E>(rho[i], vx[i], vy[i], vz[i], f);
    if (op & OP_BB) {
#pragma unroll
        for (int d = 0; d < 13; ++d) {
            const float tmp = f[d];
            f[d] = f[26 - d];
            f[26 - d] = tmp;
        }
    }
    if (op & OP_COLLIDE) collide_fast<E>(inv_tau, f);
}

}  // namespace culbm
