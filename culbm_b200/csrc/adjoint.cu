// Discrete adjoint of the D3Q27 BGK step with a soft-obstacle field, for the
// pressure-drop objective declared in include/culbm.h (culbm_adj_*).  No
// reference counterpart: cuLBM has no gradient code.
//
// Forward step (one thread per cell, pull with the reference's per-axis clamp):
//     f1 = EQU ? feq(rho_in, u_in) : f          (f pulled from the state)
//     f2 = BOUNCE_BACK ? B(f1) : f1              (B(g)_d = g_{26-d})
//     f3 = COLLIDE ? C(f2) + s (B(f2) - C(f2)) : f2,   C = BGK with rate w = invTau
// stored back for every STORE cell.  With s = 0 and FP32 or FP64 storage
// this is the plain step bit for bit (the soft term is skipped, not
// multiplied by zero).  With a 16-bit storage format the cell arithmetic is
// still the reference-order FP32 update, not the compact form the plain
// 16-bit step uses; loads and stores round as the plain step does.
//
// Adjoint step (reverse time, one thread per cell s):
//   * gather: lambda_d(s) = sum of nu_d(y) over the cells y whose pull of
//     direction d reads s (y = s + c_d and, at the boundary, the clamp readers)
//     - the transpose of the pull, written as a gather so no atomics are needed;
//   * reverse of the cell update with the Jacobian of C written out:
//     (J_C^T l)_e = (1-w) l_e + w [a_rho + c_e.b - u.b],
//     a_rho = L0 + 3 Lcu + 9/2 Lcu2 - 3/2 |u|^2 L0,  b = 3 L + 9 Lccu - 3 u L0,
//     with L0 = sum w_d l_d, L = sum w_d l_d c_d, Lcu = sum w_d l_d (c_d.u),
//     Lcu2 = sum w_d l_d (c_d.u)^2, Lccu = sum w_d l_d c_d (c_d.u);
//   * nu(s) = adjoint of the pulled populations, plus dJ/df of the objective;
//   * per-cell FP64 accumulators: dJ/ds += <l, B(f2) - C(f2)>,
//     dJ/dw += (1-s) <l, feq - f2>, and at EQU cells dJ/d(rho_in, u_in) from
//     d feq/d(rho, u).
// States are recomputed from checkpoints taken every K steps.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sim_internal.cuh"

namespace culbm {
namespace adj {

template <typename S, typename R>
struct Args {
    Domain dom;
    const uint8_t* ops;
    const float* rho;
    const float* vx;
    const float* vy;
    const float* vz;
    const float* soft;
    R inv_tau;
    Pops<S> src;      // state F^t
    Pops<S> dst;      // forward: F^{t+1}
    R* nu_in[27];     // adjoint: nu^{t+1}
    R* nu_out[27];    // adjoint: nu^t
    double* g_soft;
    double* g_tau;
    double* g_mac[4];
    int plane_in, plane_out;
    R obj_in, obj_out;   // dJ/df_d of one in/out plane cell at this time (0 outside the window)
    uint32_t seed;
    double* rho_plane;   // forward: rho of the two measurement planes of the pulled state, this step
                         // (null outside the objective window); [2][ny*nz]
    double* g_tau_block; // adjoint: one FP64 accumulator per warp
    const int* equ_cells; // adjoint: the EQU cells, increasing
    int n_equ;
};

// Pull of the 27 populations of cell (x, y, z) from the state a.src with the
// per-axis clamp (the same rule as the plain pull step).
// With ROWS == ROWS_INNER the cell is known to lie off the y and z faces;
// RAW loads the stored values without the format's scale (ld_stream_raw).
template <int ROWS = ROWS_OUTER, bool RAW = false, typename S, typename R>
__device__ __forceinline__ void pull_state(const Args<S, R>& a, int x, int y, int z, int i, R* f)
{
    const Domain& D = a.dom;
    constexpr bool inner = ROWS == ROWS_INNER;
    const int ndx = (x == 0) ? 0 : -1, pdx = (x == D.nx - 1) ? 0 : 1;
    const int ndy = (!inner && y == 0) ? 0 : -D.nx, pdy = (!inner && y == D.ny - 1) ? 0 : D.nx;
    const int ndz = (!inner && z == 0) ? 0 : -D.nxy, pdz = (!inner && z == D.nz - 1) ? 0 : D.nxy;
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const int ox = cx_of(d) == 1 ? ndx : cx_of(d) == -1 ? pdx : 0;
        const int oy = cy_of(d) == 1 ? ndy : cy_of(d) == -1 ? pdy : 0;
        const int oz = cz_of(d) == 1 ? ndz : cz_of(d) == -1 ? pdz : 0;
        const S* p = a.src.p[d] + (i + ox + oy + oz);
        f[d] = RAW ? ld_stream_raw<S, R>(p) : Cvt<S, R>::ld(p);
    }
}

// Boundary handling and soft collision of the forward model (in place on f).
template <typename R>
__device__ __forceinline__ void soft_update(uint8_t op, R inv_tau, R s, const float* rho, const float* vx,
                                            const float* vy, const float* vz, int i, R* f)
{
    using A = Rn<R>;
    if (op & OP_EQU) equilibrium<R>(R(rho[i]), R(vx[i]), R(vy[i]), R(vz[i]), f);
    if (op & OP_BB) {
#pragma unroll
        for (int d = 0; d < 13; ++d) {
            const R t = f[d];
            f[d] = f[26 - d];
            f[26 - d] = t;
        }
    }
    if (!(op & OP_COLLIDE)) return;
    R r, ux, uy, uz;
    moments(f, r, ux, uy, uz);
    EquTerms<R> t;
    equ_terms(r, ux, uy, uz, t);
    const R om = A::sub(R(1), inv_tau);
    const bool soft = s != R(0);
#pragma unroll
    for (int d = 0; d < 13; ++d) {
        const int e = 26 - d;
        const R fd = f[d], fe = f[e];
        const R cd = bgk_relax(t, inv_tau, om, d, fd);
        const R ce = bgk_relax(t, inv_tau, om, e, fe);
        f[d] = soft ? A::add(cd, A::mul(s, A::sub(fe, cd))) : cd;
        f[e] = soft ? A::add(ce, A::mul(s, A::sub(fd, ce))) : ce;
    }
    const R c13 = bgk_relax(t, inv_tau, om, 13, f[13]);
    f[13] = soft ? A::add(c13, A::mul(s, A::sub(f[13], c13))) : c13;
}

template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1) k_soft_step(const __grid_constant__ Args<S, R> a)
{
    const CellCoord c = cell_of_thread(a.dom);
    if (!c.valid) return;
    const uint8_t op = a.ops[c.i];
    R f[27];
    if (op & OP_LOAD) {
        pull_state(a, c.x, c.y, c.z, c.i, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    if (a.rho_plane && (c.x == a.plane_in || c.x == a.plane_out)) {
        // objective: rho of the pulled state on the measurement planes
        double r = 0.0;
        if (op & OP_COLLIDE) {
            R rr, ux, uy, uz;
            moments(f, rr, ux, uy, uz);
            r = static_cast<double>(rr);
        }
        const int q = c.y + a.dom.ny * c.z;
        if (c.x == a.plane_in) a.rho_plane[q] = r;
        if (c.x == a.plane_out) a.rho_plane[a.dom.ny * a.dom.nz + q] = r;
    }
    soft_update<R>(op, a.inv_tau, R(a.soft[c.i]), a.rho, a.vx, a.vy, a.vz, c.i, f);
    if (op & OP_STORE) {
        const uint32_t hc = cell_hash(static_cast<uint32_t>(c.i), a.seed);
#pragma unroll
        for (int d = 0; d < 27; ++d) put(a.dst.p[d] + c.i, f[d], hc, d);
    }
}

// rho of the pulled state on the two measurement planes (the last state of
// the window, which no step pulls).
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_plane_rho(const __grid_constant__ Args<S, R> a)
{
    const Domain& D = a.dom;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= D.ny * D.nz) return;
    const int y = q % D.ny, z = q / D.ny;
    for (int side = 0; side < 2; ++side) {
        const int px = side ? a.plane_out : a.plane_in;
        const int i = px + D.nx * (y + D.ny * z);
        double r = 0.0;
        if (a.ops[i] & OP_COLLIDE) {
            R f[27], rr, ux, uy, uz;
            pull_state(a, px, y, z, i, f);
            moments(f, rr, ux, uy, uz);
            r = static_cast<double>(rr);
        }
        a.rho_plane[side * D.ny * D.nz + q] = r;
    }
}

// Sums each recorded plane in a fixed order: block b sums plane b of
// planes[b][m], writes out[b].
__global__ void __launch_bounds__(1024) k_sum_planes(const double* planes, int m, double* out)
{
    const double* p = planes + static_cast<long long>(blockIdx.x) * m;
    double acc = 0.0;
    for (int q = threadIdx.x; q < m; q += blockDim.x) acc += p[q];
    __shared__ double sh[1024];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// Per-population weights of the objective at time t, for every cell.
template <typename S, typename R>
__device__ __forceinline__ R objective_term(const Args<S, R>& a, int x, uint8_t op)
{
    if (!(op & OP_COLLIDE)) return R(0);
    R g = R(0);
    if (x == a.plane_in) g += a.obj_in;
    if (x == a.plane_out) g += a.obj_out;
    return g;
}

// nu^T: the objective's dJ/df at the last state only.
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_adj_init(const __grid_constant__ Args<S, R> a)
{
    const CellCoord c = cell_of_thread(a.dom);
    if (!c.valid) return;
    const R g = objective_term(a, c.x, a.ops[c.i]);
#pragma unroll
    for (int d = 0; d < 27; ++d) a.nu_out[d][c.i] = g;
}

// (a_rho, b) of sum_d l_d d feq_d / d(rho, u) at velocity u: a_rho and
// rho * b are the rho and u components (see the file header).
template <typename R>
__device__ __forceinline__ void feq_vjp(const R* l, R ux, R uy, R uz, R& a_rho, R& bx, R& by, R& bz)
{
    R L0 = 0, Lx = 0, Ly = 0, Lz = 0, Lcu = 0, Lcu2 = 0, Lccx = 0, Lccy = 0, Lccz = 0;
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const R cx = R(cx_of(d)), cy = R(cy_of(d)), cz = R(cz_of(d));
        const R wl = weight<R>(d) * l[d];
        const R cu = cx * ux + cy * uy + cz * uz;
        L0 += wl;
        Lx += wl * cx;
        Ly += wl * cy;
        Lz += wl * cz;
        Lcu += wl * cu;
        Lcu2 += wl * cu * cu;
        Lccx += wl * cx * cu;
        Lccy += wl * cy * cu;
        Lccz += wl * cz * cu;
    }
    const R uu = ux * ux + uy * uy + uz * uz;
    a_rho = L0 + R(3) * Lcu + R(4.5) * Lcu2 - R(1.5) * uu * L0;
    bx = R(3) * Lx + R(9) * Lccx - R(3) * ux * L0;
    by = R(3) * Ly + R(9) * Lccy - R(3) * uy * L0;
    bz = R(3) * Lz + R(9) * Lccz - R(3) * uz * L0;
}

// FP64 warp sum of v added to the warp's own accumulator slots[warp] (no
// atomics and no block barrier: each warp owns its slot, so the result does
// not depend on scheduling, and a warp leaves as soon as it is done).  All
// 32 lanes must arrive.
__device__ __forceinline__ void warp_accumulate(double v, double* slots)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    if ((t & 31) == 0) slots[t >> 5] += v;
}

// Adjoint of the stored population d of cell c: the sum of nu_d over the
// cells whose pull of d reads c.  Off the y and z faces (ROWS_INNER) these
// are the streaming target c + c_d, when it lies inside, and at an x-face the
// cell (x, y + cy, z + cz) whose pull leaves the domain through that face and
// is clamped back to c.  Cells on a y or z face (ROWS_OUTER) enumerate the
// clamp readers in general.
template <int d, int ROWS, typename S, typename R>
__device__ __forceinline__ R gather_lambda(const Args<S, R>& a, const CellCoord& c)
{
    const Domain& D = a.dom;
    constexpr int cx = cx_of(d);
    if constexpr (ROWS == ROWS_INNER) {
        const R* nu = a.nu_in[d] + (c.i + nb_off(D, d));
        if constexpr (cx == 0) {
            return *nu;
        } else {
            const bool leaves = cx == 1 ? c.x == D.nx - 1 : c.x == 0;
            const bool clamped = cx == 1 ? c.x == 0 : c.x == D.nx - 1;
            R v = leaves ? R(0) : *nu;
            if (clamped) v += *(nu - cx);
            return v;
        }
    } else {
        R v = inside(D, c.x + cx, c.y + cy_of(d), c.z + cz_of(d)) ? a.nu_in[d][c.i + nb_off(D, d)] : R(0);
        for_each_clamp_reader<d>(D, c.x, c.y, c.z,
                                 [&](int yx, int yy, int yz) { v += a.nu_in[d][yx + D.nx * (yy + D.ny * yz)]; });
        return v;
    }
}

// <l, f1> and <l, B(f1)> accumulated while f1 is pulled (l gathered first),
// so that f1 is never held: with bounce-back f2 = B(f1) they are <l, B(f2)>
// and <l, f2>.
template <typename R>
struct PullDots {
    R a = R(0), b = R(0);
    template <int d>
    __device__ __forceinline__ void add(const R* l, R v)
    {
        a += l[d] * v;
        b += l[26 - d] * v;
    }
};

// r = sum f1 and j = sum c f1 accumulated while pulling, in direction order.
template <typename R>
struct MomentAcc {
    R r = R(0), x = R(0), y = R(0), z = R(0);
    template <int d>
    __device__ __forceinline__ void add(R v)
    {
        r += v;
        if constexpr (cx_of(d) == 1) x += v;
        if constexpr (cx_of(d) == -1) x -= v;
        if constexpr (cy_of(d) == 1) y += v;
        if constexpr (cy_of(d) == -1) y -= v;
        if constexpr (cz_of(d) == 1) z += v;
        if constexpr (cz_of(d) == -1) z -= v;
    }
    // rho and u of f2 = B(f1) if bb else f1 (bounce-back keeps rho and
    // negates j), f = fscale * the staged values; plain arithmetic (the
    // linearisation point of the adjoint).
    __device__ __forceinline__ void finish(R fscale, bool bb, R& rho, R& ux, R& uy, R& uz) const
    {
        rho = R(1) + fscale * r;
        R inv;
        if constexpr (sizeof(R) == 4)
            inv = __frcp_rn(rho);
        else
            inv = R(1) / rho;
        inv *= bb ? -fscale : fscale;
        ux = x * inv;
        uy = y * inv;
        uz = z * inv;
    }
};

template <typename R>
__device__ __forceinline__ void swap_pairs_if(bool c, R* v)
{
#pragma unroll
    for (int d = 0; d < 13; ++d) {
        const R p = v[d], q = v[26 - d];
        v[d] = c ? q : p;
        v[26 - d] = c ? p : q;
    }
}

// The ten weighted sums sum_d w_d c_d^k l_d (k = 0, 1, 2) of l by per-axis
// factorisation: w_d = W(cx) W(cy) W(cz) with W(0) = 4/6 and W(+-1) = 1/6,
// so three passes of 1D three-point moments (x, then y, then z) give them,
// each times 216.  Direction d = (cx+1) + 3 (cy+1) + 9 (cz+1).
template <typename R>
struct LSums {
    R m0, mx, my, mz, mxx, myy, mzz, mxy, mxz, myz;
};

template <typename R>
__device__ __forceinline__ LSums<R> weighted_sums(const R* l)
{
    R x0[9], x1[9], x2[9];   // per (cy, cz) line: 6 x {W-sum, W-sum cx, W-sum cx^2}
#pragma unroll
    for (int j = 0; j < 9; ++j) {
        const R lo = l[3 * j], mid = l[3 * j + 1], hi = l[3 * j + 2];
        x2[j] = lo + hi;
        x0[j] = R(4) * mid + x2[j];
        x1[j] = hi - lo;
    }
    R y00[3], y10[3], y20[3], y01[3], y11[3], y02[3];   // per cz
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int j = 3 * k;
        y02[k] = x0[j] + x0[j + 2];
        y00[k] = R(4) * x0[j + 1] + y02[k];
        y01[k] = x0[j + 2] - x0[j];
        y10[k] = R(4) * x1[j + 1] + (x1[j] + x1[j + 2]);
        y11[k] = x1[j + 2] - x1[j];
        y20[k] = R(4) * x2[j + 1] + (x2[j] + x2[j + 2]);
    }
    LSums<R> m;
    m.mzz = y00[0] + y00[2];
    m.m0 = R(4) * y00[1] + m.mzz;
    m.mz = y00[2] - y00[0];
    m.mx = R(4) * y10[1] + (y10[0] + y10[2]);
    m.mxz = y10[2] - y10[0];
    m.my = R(4) * y01[1] + (y01[0] + y01[2]);
    m.myz = y01[2] - y01[0];
    m.mxx = R(4) * y20[1] + (y20[0] + y20[2]);
    m.myy = R(4) * y02[1] + (y02[0] + y02[2]);
    m.mxy = R(4) * y11[1] + (y11[0] + y11[2]);
    return m;
}

// Reverse of bounce-back and soft collision for one cell, linearised at
// f2 = B(f1) if the cell bounces back, else f1, with f = fscale * the pulled
// values (possibly raw 16-bit values), (rho, u) its moments and
// dots = (<l, f1>, <l, B(f1)>) of the pulled values; plain arithmetic.  l
// enters as the adjoint of the stored populations and leaves as the adjoint
// of f1; gs and gw are the cell's dJ/ds and dJ/dw (0 unless it collides and
// stores).  With P = <l, f2>, Q = <l, B(f2)>, E = <l, feq(f2)>:
//     dJ/ds = <l, B(f2) - C(f2)> = (Q - P) - w (E - P),
//     dJ/dw = (1 - s) <l, feq - f2> = (1 - s) (E - P),
// and E = (rho - 1) a_rho + 3 Lcu + 9/2 Lcu2 - 3/2 |u|^2 L0 comes from the
// same weighted sums as J_C^T, so no per-direction equilibrium is formed:
// with M = sum w c c^T l, Lcu = u.L, Lccu = M u and Lcu2 = u.M u.
template <typename R>
__device__ __forceinline__ void reverse_cell(uint8_t op, R w, R s, R fscale, const PullDots<R>& dots, R rho, R ux,
                                             R uy, R uz, R* l, R& gs, R& gw)
{
    const bool bb = (op & OP_BB) != 0, col = (op & OP_COLLIDE) && (op & OP_STORE);
    const R uu = ux * ux + uy * uy + uz * uz;
    const R P = fscale * (bb ? dots.b : dots.a);
    const R QmP = fscale * (bb ? dots.a - dots.b : dots.b - dots.a);
    const LSums<R> m = weighted_sums(l);
    constexpr R k216 = R(1) / R(216);
    const R L0 = k216 * m.m0, Lx = k216 * m.mx, Ly = k216 * m.my, Lz = k216 * m.mz;
    const R Mux = k216 * (m.mxx * ux + m.mxy * uy + m.mxz * uz);
    const R Muy = k216 * (m.mxy * ux + m.myy * uy + m.myz * uz);
    const R Muz = k216 * (m.mxz * ux + m.myz * uy + m.mzz * uz);
    const R Lcu = ux * Lx + uy * Ly + uz * Lz;
    const R Lcu2 = ux * Mux + uy * Muy + uz * Muz;
    const R a1 = R(3) * Lcu + R(4.5) * Lcu2 - R(1.5) * uu * L0;
    const R ar = L0 + a1;
    const R emp = ((rho - R(1)) * ar + a1) - P;
    gs = col ? QmP - w * emp : R(0);
    gw = col ? (R(1) - s) * emp : R(0);
    if (!col) {
        if (bb) swap_pairs_if(true, l);
        return;
    }
    // l <- (1-s) J_C^T l + s B(l),  (J_C^T l)_e = (1-w) l_e + w (a_rho + c_e.b - u.b):
    // l_e <- (1-s)(1-w) l_e + s l_{26-e} + t_e,  t_e = (1-s) w (a_rho - u.b + c_e.b)
    const R bx = w * (R(3) * Lx + R(9) * Mux - R(3) * ux * L0);
    const R by = w * (R(3) * Ly + R(9) * Muy - R(3) * uy * L0);
    const R bz = w * (R(3) * Lz + R(9) * Muz - R(3) * uz * L0);
    const R sc = R(1) - s;
    const R q = sc * (w * ar - (ux * bx + uy * by + uz * bz));
    const R tx = sc * bx, ty = sc * by, tz = sc * bz;
    const R keep = sc * (R(1) - w);
    R t[27];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R qz = k == 1 ? q : (k == 0 ? q - tz : q + tz);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const R qy = j == 1 ? qz : (j == 0 ? qz - ty : qz + ty);
            const int d = 3 * j + 9 * k;
            t[d] = qy - tx;
            t[d + 1] = qy;
            t[d + 2] = qy + tx;
        }
    }
#pragma unroll
    for (int d = 0; d < 13; ++d) {
        const int e = 26 - d;
        const R ld = l[d], le = l[e];
        l[d] = keep * ld + (s * le + t[d]);
        l[e] = keep * le + (s * ld + t[e]);
    }
    l[13] = keep * l[13] + (s * l[13] + t[13]);
    if (bb) swap_pairs_if(true, l);
}

// Reverse of one cell update at step t for a cell without EQU (EQU cells
// only get nu = dJ/df here; adj_equ_cell does the rest of their work).  The
// pull and the gather stay inside the domain for every cell, so all loads
// are issued without looking at the op byte.  l is gathered first and the
// pulled values are folded into the moments and dots as they arrive.  l is
// left unmasked for cells that do not store: their gs and gw are zero and
// their nu is dJ/df alone.
template <int ROWS, typename S, typename R>
__device__ __forceinline__ void adj_cell(const Args<S, R>& a, const CellCoord c, double& gtau_local)
{
    const Domain& D = a.dom;
    const uint8_t op = a.ops[c.i];
    const R s = R(a.soft[c.i]);
    const bool load = (op & OP_LOAD) != 0, store = (op & OP_STORE) != 0, equ = (op & OP_EQU) != 0;
    MomentAcc<R> m;
    PullDots<R> dots;
    R l[27];
    // warps of inner rows without an x-face lane (a warp-uniform choice) pull
    // and gather without any clamp handling
    const int xw = c.x - (threadIdx.x & 31);
    if (ROWS == ROWS_INNER && xw != 0 && xw + 31 < D.nx - 1) {
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            l[d] = a.nu_in[d][c.i + nb_off(D, d)];
        });
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            const R v = ld_stream_raw<S, R>(a.src.p[d] + (c.i - nb_off(D, d)));
            m.template add<d>(v);
            dots.template add<d>(l, v);
        });
    } else {
        constexpr bool inner = ROWS == ROWS_INNER;
        const int ndx = (c.x == 0) ? 0 : -1, pdx = (c.x == D.nx - 1) ? 0 : 1;
        const int ndy = (!inner && c.y == 0) ? 0 : -D.nx, pdy = (!inner && c.y == D.ny - 1) ? 0 : D.nx;
        const int ndz = (!inner && c.z == 0) ? 0 : -D.nxy, pdz = (!inner && c.z == D.nz - 1) ? 0 : D.nxy;
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            l[d] = gather_lambda<d, ROWS>(a, c);
        });
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            const int ox = cx_of(d) == 1 ? ndx : cx_of(d) == -1 ? pdx : 0;
            const int oy = cy_of(d) == 1 ? ndy : cy_of(d) == -1 ? pdy : 0;
            const int oz = cz_of(d) == 1 ? ndz : cz_of(d) == -1 ? pdz : 0;
            const R v = ld_stream_raw<S, R>(a.src.p[d] + (c.i + ox + oy + oz));
            m.template add<d>(v);
            dots.template add<d>(l, v);
        });
    }
    // a cell that does not load has f1 = 0: its sums restart from zero
    if (!load) {
        m = MomentAcc<R>{};
        dots = PullDots<R>{};
    }
    constexpr R fscale = R(RawScale<S>::value);
    R rho, ux, uy, uz, gs, gw;
    m.finish(fscale, (op & OP_BB) != 0, rho, ux, uy, uz);
    reverse_cell(op, a.inv_tau, s, fscale, dots, rho, ux, uy, uz, l, gs, gw);
    if (!equ && (op & OP_COLLIDE) && store) {
        a.g_soft[c.i] += static_cast<double>(gs);
        gtau_local = static_cast<double>(gw);
    }
    const bool pulls = load && store && !equ;
    const R g = objective_term(a, c.x, op);
    if (!pulls)
#pragma unroll
        for (int d = 0; d < 27; ++d) l[d] = R(0);
    if (g != R(0))
#pragma unroll
        for (int d = 0; d < 27; ++d) l[d] += g;
#pragma unroll
    for (int d = 0; d < 27; ++d) a.nu_out[d][c.i] = l[d];
}

// The EQU cell i of one adjoint step: f1 = feq(rho_in, u_in), the gather
// with the general clamp rule, the reverse of bounce-back and collision, and
// dJ/d(rho_in, u_in) from d feq / d(rho, u).  Its nu (no pull, so dJ/df
// only) is written by adj_cell.
template <typename S, typename R>
__device__ __forceinline__ void adj_equ_cell(const Args<S, R>& a, int i, double& gtau_local)
{
    const Domain& D = a.dom;
    CellCoord c;
    c.i = i;
    c.x = i % D.nx;
    c.y = (i / D.nx) % D.ny;
    c.z = i / D.nxy;
    c.valid = true;
    const uint8_t op = a.ops[i];
    const R r_in = R(a.rho[i]), vx = R(a.vx[i]), vy = R(a.vy[i]), vz = R(a.vz[i]);
    R l[27];
    const bool store = (op & OP_STORE) != 0;
    for_dirs([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        l[d] = store ? gather_lambda<d, ROWS_OUTER>(a, c) : R(0);
    });
    MomentAcc<R> m;
    PullDots<R> dots;
    {
        R f[27];
        equilibrium<R>(r_in, vx, vy, vz, f);
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            m.template add<d>(f[d]);
            dots.template add<d>(l, f[d]);
        });
    }
    R rho, ux, uy, uz, gs, gw;
    m.finish(R(1), (op & OP_BB) != 0, rho, ux, uy, uz);
    reverse_cell(op, a.inv_tau, R(a.soft[i]), R(1), dots, rho, ux, uy, uz, l, gs, gw);
    if ((op & OP_COLLIDE) && store) {
        a.g_soft[i] += static_cast<double>(gs);
        gtau_local = static_cast<double>(gw);
    }
    R ar, bx, by, bz;
    feq_vjp(l, vx, vy, vz, ar, bx, by, bz);
    a.g_mac[0][i] += static_cast<double>(ar);
    a.g_mac[1][i] += static_cast<double>(r_in * bx);
    a.g_mac[2][i] += static_cast<double>(r_in * by);
    a.g_mac[3][i] += static_cast<double>(r_in * bz);
}

// Grid of one adjoint-step launch: equ_z grid-z slices of blocks that take
// the EQU cells, 256 per block (the longest per-thread work, scheduled
// first), then the slices of split_grid (outer rows, then inner rows).
struct AdjLayout {
    int equ_z;
};

inline AdjLayout adj_layout(const Domain& D, int n_equ)
{
    const long long per_slice = 1ll * ((D.nx + 31) / 32) * ((D.ny + 7) / 8);
    const long long equ_blocks = (n_equ + 255) / 256;
    return {static_cast<int>((equ_blocks + per_slice - 1) / per_slice)};
}

inline dim3 adj_grid(const Domain& D, int n_equ)
{
    const dim3 g = split_grid(D);
    return dim3(g.x, g.y, g.z + adj_layout(D, n_equ).equ_z);
}

// One adjoint step over all cells (block-uniform roles); each warp adds its
// invTau gradient into its own slot of g_tau_block (8 per block).
template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 1)
    k_adj_step(const __grid_constant__ Args<S, R> a, AdjLayout L)
{
    double gtau_local = 0.0;
    if (static_cast<int>(blockIdx.z) < L.equ_z) {
        const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        const int k = blk * 256 + threadIdx.x + 32 * threadIdx.y;
        if (k < a.n_equ) adj_equ_cell(a, a.equ_cells[k], gtau_local);
    } else {
        CellCoord c;
        const int kind = split_cell(a.dom, L.equ_z, c);
        if (kind == ROWS_OUTER)
            adj_cell<ROWS_OUTER>(a, c, gtau_local);
        else if (kind == ROWS_INNER)
            adj_cell<ROWS_INNER>(a, c, gtau_local);
    }
    warp_accumulate(gtau_local, a.g_tau_block + 8ll * (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)));
}

template <typename S>
__global__ void k_fill_rest(S* base, long long count)
{
    using R = typename ArithOf<S>::type;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < count;
         j += (long long)gridDim.x * blockDim.x)
        Cvt<S, R>::st(base + j, R(0));
}

// An FP32 state narrowed to the 16-bit format S, population d of cell i
// rounded as a step seeded by `seed` stores it (grid y = direction).
template <typename S>
__global__ void __launch_bounds__(256) k_narrow_state(const float* src, S* dst, long long n, uint32_t seed)
{
    const int d = blockIdx.y;
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += 256ll * gridDim.x)
        put(dst + d * n + i, src[d * n + i], cell_hash(static_cast<uint32_t>(i), seed), d);
}

}  // namespace adj
}  // namespace culbm

using namespace culbm;

struct culbm_adj {
    culbm_adj_config cfg{};
    Domain dom{};
    long long n = 0;
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    size_t esize = 4, rsize = 4;
    uint8_t* d_ops = nullptr;
    uint32_t* d_flag = nullptr;
    float* d_mac[4] = {};
    float* d_soft = nullptr;
    double inv_tau = 0.5;
    int K = 0, K2 = 0;          // checkpoint strides: outer, inner (0: one level)
    int nckpt = 0, ninner = 0, nseg = 0;
    void* d_ckpt = nullptr;     // nckpt states: F^t for t = 0, K, 2K, ...
    void* d_inner = nullptr;    // ninner states inside one outer segment (two levels only)
    void* d_seg = nullptr;      // nseg states (at least 2)
    bool mixed = false;         // FP32 forward pass, 16-bit checkpoints (checkpoint_storage)
    int state_storage = 0;      // storage of the checkpoint, inner and segment states
    void* d_fwd[2] = {nullptr, nullptr};   // FP32 ping-pong states of the mixed forward pass
    void* d_nu = nullptr;       // 2 x 27 N of the arithmetic type
    double* d_gsoft = nullptr;
    double* d_gtau = nullptr;
    double* d_gmac = nullptr;   // 4 N
    double* d_psum = nullptr;   // 2 per time step of the window
    double* d_rho_plane = nullptr;  // window x 2 planes x ny*nz
    long long n_tau_blocks = 0;     // warps of one adjoint-step launch (one FP64 slot each)
    long long tau_capacity = 0;
    int* d_equ = nullptr;           // EQU cells, increasing
    int n_equ = 0, equ_capacity = 0;
    int n_in = 0, n_out = 0;
    uint64_t device_bytes = 0;
    float t_fwd = 0, t_rec = 0, t_adj = 0;
    std::vector<uint32_t> h_flag;
};

namespace {

culbm_status adj_alloc(culbm_adj* a, void** p, size_t bytes, const char* what)
{
    cudaError_t e = injection_gate();
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? CULBM_ERR_OUT_OF_MEMORY : CULBM_ERR_CUDA,
                    std::string("device allocation for ") + what + " failed: " + cudaGetErrorString(e));
    }
    a->device_bytes += bytes;
    return CULBM_OK;
}

void adj_release(culbm_adj* a)
{
    if (!a) return;
    cudaSetDevice(a->dev);
    if (a->stream) cudaStreamSynchronize(a->stream);
    cudaFree(a->d_ops);
    cudaFree(a->d_flag);
    for (auto& p : a->d_mac) cudaFree(p);
    cudaFree(a->d_soft);
    cudaFree(a->d_ckpt);
    cudaFree(a->d_inner);
    cudaFree(a->d_seg);
    cudaFree(a->d_fwd[0]);
    cudaFree(a->d_fwd[1]);
    cudaFree(a->d_nu);
    cudaFree(a->d_gsoft);
    cudaFree(a->d_gtau);
    cudaFree(a->d_equ);
    cudaFree(a->d_gmac);
    cudaFree(a->d_psum);
    cudaFree(a->d_rho_plane);
    for (auto& e : a->ev)
        if (e) cudaEventDestroy(e);
    if (a->stream) cudaStreamDestroy(a->stream);
    delete a;
}

template <class F>
culbm_status adj_with_storage(const culbm_adj* a, F&& f)
{
    switch (a->state_storage) {
        case CULBM_STORAGE_F32: return f(Tag<float>{});
        case CULBM_STORAGE_F16: return f(Tag<__half>{});
        case CULBM_STORAGE_F16_SR: return f(Tag<Half16SR>{});
        case CULBM_STORAGE_F64: return f(Tag<double>{});
        default: return fail(CULBM_ERR_UNSUPPORTED, "adjoint storage must be F32, F16, F16_SR or F64");
    }
}

enum StateSet { CKPT, INNER, SEG };

template <typename S>
S* state_ptr(culbm_adj* a, StateSet set, int slot)
{
    S* base = static_cast<S*>(set == CKPT ? a->d_ckpt : set == INNER ? a->d_inner : a->d_seg);
    return base + static_cast<long long>(slot) * 27 * a->n;
}

template <typename S>
adj::Args<S, typename ArithOf<S>::type> base_args(culbm_adj* a)
{
    using R = typename ArithOf<S>::type;
    adj::Args<S, R> g{};
    g.dom = a->dom;
    g.ops = a->d_ops;
    g.rho = a->d_mac[0];
    g.vx = a->d_mac[1];
    g.vy = a->d_mac[2];
    g.vz = a->d_mac[3];
    g.soft = a->d_soft;
    g.inv_tau = static_cast<R>(a->inv_tau);
    g.g_soft = a->d_gsoft;
    g.g_tau = a->d_gtau;
    for (int k = 0; k < 4; ++k) g.g_mac[k] = a->d_gmac + k * a->n;
    g.plane_in = a->cfg.plane_x[0];
    g.plane_out = a->cfg.plane_x[1];
    return g;
}

template <typename S, typename R>
void set_pops(Pops<S>& p, S* base, long long n)
{
    p.set(base, n);
}

// Forward steps t in [t_begin, t_end) from state `src`; states written to the
// slots chosen by `slot_of(t+1)`; objective partial sums recorded when asked.
template <typename S, class SlotOf>
culbm_status forward_run(culbm_adj* a, int t_begin, int t_end, S* src, SlotOf slot_of, bool record)
{
    using R = typename ArithOf<S>::type;
    auto g = base_args<S>(a);
    const dim3 grid = cell_grid(a->dom), block = cell_block();
    const int t0 = a->cfg.window[0], t1 = a->cfg.window[1];
    const long long plane = 2ll * a->dom.ny * a->dom.nz;
    S* cur = src;
    for (int t = t_begin; t < t_end; ++t) {
        S* dst = slot_of(t + 1);
        set_pops<S, R>(g.src, cur, a->n);
        set_pops<S, R>(g.dst, dst, a->n);
        g.seed = step_seed(static_cast<uint32_t>(t));
        g.rho_plane = (record && t >= t0 && t <= t1) ? a->d_rho_plane + (t - t0) * plane : nullptr;
        adj::k_soft_step<S, R><<<grid, block, 0, a->stream>>>(g);
        CULBM_CUDA(cudaGetLastError());
        cur = dst;
    }
    if (record && t_end >= t0 && t_end <= t1) {
        set_pops<S, R>(g.src, cur, a->n);
        g.rho_plane = a->d_rho_plane + (t_end - t0) * plane;
        adj::k_plane_rho<S, R><<<(a->dom.ny * a->dom.nz + 255) / 256, 256, 0, a->stream>>>(g);
        CULBM_CUDA(cudaGetLastError());
    }
    return CULBM_OK;
}

template <typename S>
culbm_status fill_rest(culbm_adj* a, S* state)
{
    adj::k_fill_rest<S><<<1184, 256, 0, a->stream>>>(state, 27ll * a->n);
    CULBM_CUDA(cudaGetLastError());
    return CULBM_OK;
}

culbm_status objective(culbm_adj* a, double* J)
{
    const int t0 = a->cfg.window[0], t1 = a->cfg.window[1];
    const int nt = t1 - t0 + 1;
    adj::k_sum_planes<<<2 * nt, 1024, 0, a->stream>>>(a->d_rho_plane, a->dom.ny * a->dom.nz, a->d_psum);
    CULBM_CUDA(cudaGetLastError());
    std::vector<double> ps(2 * nt);
    CULBM_CUDA(cudaMemcpyAsync(ps.data(), a->d_psum, ps.size() * sizeof(double), cudaMemcpyDeviceToHost, a->stream));
    CULBM_CUDA(cudaStreamSynchronize(a->stream));
    double acc = 0.0;
    for (int k = 0; k < nt; ++k) acc += ps[2 * k] / (3.0 * a->n_in) - ps[2 * k + 1] / (3.0 * a->n_out);
    *J = acc / nt;
    return CULBM_OK;
}

float elapsed(culbm_adj* a)
{
    float ms = 0;
    cudaEventRecord(a->ev[1], a->stream);
    cudaEventSynchronize(a->ev[1]);
    cudaEventElapsedTime(&ms, a->ev[0], a->ev[1]);
    cudaEventRecord(a->ev[0], a->stream);
    return ms;
}

template <typename S>
culbm_status run_forward(culbm_adj* a, bool checkpoints)
{
    const int T = a->cfg.window[1], K = a->K;
    S* s0 = state_ptr<S>(a, CKPT, 0);
    CULBM_TRY(fill_rest<S>(a, s0));
    // With one checkpoint level, the states of the last segment go straight to
    // the segment slots where its reverse sweep reads them (no recompute).
    const int tb_last = ((std::max(T, 1) - 1) / K) * K;
    const bool keep_last = checkpoints && a->K2 == 0;
    auto slot_of = [&](int t) -> S* {
        if (checkpoints && t % K == 0) return state_ptr<S>(a, CKPT, t / K);
        if (keep_last && t > tb_last) return state_ptr<S>(a, SEG, t - tb_last - 1);
        return state_ptr<S>(a, SEG, t & 1);
    };
    return forward_run<S>(a, 0, T, s0, slot_of, true);
}

// The forward pass of the mixed mode: FP32 states (ping-pong), the objective
// recorded from them, and every K-th state narrowed into its 16-bit
// checkpoint slot (format S).
template <typename S>
culbm_status run_forward_mixed(culbm_adj* a, bool checkpoints)
{
    if constexpr (!Is16<S>::value) {
        return fail(CULBM_ERR_UNSUPPORTED, "16-bit checkpoint storage only");
    } else {
    const int T = a->cfg.window[1], K = a->K;
    float* b[2] = {static_cast<float*>(a->d_fwd[0]), static_cast<float*>(a->d_fwd[1])};
    CULBM_TRY(fill_rest<float>(a, b[0]));
    const dim3 ng(592, 27);
    auto narrow = [&](int t) -> culbm_status {
        adj::k_narrow_state<S><<<ng, 256, 0, a->stream>>>(b[t & 1], state_ptr<S>(a, CKPT, t / K), a->n,
                                                         step_seed(static_cast<uint32_t>(t > 0 ? t - 1 : 0)));
        CULBM_CUDA(cudaGetLastError());
        return CULBM_OK;
    };
    if (checkpoints) CULBM_TRY(narrow(0));
    for (int tb = 0; tb < T; tb += K) {
        const int te = std::min(T, tb + K);
        CULBM_TRY(forward_run<float>(a, tb, te, b[tb & 1], [&](int t) -> float* { return b[t & 1]; }, true));
        if (checkpoints && te % K == 0) CULBM_TRY(narrow(te));
    }
    return CULBM_OK;
    }
}

// Reverse sweep over the steps t in [tb, te) (te - tb <= nseg + 1) starting
// from the state F^tb: recompute F^{tb+1} .. F^{te-1} into the segment
// slots (unless they are already there), then run the adjoint steps
// te-1 .. tb.
template <typename S>
culbm_status adjoint_segment(culbm_adj* a, int tb, int te, S* start, adj::Args<S, typename ArithOf<S>::type>& g,
                             typename ArithOf<S>::type* const nu[2], int& cur, float& rec, float& adjms,
                             bool states_present = false)
{
    using R = typename ArithOf<S>::type;
    const int t0 = a->cfg.window[0], t1 = a->cfg.window[1];
    const double nT = t1 - t0 + 1;
    const R obj_in = static_cast<R>(1.0 / (3.0 * a->n_in * nT));
    const R obj_out = static_cast<R>(-1.0 / (3.0 * a->n_out * nT));
    const dim3 block = cell_block();
    const adj::AdjLayout L = adj::adj_layout(a->dom, a->n_equ);
    const dim3 gr = adj::adj_grid(a->dom, a->n_equ);
    auto slot_of = [&](int t) -> S* { return state_ptr<S>(a, SEG, t - tb - 1); };
    if (!states_present) CULBM_TRY(forward_run<S>(a, tb, te - 1, start, slot_of, false));
    rec += elapsed(a);
    for (int t = te - 1; t >= tb; --t) {
        S* st = (t == tb) ? start : state_ptr<S>(a, SEG, t - tb - 1);
        set_pops<S, R>(g.src, st, a->n);
        for (int d = 0; d < 27; ++d) {
            g.nu_in[d] = nu[cur] + d * a->n;
            g.nu_out[d] = nu[1 - cur] + d * a->n;
        }
        const bool in_win = t >= t0 && t <= t1;
        g.obj_in = in_win ? obj_in : R(0);
        g.obj_out = in_win ? obj_out : R(0);
        adj::k_adj_step<S, R><<<gr, block, 0, a->stream>>>(g, L);
        CULBM_CUDA(cudaGetLastError());
        cur = 1 - cur;
    }
    adjms += elapsed(a);
    return CULBM_OK;
}

template <typename S>
culbm_status run_gradient(culbm_adj* a)
{
    using R = typename ArithOf<S>::type;
    const int T = a->cfg.window[1], K = a->K, K2 = a->K2;
    const int t0 = a->cfg.window[0], t1 = a->cfg.window[1];
    const double nT = t1 - t0 + 1;
    const dim3 grid = cell_grid(a->dom), block = cell_block();

    CULBM_CUDA(cudaEventRecord(a->ev[0], a->stream));
    if (a->mixed) {
        CULBM_TRY(run_forward_mixed<S>(a, true));
    } else {
        CULBM_TRY(run_forward<S>(a, true));
    }
    a->t_fwd = elapsed(a);

    CULBM_CUDA(cudaMemsetAsync(a->d_gsoft, 0, a->n * sizeof(double), a->stream));
    CULBM_CUDA(cudaMemsetAsync(a->d_gtau, 0, a->n_tau_blocks * sizeof(double), a->stream));
    CULBM_CUDA(cudaMemsetAsync(a->d_gmac, 0, 4 * a->n * sizeof(double), a->stream));
    R* const nu[2] = {static_cast<R*>(a->d_nu), static_cast<R*>(a->d_nu) + 27 * a->n};
    auto g = base_args<S>(a);
    g.g_tau_block = a->d_gtau;
    g.equ_cells = a->d_equ;
    g.n_equ = a->n_equ;
    int cur = 0;
    {
        for (int d = 0; d < 27; ++d) g.nu_out[d] = nu[cur] + d * a->n;
        g.obj_in = (T >= t0 && T <= t1) ? static_cast<R>(1.0 / (3.0 * a->n_in * nT)) : R(0);
        g.obj_out = (T >= t0 && T <= t1) ? static_cast<R>(-1.0 / (3.0 * a->n_out * nT)) : R(0);
        adj::k_adj_init<S, R><<<grid, block, 0, a->stream>>>(g);
        CULBM_CUDA(cudaGetLastError());
    }
    float rec = 0, adjms = 0;
    CULBM_CUDA(cudaEventRecord(a->ev[0], a->stream));
    for (int k = (T - 1) / K; k >= 0; --k) {
        const int tb = k * K, te = std::min(T, (k + 1) * K);
        S* ck = state_ptr<S>(a, CKPT, k);
        if (K2 == 0) {
            // the forward pass left the last segment's states in place
            // (not in the mixed mode, whose forward states are FP32)
            const bool last = !a->mixed && k == (T - 1) / K;
            CULBM_TRY(adjoint_segment<S>(a, tb, te, ck, g, nu, cur, rec, adjms, last));
            continue;
        }
        // two levels: one pass over the outer segment stores F^{tb + j K2},
        // then each inner segment is swept in reverse
        const int nin = (te - tb - 1) / K2;
        if (nin > 0) {
            auto slot_of = [&](int t) -> S* {
                const int r = t - tb;
                return r % K2 == 0 ? state_ptr<S>(a, INNER, r / K2 - 1) : state_ptr<S>(a, SEG, t & 1);
            };
            CULBM_TRY(forward_run<S>(a, tb, tb + nin * K2, ck, slot_of, false));
            rec += elapsed(a);
        }
        for (int j = nin; j >= 0; --j) {
            const int sb = tb + j * K2, se = std::min(te, sb + K2);
            S* start = j ? state_ptr<S>(a, INNER, j - 1) : ck;
            CULBM_TRY(adjoint_segment<S>(a, sb, se, start, g, nu, cur, rec, adjms));
        }
    }
    a->t_rec = rec;
    a->t_adj = adjms;
    return CULBM_OK;
}

// Checkpoint plan: outer stride K, inner stride K2 (0: one level) and the
// number of full states each needs.
struct CkptPlan {
    int K = 1, K2 = 0, nckpt = 0, ninner = 0, nseg = 0;
    long long states() const { return 1ll * nckpt + ninner + nseg; }
};

CkptPlan make_plan(int T, int K, int K2)
{
    CkptPlan p;
    p.K = K;
    p.K2 = K2;
    p.nckpt = (T + K - 1) / K + 1;
    p.ninner = K2 ? (K - 1) / K2 : 0;
    p.nseg = std::max((K2 ? K2 : K) - 1, 2);
    return p;
}

// Smallest plan (in states) of one level, else of two levels, within
// max_states; one level recomputes every step once, two levels twice.
bool choose_plan(int T, long long max_states, CkptPlan& out)
{
    T = std::max(T, 1);
    CkptPlan best;
    bool have = false;
    for (int K = 1; K <= T; ++K) {
        const CkptPlan p = make_plan(T, K, 0);
        if (!have || p.states() < best.states()) best = p, have = true;
    }
    if (best.states() <= max_states) {
        out = best;
        return true;
    }
    have = false;
    for (int K = 3; K <= T; ++K) {
        const int s = std::max(1, static_cast<int>(std::lround(std::sqrt(static_cast<double>(K)))));
        for (int K2 = std::max(1, s / 2); K2 <= std::min(K - 1, 2 * s + 1); ++K2) {
            const CkptPlan p = make_plan(T, K, K2);
            if (!have || p.states() < best.states()) best = p, have = true;
        }
    }
    out = best;
    return have && best.states() <= max_states;
}

}  // namespace

extern "C" {

culbm_status culbm_adj_config_init(culbm_adj_config* cfg)
{
    if (!cfg) return fail(CULBM_ERR_INVALID_ARGUMENT, "cfg is NULL");
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->domain_dim[0] = 128;
    cfg->domain_dim[1] = 64;
    cfg->domain_dim[2] = 64;
    cfg->inv_tau = 0.5f;
    cfg->window[0] = 300;
    cfg->window[1] = 500;
    cfg->plane_x[0] = 1;
    cfg->plane_x[1] = -1;   // nx - 2
    cfg->checkpoint_every = 50;
    cfg->precision = 0;
    cfg->storage = CULBM_STORAGE_F32;
    return CULBM_OK;
}

culbm_status culbm_adj_create(const culbm_adj_config* cfg, culbm_adj** out)
{
    if (!cfg || !out) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    const culbm_adj_config& c = *cfg;
    for (int k = 0; k < 3; ++k)
        if (c.domain_dim[k] < 1) return fail(CULBM_ERR_INVALID_ARGUMENT, "domain_dim must be positive");
    const unsigned long long n = 1ull * c.domain_dim[0] * c.domain_dim[1] * c.domain_dim[2];
    if (n >= (1ull << 31) || c.domain_dim[2] > 65535) return fail(CULBM_ERR_INVALID_ARGUMENT, "domain too large");
    if (c.window[0] < 0 || c.window[1] < c.window[0]) return fail(CULBM_ERR_INVALID_ARGUMENT, "bad objective window");
    if (!(c.inv_tau > 0.0f && c.inv_tau < 2.0f)) return fail(CULBM_ERR_INVALID_ARGUMENT, "invTau must lie in (0, 2)");
    const bool f64 = c.precision == 1;
    if (c.precision != 0 && c.precision != 1) return fail(CULBM_ERR_INVALID_ARGUMENT, "precision must be 0 or 1");
    if (f64 != (c.storage == CULBM_STORAGE_F64))
        return fail(CULBM_ERR_UNSUPPORTED, "FP64 precision goes with FP64 storage and only with it");
    culbm_adj* a = new culbm_adj();
    a->cfg = c;
    if (a->cfg.plane_x[1] < 0) a->cfg.plane_x[1] = static_cast<int>(c.domain_dim[0]) - 2;
    for (int k = 0; k < 2; ++k)
        if (a->cfg.plane_x[k] < 0 || a->cfg.plane_x[k] >= static_cast<int>(c.domain_dim[0])) {
            delete a;
            return fail(CULBM_ERR_INVALID_ARGUMENT, "measurement plane outside the domain");
        }
    a->dev = c.dev_id;
    a->dom.nx = c.domain_dim[0];
    a->dom.ny = c.domain_dim[1];
    a->dom.nz = c.domain_dim[2];
    a->dom.nxy = a->dom.nx * a->dom.ny;
    a->n = static_cast<long long>(n);
    a->dom.n = static_cast<int>(n);
    a->inv_tau = c.inv_tau;
    a->state_storage = c.storage;
    if (c.checkpoint_storage != 0 && c.checkpoint_storage != c.storage) {
        if (c.storage != CULBM_STORAGE_F32 ||
            (c.checkpoint_storage != CULBM_STORAGE_F16 && c.checkpoint_storage != CULBM_STORAGE_F16_SR)) {
            delete a;
            return fail(CULBM_ERR_UNSUPPORTED, "checkpoint_storage F16 or F16_SR goes with storage F32");
        }
        a->mixed = true;
        a->state_storage = c.checkpoint_storage;
    }
    a->esize = a->state_storage == CULBM_STORAGE_F64 ? 8 : a->state_storage == CULBM_STORAGE_F32 ? 4 : 2;
    a->rsize = f64 ? 8 : 4;
    const int T = c.window[1];
    const double state_bytes = 27.0 * n * a->esize;
    if (c.checkpoint_inner < 0 || (c.checkpoint_inner > 0 && c.checkpoint_inner >= c.checkpoint_every)) {
        delete a;
        return fail(CULBM_ERR_INVALID_ARGUMENT, "checkpoint_inner must be 0 or lie in [1, checkpoint_every)");
    }
    auto body = [&]() -> culbm_status {
        CULBM_CUDA(cudaSetDevice(a->dev));
        CULBM_CUDA(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
        CULBM_CUDA(cudaEventCreate(&a->ev[0]));
        CULBM_CUDA(cudaEventCreate(&a->ev[1]));
        // everything but the states (an upper bound): adjoint populations,
        // per-cell inputs and gradients, EQU list and block slots, objective
        // planes and sums
        const double fixed = 2.0 * 27 * n * a->rsize + 5.0 * 8 * n + 27.0 * n +
                             16.0 * (c.window[1] - c.window[0] + 1) * (1.0 + c.domain_dim[1] * c.domain_dim[2]) +
                             (a->mixed ? 2.0 * 27 * n * sizeof(float) : 0.0);
        double budget = static_cast<double>(c.hbm_budget_bytes);
        if (budget == 0) {
            size_t free_b = 0, total_b = 0;
            CULBM_CUDA(cudaMemGetInfo(&free_b, &total_b));
            budget = 0.95 * static_cast<double>(free_b) - (256 << 20);
        }
        CkptPlan plan;
        if (c.checkpoint_every > 0) {
            plan = make_plan(T, c.checkpoint_every, c.checkpoint_inner);
        } else {
            const long long max_states = static_cast<long long>(std::max(0.0, (budget - fixed) / state_bytes));
            if (!choose_plan(T, max_states, plan))
                return fail(CULBM_ERR_OUT_OF_MEMORY,
                            "no checkpoint plan fits: the smallest needs " +
                                std::to_string((plan.states() * state_bytes + fixed) / 1e9) + " GB of " +
                                std::to_string(budget / 1e9) + " GB");
        }
        a->K = plan.K;
        a->K2 = plan.K2;
        a->nckpt = plan.nckpt;
        a->ninner = plan.ninner;
        a->nseg = plan.nseg;
        const double need = plan.states() * state_bytes + fixed;
        if (c.hbm_budget_bytes && need > static_cast<double>(c.hbm_budget_bytes))
            return fail(CULBM_ERR_OUT_OF_MEMORY, "adjoint needs " + std::to_string(need / 1e9) +
                                                     " GB, over the HBM budget of " +
                                                     std::to_string(c.hbm_budget_bytes / 1e9) + " GB");
        void* p = nullptr;
        CULBM_TRY(adj_alloc(a, &p, n, "op bytes"));
        a->d_ops = static_cast<uint8_t*>(p);
        for (int k = 0; k < 4; ++k) {
            CULBM_TRY(adj_alloc(a, &p, n * sizeof(float), "macroscopic inputs"));
            a->d_mac[k] = static_cast<float*>(p);
        }
        CULBM_TRY(adj_alloc(a, &p, n * sizeof(float), "soft field"));
        a->d_soft = static_cast<float*>(p);
        CULBM_TRY(adj_alloc(a, &a->d_ckpt, static_cast<size_t>(a->nckpt * state_bytes), "checkpoints"));
        if (a->ninner)
            CULBM_TRY(adj_alloc(a, &a->d_inner, static_cast<size_t>(a->ninner * state_bytes), "inner checkpoints"));
        CULBM_TRY(adj_alloc(a, &a->d_seg, static_cast<size_t>(a->nseg * state_bytes), "recompute segment"));
        if (a->mixed)
            for (int k = 0; k < 2; ++k)
                CULBM_TRY(adj_alloc(a, &a->d_fwd[k], 27ull * n * sizeof(float), "FP32 forward states"));
        CULBM_TRY(adj_alloc(a, &a->d_nu, 2ull * 27 * n * a->rsize, "adjoint populations"));
        CULBM_TRY(adj_alloc(a, &p, n * sizeof(double), "soft gradient"));
        a->d_gsoft = static_cast<double*>(p);
        CULBM_TRY(adj_alloc(a, &p, 4 * n * sizeof(double), "EQU input gradients"));
        a->d_gmac = static_cast<double*>(p);
        const long long nt = c.window[1] - c.window[0] + 1;
        CULBM_TRY(adj_alloc(a, &p, 2ull * nt * sizeof(double), "objective sums"));
        a->d_psum = static_cast<double*>(p);
        CULBM_TRY(adj_alloc(a, &p, 2ull * nt * a->dom.ny * a->dom.nz * sizeof(double), "objective planes"));
        a->d_rho_plane = static_cast<double*>(p);
        return CULBM_OK;
    };
    const culbm_status st = body();
    if (st != CULBM_OK) {
        const std::string msg = culbm_last_error();
        adj_release(a);
        set_last_error(msg);
        return st;
    }
    const culbm_status st2 = culbm_adj_set_state(a, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (st2 != CULBM_OK) {
        const std::string msg = culbm_last_error();
        adj_release(a);
        set_last_error(msg);
        return st2;
    }
    *out = a;
    return CULBM_OK;
}

culbm_status culbm_adj_destroy(culbm_adj* adj)
{
    adj_release(adj);
    return CULBM_OK;
}

culbm_status culbm_adj_set_state(culbm_adj* a, const uint32_t* flag, const float* rho, const float* vx,
                                 const float* vy, const float* vz, const float* soft)
{
    if (!a) return fail(CULBM_ERR_INVALID_ARGUMENT, "adjoint handle is NULL");
    CULBM_CUDA(cudaSetDevice(a->dev));
    const Domain& D = a->dom;
    const size_t n = static_cast<size_t>(a->n);
    std::vector<uint8_t> ops(n);
    std::vector<int> equ;
    constexpr uint32_t kFluid = FLAG_LOAD | FLAG_COLLIDE | FLAG_STORE;
    int n_in = 0, n_out = 0;
    for (int z = 0; z < D.nz; ++z)
        for (int y = 0; y < D.ny; ++y)
            for (int x = 0; x < D.nx; ++x) {
                const size_t i = x + static_cast<size_t>(D.nx) * (y + static_cast<size_t>(D.ny) * z);
                const uint32_t fl = flag ? flag[i] : kFluid;
                if ((fl & 0x1Fu) != 0 && !(fl & FLAG_STORE))
                    return fail(CULBM_ERR_INVALID_ARGUMENT, "adjoint model: every active cell needs STORE");
                uint8_t op = static_cast<uint8_t>(fl & 0x1Fu);
                ops[i] = op;
                if (op & OP_EQU) equ.push_back(static_cast<int>(i));
                if (op & OP_COLLIDE) {
                    n_in += x == a->cfg.plane_x[0];
                    n_out += x == a->cfg.plane_x[1];
                }
            }
    if (n_in == 0 || n_out == 0) return fail(CULBM_ERR_INVALID_ARGUMENT, "a measurement plane has no COLLIDE cell");
    a->n_in = n_in;
    a->n_out = n_out;
    CULBM_CUDA(cudaStreamSynchronize(a->stream));
    const int n_equ = static_cast<int>(equ.size());
    // the EQU list and the invTau block slots of the adjoint-step launch
    // (whose grid grows with the EQU count) are sized here
    a->n_equ = 0;
    if (n_equ > a->equ_capacity) {
        CULBM_CUDA(cudaFree(a->d_equ));
        a->d_equ = nullptr;
        a->device_bytes -= a->equ_capacity * sizeof(int);
        a->equ_capacity = 0;
        void* p = nullptr;
        CULBM_TRY(adj_alloc(a, &p, n_equ * sizeof(int), "EQU cell list"));
        a->d_equ = static_cast<int*>(p);
        a->equ_capacity = n_equ;
    }
    {
        const dim3 gr = adj::adj_grid(a->dom, n_equ);
        if (gr.z > 65535)
            return fail(CULBM_ERR_INVALID_ARGUMENT, "nz plus the EQU blocks of the adjoint step exceed grid z 65535");
        const long long slots = 8ll * gr.x * gr.y * gr.z;   // one per warp
        if (slots > a->tau_capacity) {
            CULBM_CUDA(cudaFree(a->d_gtau));
            a->d_gtau = nullptr;
            a->device_bytes -= a->tau_capacity * sizeof(double);
            a->tau_capacity = 0;
            void* p = nullptr;
            CULBM_TRY(adj_alloc(a, &p, slots * sizeof(double), "invTau gradient"));
            a->d_gtau = static_cast<double*>(p);
            a->tau_capacity = slots;
        }
        a->n_tau_blocks = slots;
    }
    a->n_equ = n_equ;
    if (n_equ)
        CULBM_CUDA(cudaMemcpyAsync(a->d_equ, equ.data(), n_equ * sizeof(int), cudaMemcpyHostToDevice, a->stream));
    CULBM_CUDA(cudaMemcpyAsync(a->d_ops, ops.data(), n, cudaMemcpyHostToDevice, a->stream));
    const float* mac[4] = {rho, vx, vy, vz};
    const float dflt[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    std::vector<float> tmp;
    for (int k = 0; k < 4; ++k) {
        const float* src = mac[k];
        if (!src) {
            tmp.assign(n, dflt[k]);
            src = tmp.data();
        }
        CULBM_CUDA(cudaMemcpyAsync(a->d_mac[k], src, n * sizeof(float), cudaMemcpyHostToDevice, a->stream));
        CULBM_CUDA(cudaStreamSynchronize(a->stream));
    }
    if (soft) {
        for (size_t i = 0; i < n; ++i)
            if (!(soft[i] >= 0.0f && soft[i] <= 1.0f))
                return fail(CULBM_ERR_INVALID_ARGUMENT, "soft field values must lie in [0, 1]");
        CULBM_CUDA(cudaMemcpyAsync(a->d_soft, soft, n * sizeof(float), cudaMemcpyHostToDevice, a->stream));
    } else {
        CULBM_CUDA(cudaMemsetAsync(a->d_soft, 0, n * sizeof(float), a->stream));
    }
    CULBM_CUDA(cudaStreamSynchronize(a->stream));
    return CULBM_OK;
}

culbm_status culbm_adj_set_inv_tau(culbm_adj* a, double inv_tau)
{
    if (!a) return fail(CULBM_ERR_INVALID_ARGUMENT, "adjoint handle is NULL");
    if (!(inv_tau > 0.0 && inv_tau < 2.0)) return fail(CULBM_ERR_INVALID_ARGUMENT, "invTau must lie in (0, 2)");
    a->inv_tau = inv_tau;
    return CULBM_OK;
}

culbm_status culbm_adj_forward(culbm_adj* a, double* J)
{
    if (!a || !J) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    CULBM_CUDA(cudaSetDevice(a->dev));
    CULBM_CUDA(cudaEventRecord(a->ev[0], a->stream));
    CULBM_TRY(adj_with_storage(a, [&](auto tag) {
        using S = typename decltype(tag)::type;
        return a->mixed ? run_forward_mixed<S>(a, false) : run_forward<S>(a, false);
    }));
    a->t_fwd = elapsed(a);
    return objective(a, J);
}

culbm_status culbm_adj_gradient(culbm_adj* a, double* J, double* dJ_dinv_tau, double* dJ_dsoft, double* dJ_dmac)
{
    if (!a) return fail(CULBM_ERR_INVALID_ARGUMENT, "adjoint handle is NULL");
    CULBM_CUDA(cudaSetDevice(a->dev));
    CULBM_TRY(adj_with_storage(a, [&](auto tag) { return run_gradient<typename decltype(tag)::type>(a); }));
    double j = 0;
    CULBM_TRY(objective(a, &j));
    if (J) *J = j;
    const size_t n = static_cast<size_t>(a->n);
    if (dJ_dinv_tau) {
        std::vector<double> g(static_cast<size_t>(a->n_tau_blocks));
        CULBM_CUDA(cudaMemcpy(g.data(), a->d_gtau, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
        double s = 0;
        for (double v : g) s += v;
        *dJ_dinv_tau = s;
    }
    if (dJ_dsoft) CULBM_CUDA(cudaMemcpy(dJ_dsoft, a->d_gsoft, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (dJ_dmac) CULBM_CUDA(cudaMemcpy(dJ_dmac, a->d_gmac, 4 * n * sizeof(double), cudaMemcpyDeviceToHost));
    return CULBM_OK;
}

culbm_status culbm_adj_get_info(culbm_adj* a, culbm_adj_info* info)
{
    if (!a || !info) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->checkpoint_every = a->K;
    info->checkpoints = a->nckpt;
    info->checkpoint_inner = a->K2;
    info->inner_checkpoints = a->ninner;
    info->device_bytes = a->device_bytes;
    info->forward_ms = a->t_fwd;
    info->recompute_ms = a->t_rec;
    info->adjoint_ms = a->t_adj;
    info->steps = static_cast<uint64_t>(a->cfg.window[1]);
    return CULBM_OK;
}

}  // extern "C"
