// Whole-domain step kernels: pull double-buffer and in-place (AA pattern),
// plus the moment (dump), state export/import and fill kernels that know how
// each layout stores the populations.
//
// Layout in HBM: structure of arrays, one array per direction d, cell index
// i = x + nx*(y + ny*z) (x fastest), exactly the reference's order
// (src/simulator/single_dev_expt/kernel.cu:48-51) so that dumps and init
// files map 1:1.  Each direction has its own base pointer in the kernel
// parameters (constant bank), so no per-direction 64-bit offset is kept in
// registers.
//
// Edge semantics: the reference's pull clamps each neighbour offset component
// to 0 at the domain boundary (kernel.cu:2506-2511), so a boundary cell pulls
// a direction whose source is outside from the source with the offending
// components replaced by its own (itself for face-normal directions, a
// neighbour along the face otherwise).  The pull kernel does the same.  The
// in-place kernels reproduce it bit for bit with a small side buffer ("edge
// buffer") that holds, for each boundary cell and each such direction, the
// post-collision population of that clamped source.
#pragma once

#include <type_traits>

#include "d3q27.cuh"
#include "storage.cuh"

namespace culbm {

struct Domain {
    int nx, ny, nz;
    int nxy;   // nx*ny
    int n;     // nx*ny*nz (< 2^31, checked on the host)
};

// The 27 population planes of one buffer, one base pointer per direction
// (kernel parameters, so no per-plane offset sits in a register).
template <typename S>
struct Pops {
    S* p[27];
    __host__ void set(S* b, long long stride)
    {
        for (int d = 0; d < 27; ++d) p[d] = b + d * stride;
    }
};

// Edge buffer: six face blocks (x-low, x-high, y-low, y-high, z-low, z-high),
// each 9 directions x face cells.  A clamped (cell, d) pair is filed under
// the first axis (x, then y, then z) along which cell - c_d leaves the domain;
// the nine directions of a face are indexed by the two other components.
struct EdgeLayout {
    long long off[6];
};

template <typename S, typename R>
struct StepArgs {
    Domain dom;
    const uint8_t* ops;
    const float* rho;
    const float* vx;
    const float* vy;
    const float* vz;
    R inv_tau;
    Pops<S> src;   // pull: read buffer.  in-place: the single buffer.
    Pops<S> dst;   // pull: write buffer.  in-place: same buffer as src.
    S* edge;       // in-place only
    EdgeLayout el;
    int ring_nz;   // LAYOUT_PULL_RING: planes in the ring buffer
    int ring_off;  // LAYOUT_PULL_RING: ring plane of domain plane z = 0
    uint32_t seed; // step_seed of the time step being written (stochastic rounding)
};

__device__ __forceinline__ int nb_off(const Domain& D, int d)
{
    return cx_of(d) + cy_of(d) * D.nx + cz_of(d) * D.nxy;
}

__device__ __forceinline__ bool inside(const Domain& D, int x, int y, int z)
{
    return (unsigned)x < (unsigned)D.nx && (unsigned)y < (unsigned)D.ny && (unsigned)z < (unsigned)D.nz;
}

// Element index of the edge-buffer slot of (x,y,z,d); only valid when
// (x,y,z) - c_d is outside the domain.
__device__ __forceinline__ long long edge_slot(const Domain& D, const EdgeLayout& L, int x, int y, int z, int d)
{
    const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
    const int sx = x - cx, sy = y - cy;
    if ((unsigned)sx >= (unsigned)D.nx) {
        const int j = (cy + 1) + 3 * (cz + 1);
        return L.off[sx < 0 ? 0 : 1] + (long long)j * D.ny * D.nz + y + (long long)D.ny * z;
    }
    if ((unsigned)sy >= (unsigned)D.ny) {
        const int j = (cx + 1) + 3 * (cz + 1);
        return L.off[sy < 0 ? 2 : 3] + (long long)j * D.nx * D.nz + x + (long long)D.nx * z;
    }
    const int sz = z - cz;
    const int j = (cx + 1) + 3 * (cy + 1);
    return L.off[sz < 0 ? 4 : 5] + (long long)j * D.nx * D.ny + x + (long long)D.nx * y;
}

// The reference clamps a pull per axis: a component of x - c_d that leaves
// the domain is replaced by x's own component, the others are kept.  So the
// clamped source of (y, d) is s = clamp(y - c_d), usually a neighbour of y and
// not y itself.  For a source cell s and direction d this visits every
// boundary cell y != s + c_d whose clamped pull in direction d reads s: take
// y = s + c_d and put back s's own component on any non-empty subset of the
// axes along which s - c_d leaves the domain.
template <int D_, class F>
__device__ __forceinline__ void for_each_clamp_reader(const Domain& D, int sx, int sy, int sz, F&& fn)
{
    constexpr int cx = cx_of(D_), cy = cy_of(D_), cz = cz_of(D_);
    const bool kx = cx != 0 && (unsigned)(sx - cx) >= (unsigned)D.nx;
    const bool ky = cy != 0 && (unsigned)(sy - cy) >= (unsigned)D.ny;
    const bool kz = cz != 0 && (unsigned)(sz - cz) >= (unsigned)D.nz;
#pragma unroll
    for (int m = 1; m < 8; ++m) {
        if ((m & 1) && !kx) continue;
        if ((m & 2) && !ky) continue;
        if ((m & 4) && !kz) continue;
        const int yx = (m & 1) ? sx : sx + cx;
        const int yy = (m & 2) ? sy : sy + cy;
        const int yz = (m & 4) ? sz : sz + cz;
        if (inside(D, yx, yy, yz)) fn(yx, yy, yz);
    }
}

// How the current state stores "the population f_d that cell x pulls next":
//   LAYOUT_PULL  standard: post-collision f*_d(y) at [d][y]; pull from x - c_d,
//                clamped per axis at the boundary (pull double buffer, tiles).
//   LAYOUT_AA_A  reversed own: f*_d(y) at [26-d][y]; pull from x - c_d,
//                clamped values from the edge buffer (in-place, after an even
//                step and at start).
//   LAYOUT_AA_B  streamed: the pulled value already sits at [d][x]
//                (in-place, after an odd step).
//   LAYOUT_PULL_RING  standard, in the z-rotating ring buffer of the blocked
//                in-place policy: domain plane z lives at ring plane
//                (z + ring_off) mod ring_nz.
enum Layout : int { LAYOUT_PULL = 0, LAYOUT_AA_A = 1, LAYOUT_AA_B = 2, LAYOUT_PULL_RING = 3 };

template <typename S, typename R>
__device__ __forceinline__ long long ring_index(const StepArgs<S, R>& a, int x, int y, int z)
{
    int pz = z + a.ring_off;
    if (pz >= a.ring_nz) pz -= a.ring_nz;
    return (long long)pz * a.dom.nxy + (long long)y * a.dom.nx + x;
}

// The cell update of storage format S on f (raw values 2^E f with RAW, E =
// ScaleExp<S>): the compact form for the 16-bit formats (their stored
// rounding dominates, see cell_update_fast), the reference's exact operation
// order for FP32 and FP64.
template <typename S, bool RAW, typename R>
__device__ __forceinline__ void cell_update_for(uint8_t op, R inv_tau, const float* __restrict__ rho,
                                                const float* __restrict__ vx, const float* __restrict__ vy,
                                                const float* __restrict__ vz, int64_t i, R* f)
{
    constexpr int E = RAW ? ScaleExp<S>::value : 0;
    if constexpr (Is16<S>::value)
        cell_update_fast<E>(op, inv_tau, rho, vx, vy, vz, i, f);
    else
        cell_update<R, E>(op, inv_tau, rho, vx, vy, vz, i, f);
}

// Load of a stored population from global memory: the value f, or with RAW
// its raw form 2^E * f (E = ScaleExp<S>) for the step kernels, which fold the
// scale into the cell update and stream the planes (ld_stream_raw).
template <bool RAW, typename S, typename R>
__device__ __forceinline__ R ld_as(const S* p)
{
    if constexpr (RAW)
        return ld_stream_raw<S, R>(p);
    else
        return Cvt<S, R>::ld(p);
}

// Store counterpart of ld_as.
template <bool RAW, typename S, typename R>
__device__ __forceinline__ void put_as(S* p, R v, uint32_t hcell, int d)
{
    if constexpr (RAW)
        put_raw(p, v, hcell, d);
    else
        put(p, v, hcell, d);
}

template <int LAYOUT, bool RAW = false, typename S, typename R>
__device__ __forceinline__ void load_pulled(const StepArgs<S, R>& a, int x, int y, int z, int i, bool edge, R* f)
{
    const Domain& D = a.dom;
    if (LAYOUT == LAYOUT_PULL) {
        const int ndx = (x == 0) ? 0 : -1, pdx = (x == D.nx - 1) ? 0 : 1;
        const int ndy = (y == 0) ? 0 : -D.nx, pdy = (y == D.ny - 1) ? 0 : D.nx;
        const int ndz = (z == 0) ? 0 : -D.nxy, pdz = (z == D.nz - 1) ? 0 : D.nxy;
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int ox = cx_of(d) == 1 ? ndx : cx_of(d) == -1 ? pdx : 0;
            const int oy = cy_of(d) == 1 ? ndy : cy_of(d) == -1 ? pdy : 0;
            const int oz = cz_of(d) == 1 ? ndz : cz_of(d) == -1 ? pdz : 0;
            f[d] = ld_as<RAW, S, R>(a.src.p[d] + (i + ox + oy + oz));
        }
    } else if (LAYOUT == LAYOUT_PULL_RING) {
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            int sx = x - cx_of(d), sy = y - cy_of(d), sz = z - cz_of(d);
            if ((unsigned)sx >= (unsigned)D.nx) sx = x;
            if ((unsigned)sy >= (unsigned)D.ny) sy = y;
            if ((unsigned)sz >= (unsigned)D.nz) sz = z;
            f[d] = ld_as<RAW, S, R>(a.src.p[d] + ring_index(a, sx, sy, sz));
        }
    } else if (LAYOUT == LAYOUT_AA_A) {
        if (!edge) {
#pragma unroll
            for (int d = 0; d < 27; ++d) f[d] = ld_as<RAW, S, R>(a.src.p[26 - d] + (i - nb_off(D, d)));
        } else {
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                if (inside(D, x - cx_of(d), y - cy_of(d), z - cz_of(d)))
                    f[d] = ld_as<RAW, S, R>(a.src.p[26 - d] + (i - nb_off(D, d)));
                else
                    f[d] = ld_as<RAW, S, R>(a.edge + edge_slot(D, a.el, x, y, z, d));
            }
        }
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = ld_as<RAW, S, R>(a.src.p[d] + i);
    }
}

struct CellCoord {
    int x, y, z, i;
    bool valid;
};

// Cell of this thread in a cell_grid launch over the planes z0, z0 + 1, ...
// (grid z = the number of planes).
__device__ __forceinline__ CellCoord cell_of_thread(const Domain& D, int z0 = 0)
{
    CellCoord c;
    c.x = blockIdx.x * blockDim.x + threadIdx.x;
    c.y = blockIdx.y * blockDim.y + threadIdx.y;
    c.z = z0 + static_cast<int>(blockIdx.z);
    c.valid = c.x < D.nx && c.y < D.ny;
    c.i = c.x + D.nx * (c.y + D.ny * c.z);
    return c;
}

// One pull step src -> dst over the planes z0 .. z0 + gridDim.z - 1 (the
// whole domain with z0 = 0 and a cell_grid launch).
// Replaces StaticD3Q27PullKernel, reference kernel.cu:2489-2632.
template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1)
    k_pull_step(const __grid_constant__ StepArgs<S, R> a, int z0)
{
    const CellCoord c = cell_of_thread(a.dom, z0);
    if (!c.valid) return;
    const uint8_t op = a.ops[c.i];
    R f[27];
    if (op & OP_LOAD) {
        load_pulled<LAYOUT_PULL, true>(a, c.x, c.y, c.z, c.i, false, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.i, f);
    if (op & OP_STORE)
        put27_raw<S>(f, cell_hash(static_cast<uint32_t>(c.i), a.seed), [&](int d) { return a.dst.p[d] + c.i; });
}

// In-place odd step (layout A -> B): each cell pulls f_d from the reversed
// slot of x - c_d and pushes its post-collision f_d into slot d of x + c_d.
// Cell x reads and writes exactly the same set of locations, so no other
// thread touches them.  Boundary cells take clamped values from the edge
// buffer, and a cell that is the clamped source of boundary cells y (see
// for_each_clamp_reader) also writes f_d into slot d of each such y: nobody
// else reads or writes that slot during the step, and y reads it next step.
//
// Each in-place step is one launch over two disjoint sets of x-rows (cells
// of different rows never touch the same locations in a step's pattern, so
// the order does not matter):
//   ROWS_INNER: rows with 0 < y < ny-1 and 0 < z < nz-1.  Only the x-faces
//     of such a row are on the boundary, and there only the x component of a
//     pull can leave the domain, so the clamp handling reduces to pointer
//     selects and predicated stores; the code stays straight-line.
//   ROWS_OUTER: rows on a y or z face, processed with the general per-axis
//     clamp code (about 2 (ny + nz) of the ny*nz rows).
// Grid (split_grid): blocks of `cols` x `rows` cells (cols a multiple of 32),
// one warp per 32 cells of a row.  The
// first grid-z slices hold the outer rows (the z = 0 and z = nz-1 planes,
// then the y-face rows of the interior planes), so their longer code runs
// beside the inner rows rather than as a tail; each further slice is one
// interior z-plane of inner rows.  Rows are contiguous in x, so warp
// accesses stay coalesced, and no thread divides by a runtime value.
enum RowSet : int { ROWS_INNER = 0, ROWS_OUTER = 1 };

// Block shape of the in-place step launches (split_grid, slab_split), by
// storage format: one row of 96 cells (three warps, one 32-cell segment
// each) for FP32 and FP64, four rows of 32 for the 16-bit formats.  At the
// same 40 warps per SM, blocks of 32 x 4 ran the in-place FP32 steps 1.3 %
// faster at 288x272x280 and 0.7 % at 512x512x256 than 32 x 8, and 96 x 1
// another 0.7-0.8 %; the 16-bit steps are 0.8 % (288x272x280) and 2.1 %
// (512x512x256) faster with 32 x 4 than with 96 x 1.  The pull is
// indifferent and keeps 32 x 8.
template <typename S>
struct AaShape {
    static constexpr int cols = Is16<S>::value ? 32 : 96;
    static constexpr int rows = Is16<S>::value ? 4 : 1;
};

// Grid-z slices of the outer rows (blocks of `rows` rows).
__host__ __device__ __forceinline__ int outer_slices(const Domain& D, int rows = 8)
{
    const int rows_per_slice = ((D.ny + rows - 1) / rows) * rows;
    const int nzf = D.nz > 1 ? 2 : 1, nyf = D.ny > 1 ? 2 : 1;
    return nzf + (D.nz > 2 ? (nyf * (D.nz - 2) + rows_per_slice - 1) / rows_per_slice : 0);
}

inline dim3 split_grid(const Domain& D, int rows = 8, int cols = 32)
{
    return dim3((D.nx + cols - 1) / cols, (D.ny + rows - 1) / rows,
                outer_slices(D, rows) + (D.nz > 2 ? D.nz - 2 : 0));
}

// Cell of this thread in a split_grid launch whose grid-z slices start at
// z0 (slices below z0 belong to another role); returns ROWS_OUTER or
// ROWS_INNER, or -1 if the thread has no cell.
__device__ __forceinline__ int split_cell(const Domain& D, int z0, CellCoord& c)
{
    c.x = blockIdx.x * blockDim.x + threadIdx.x;
    if (c.x >= D.nx) return -1;
    const int bz = static_cast<int>(blockIdx.z) - z0;
    const int yy = blockIdx.y * blockDim.y + threadIdx.y;
    const int nzf = D.nz > 1 ? 2 : 1;
    const int oz = outer_slices(D, static_cast<int>(blockDim.y));
    int kind;
    if (bz < nzf) {
        if (yy >= D.ny) return -1;
        c.y = yy;
        c.z = bz ? D.nz - 1 : 0;
        kind = ROWS_OUTER;
    } else if (bz < oz) {
        const int q = (bz - nzf) * static_cast<int>(gridDim.y * blockDim.y) + yy;
        if (D.ny > 1) {
            if (q >= 2 * (D.nz - 2)) return -1;
            c.z = 1 + (q >> 1);
            c.y = (q & 1) ? D.ny - 1 : 0;
        } else {
            if (q >= D.nz - 2) return -1;
            c.z = 1 + q;
            c.y = 0;
        }
        kind = ROWS_OUTER;
    } else {
        c.z = 1 + (bz - oz);
        c.y = 1 + yy;
        if (c.y > D.ny - 2) return -1;
        kind = ROWS_INNER;
    }
    c.i = c.x + D.nx * (c.y + D.ny * c.z);
    c.valid = true;
    return kind;
}

template <typename S>
__device__ __forceinline__ const S* xface_edge_ptr(const S* edge, const Domain& D, const EdgeLayout& L, int side,
                                                   int d, int y, int z)
{
    const int j = (cy_of(d) + 1) + 3 * (cz_of(d) + 1);
    return edge + L.off[side] + (long long)j * D.ny * D.nz + y + (long long)D.ny * z;
}

template <typename S, typename R, int ROWS>
__device__ __forceinline__ void aa_odd_cell(const StepArgs<S, R>& a, const CellCoord c)
{
    const Domain& D = a.dom;
    const uint8_t op = a.ops[c.i];
    const uint32_t hc = cell_hash(static_cast<uint32_t>(c.i), a.seed);
    // Warps without an x-face lane (all but the first and last of a row) take
    // the straight path; the choice is uniform across the warp.
    const int xw = c.x - (threadIdx.x & 31);
    const bool xface = ROWS == ROWS_INNER && (xw == 0 || xw + 31 >= D.nx - 1);
    R f[27];
    if (op & OP_LOAD) {
        if (ROWS == ROWS_INNER && !xface) {
#pragma unroll
            for (int d = 0; d < 27; ++d) f[d] = ld_stream_raw<S, R>(a.src.p[26 - d] + (c.i - nb_off(D, d)));
        } else if (ROWS == ROWS_INNER) {
            // A warp with an x-face lane loads like the others, the face lane
            // from its own column for the directions whose source lies
            // outside (so every load stays in the domain), and that lane
            // alone then takes those directions from the edge buffer.
            const bool lo = c.x == 0, hi = c.x == D.nx - 1;
            const int ip = c.i + (lo ? 1 : 0), im = c.i - (hi ? 1 : 0);
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const int base = cx_of(d) == 1 ? ip : cx_of(d) == -1 ? im : c.i;
                f[d] = ld_stream_raw<S, R>(a.src.p[26 - d] + (base - nb_off(D, d)));
            }
            if (lo) {
#pragma unroll
                for (int d = 2; d < 27; d += 3) f[d] = ld_stream_raw<S, R>(xface_edge_ptr(a.edge, D, a.el, 0, d, c.y, c.z));
            }
            if (hi) {
#pragma unroll
                for (int d = 0; d < 27; d += 3) f[d] = ld_stream_raw<S, R>(xface_edge_ptr(a.edge, D, a.el, 1, d, c.y, c.z));
            }
        } else {
            load_pulled<LAYOUT_AA_A, true>(a, c.x, c.y, c.z, c.i, true, f);
        }
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.i, f);
    if (!(op & OP_STORE)) return;
    if (ROWS == ROWS_INNER && !xface) {
        put27_raw<S>(f, hc, [&](int d) { return a.dst.p[d] + (c.i + nb_off(D, d)); });
    } else if (ROWS == ROWS_INNER) {
        // streaming target x + c_d, unless it leaves the domain in x
        const bool lo = c.x == 0, hi = c.x == D.nx - 1;
        put27_raw_if<S>(f, hc, [&](int d) { return a.dst.p[d] + (c.i + nb_off(D, d)); },
                        [&](int d) { return !((cx_of(d) == 1 && hi) || (cx_of(d) == -1 && lo)); });
        // an x-face cell is the clamped source of the cell on its own face
        if (lo) {
#pragma unroll
            for (int d = 2; d < 27; d += 3) put_raw(a.dst.p[d] + (c.i + nb_off(D, d) - 1), f[d], hc, d);
        }
        if (hi) {
#pragma unroll
            for (int d = 0; d < 27; d += 3) put_raw(a.dst.p[d] + (c.i + nb_off(D, d) + 1), f[d], hc, d);
        }
    } else {
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            if (inside(D, c.x + cx_of(d), c.y + cy_of(d), c.z + cz_of(d)))
                put_raw(a.dst.p[d] + (c.i + nb_off(D, d)), f[d], hc, d);
            for_each_clamp_reader<d>(D, c.x, c.y, c.z, [&](int yx, int yy, int yz) {
                put_raw(a.dst.p[d] + (yx + D.nx * (yy + D.ny * yz)), f[d], hc, d);
            });
        });
    }
}

// In-place even step (layout B -> A): own slots in, reversed own slots out.
// A cell that is the clamped source of boundary cells y also files f_d into
// the edge-buffer slot of (y, d): the next odd step's clamped pull of y reads
// it there, because slot 26-d of the source is overwritten during that step.
template <typename S, typename R, int ROWS>
__device__ __forceinline__ void aa_even_cell(const StepArgs<S, R>& a, const CellCoord c)
{
    const Domain& D = a.dom;
    const uint8_t op = a.ops[c.i];
    const uint32_t hc = cell_hash(static_cast<uint32_t>(c.i), a.seed);
    R f[27];
    if (op & OP_LOAD) {
        load_pulled<LAYOUT_AA_B, true>(a, c.x, c.y, c.z, c.i, false, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.i, f);
    if (!(op & OP_STORE)) return;
    put27_raw<S>(f, hc, [&](int d) { return a.dst.p[26 - d] + c.i; });
    if (ROWS == ROWS_INNER) {
        if (c.x != 0 && c.x != D.nx - 1) return;
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int cx = cx_of(d);
            if (cx == 1 && c.x == 0)
                put_raw(const_cast<S*>(xface_edge_ptr(a.edge, D, a.el, 0, d, c.y + cy_of(d), c.z + cz_of(d))), f[d], hc,
                        d);
            if (cx == -1 && c.x == D.nx - 1)
                put_raw(const_cast<S*>(xface_edge_ptr(a.edge, D, a.el, 1, d, c.y + cy_of(d), c.z + cz_of(d))), f[d], hc,
                        d);
        }
    } else {
        for_dirs([&](auto dd) {
            constexpr int d = decltype(dd)::value;
            for_each_clamp_reader<d>(D, c.x, c.y, c.z, [&](int yx, int yy, int yz) {
                put_raw(a.edge + edge_slot(D, a.el, yx, yy, yz, d), f[d], hc, d);
            });
        });
    }
}

// In-place steps over both row sets (split_grid; the row kind is uniform
// over a block).
template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1) k_aa_odd(const __grid_constant__ StepArgs<S, R> a)
{
    CellCoord c;
    const int kind = split_cell(a.dom, 0, c);
    if (kind == ROWS_OUTER)
        aa_odd_cell<S, R, ROWS_OUTER>(a, c);
    else if (kind == ROWS_INNER)
        aa_odd_cell<S, R, ROWS_INNER>(a, c);
}

template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1) k_aa_even(const __grid_constant__ StepArgs<S, R> a)
{
    CellCoord c;
    const int kind = split_cell(a.dom, 0, c);
    if (kind == ROWS_OUTER)
        aa_even_cell<S, R, ROWS_OUTER>(a, c);
    else if (kind == ROWS_INNER)
        aa_even_cell<S, R, ROWS_INNER>(a, c);
}

// Grid-z layout of an in-place launch over the slab of planes za .. zb-1
// (the overlapped host run): split_grid restricted to the slab.  First the
// z-face planes the slab holds (z = 0, z = nz-1), then slices of the y-face
// rows of its interior planes, then one slice per interior plane; so the
// outer rows, with their longer clamp code, keep blocks of their own.
struct SlabSplit {
    int za;    // first plane of the slab
    int zlo;   // first interior plane (0 < z < nz-1) of the slab
    int ni;    // interior planes in the slab
    int nzf;   // z-face planes in the slab
    int nys;   // slices of y-face rows
};

__host__ __device__ inline SlabSplit slab_split(const Domain& D, int za, int zb, int rows = 8)
{
    SlabSplit q;
    q.za = za;
    q.zlo = za > 1 ? za : 1;
    const int zhi = zb < D.nz - 1 ? zb : D.nz - 1;
    q.ni = zhi > q.zlo ? zhi - q.zlo : 0;
    q.nzf = (za == 0 ? 1 : 0) + (D.nz > 1 && zb == D.nz ? 1 : 0);
    const int rows_per_slice = ((D.ny + rows - 1) / rows) * rows;
    const int nyf = D.ny > 1 ? 2 : 1;
    q.nys = (nyf * q.ni + rows_per_slice - 1) / rows_per_slice;
    return q;
}

inline dim3 slab_split_grid(const Domain& D, const SlabSplit& q, int rows = 8, int cols = 32)
{
    return dim3((D.nx + cols - 1) / cols, (D.ny + rows - 1) / rows, q.nzf + q.nys + q.ni);
}

// Cell of this thread in a slab_split_grid launch: ROWS_OUTER, ROWS_INNER
// (uniform over a block), or -1 if the thread has no cell.
__device__ __forceinline__ int slab_split_cell(const Domain& D, const SlabSplit& q, CellCoord& c)
{
    c.x = blockIdx.x * blockDim.x + threadIdx.x;
    if (c.x >= D.nx) return -1;
    const int bz = static_cast<int>(blockIdx.z);
    const int yy = blockIdx.y * blockDim.y + threadIdx.y;
    int kind;
    if (bz < q.nzf) {
        if (yy >= D.ny) return -1;
        c.y = yy;
        c.z = (bz == 0 && q.za == 0) ? 0 : D.nz - 1;
        kind = ROWS_OUTER;
    } else if (bz < q.nzf + q.nys) {
        const int r = (bz - q.nzf) * static_cast<int>(gridDim.y * blockDim.y) + yy;
        if (D.ny > 1) {
            if (r >= 2 * q.ni) return -1;
            c.z = q.zlo + (r >> 1);
            c.y = (r & 1) ? D.ny - 1 : 0;
        } else {
            if (r >= q.ni) return -1;
            c.z = q.zlo + r;
            c.y = 0;
        }
        kind = ROWS_OUTER;
    } else {
        c.z = q.zlo + (bz - q.nzf - q.nys);
        c.y = 1 + yy;
        if (c.y > D.ny - 2) return -1;
        kind = ROWS_INNER;
    }
    c.i = c.x + D.nx * (c.y + D.ny * c.z);
    c.valid = true;
    return kind;
}

// In-place steps over a slab of planes (the overlapped host run).  A cell
// of one step touches only locations within one plane of itself, so slabs
// at least two planes thick can run a step concurrently, and a slab's next
// step needs only this step done on the slab and its two neighbours.
template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1)
    k_aa_odd_slab(const __grid_constant__ StepArgs<S, R> a, SlabSplit q)
{
    CellCoord c;
    const int kind = slab_split_cell(a.dom, q, c);
    if (kind == ROWS_OUTER)
        aa_odd_cell<S, R, ROWS_OUTER>(a, c);
    else if (kind == ROWS_INNER)
        aa_odd_cell<S, R, ROWS_INNER>(a, c);
}

template <typename S, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1)
    k_aa_even_slab(const __grid_constant__ StepArgs<S, R> a, SlabSplit q)
{
    CellCoord c;
    const int kind = slab_split_cell(a.dom, q, c);
    if (kind == ROWS_OUTER)
        aa_even_cell<S, R, ROWS_OUTER>(a, c);
    else if (kind == ROWS_INNER)
        aa_even_cell<S, R, ROWS_INNER>(a, c);
}

// Moments of the pulled populations, written where the DUMP bits are set.
// Replaces StaticD3Q27PullDumpKernel, reference kernel.cu:2634-2735 (and the
// per-tile dump kernels, which compute the same values for CORRECT cells).
template <int LAYOUT, typename S, typename R>
__global__ void __launch_bounds__(256) k_moments(const __grid_constant__ StepArgs<S, R> a, const uint32_t* flag,
                                                 float* rho, float* vx, float* vy, float* vz, int z0)
{
    const CellCoord c = cell_of_thread(a.dom, z0);
    if (!c.valid) return;
    const uint32_t fl = flag[c.i];
    if ((fl & (FLAG_DUMP_RHO | FLAG_DUMP_VX | FLAG_DUMP_VY | FLAG_DUMP_VZ)) == 0) return;
    const bool edge = (a.ops[c.i] & OP_EDGE) != 0;
    R f[27], r, ux, uy, uz;
    load_pulled<LAYOUT>(a, c.x, c.y, c.z, c.i, edge, f);
    moments<R>(f, r, ux, uy, uz);
    if (fl & FLAG_DUMP_RHO) rho[c.i] = float(r);
    if (fl & FLAG_DUMP_VX) vx[c.i] = float(ux);
    if (fl & FLAG_DUMP_VY) vy[c.i] = float(uy);
    if (fl & FLAG_DUMP_VZ) vz[c.i] = float(uz);
}

// Export the pulled populations out[d*n + i] (T = float or double).
template <int LAYOUT, typename S, typename R, typename T>
__global__ void __launch_bounds__(256) k_export_pulled(const __grid_constant__ StepArgs<S, R> a, T* out)
{
    const CellCoord c = cell_of_thread(a.dom);
    if (!c.valid) return;
    const bool edge = (a.ops[c.i] & OP_EDGE) != 0;
    R f[27];
    load_pulled<LAYOUT>(a, c.x, c.y, c.z, c.i, edge, f);
#pragma unroll
    for (int d = 0; d < 27; ++d) out[(long long)d * a.dom.n + c.i] = T(f[d]);
}

// Import a state given as post-collision populations in the standard layout
// in[d*n + i] (T = float or double) into LAYOUT_PULL / LAYOUT_PULL_RING (dst)
// or LAYOUT_AA_A.
template <int LAYOUT, typename S, typename R, typename T>
__global__ void __launch_bounds__(256) k_import(const __grid_constant__ StepArgs<S, R> a, const T* in)
{
    const CellCoord c = cell_of_thread(a.dom);
    if (!c.valid) return;
    const Domain& D = a.dom;
#pragma unroll 1
    for (int d = 0; d < 27; ++d) {
        const R v = R(in[(long long)d * D.n + c.i]);
        if (LAYOUT == LAYOUT_PULL) {
            put(a.dst.p[d] + c.i, v, cell_hash(static_cast<uint32_t>(c.i), a.seed), d);
        } else if (LAYOUT == LAYOUT_PULL_RING) {
            put(a.dst.p[d] + ring_index(a, c.x, c.y, c.z), v, cell_hash(static_cast<uint32_t>(c.i), a.seed), d);
        } else {
            put(a.dst.p[26 - d] + c.i, v, cell_hash(static_cast<uint32_t>(c.i), a.seed), d);
            int sx = c.x - cx_of(d), sy = c.y - cy_of(d), sz = c.z - cz_of(d);
            if (!inside(D, sx, sy, sz)) {
                if ((unsigned)sx >= (unsigned)D.nx) sx = c.x;
                if ((unsigned)sy >= (unsigned)D.ny) sy = c.y;
                if ((unsigned)sz >= (unsigned)D.nz) sz = c.z;
                const int si = sx + D.nx * (sy + D.ny * sz);
                const R w = R(in[(long long)d * D.n + si]);
                put(a.edge + edge_slot(D, a.el, c.x, c.y, c.z, d), w, cell_hash(static_cast<uint32_t>(si), a.seed), d);
            }
        }
    }
}

// Uniform equilibrium fill feq(rho, u) of every cell (and of the edge buffer
// for LAYOUT_AA_A): the reference starts from calcEqu(1,0,0,0) everywhere
// (simulator_expt_platform.cu:230-250).
template <int LAYOUT, typename S, typename R>
__global__ void __launch_bounds__(256) k_fill_equilibrium(const __grid_constant__ StepArgs<S, R> a, R rho, R ux,
                                                          R uy, R uz)
{
    const CellCoord c = cell_of_thread(a.dom);
    if (!c.valid) return;
    const Domain& D = a.dom;
    R f[27];
    equilibrium<R>(rho, ux, uy, uz, f);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (LAYOUT == LAYOUT_PULL) {
            Cvt<S, R>::st(a.dst.p[d] + c.i, f[d]);
        } else {
            Cvt<S, R>::st(a.dst.p[26 - d] + c.i, f[d]);
            if (!inside(D, c.x - cx_of(d), c.y - cy_of(d), c.z - cz_of(d)))
                Cvt<S, R>::st(a.edge + edge_slot(D, a.el, c.x, c.y, c.z, d), f[d]);
        }
    }
}

}  // namespace culbm
