// L2 temporal blocking: innerLoop time steps over one overlapping tile while
// the tile's populations stay resident in L2.
//
// Geometry follows the reference's blocking_core (tile extent
// B = blockDim*gridDim, halo depth innerLoop-1, valid boxes from
// calcValidPrev, src/blocking_core/blocking_alogrithm.hpp:7-41).  Per round
// of I steps and per tile (x-fastest tile order, as the reference):
//
//   first  step: pull from the global state (domain clamp), store into the
//                tile buffer (or, for I = 1, straight to the global result);
//   middle steps: stream inside the tile buffer;
//   last   step: store the tile's valid cells into the global result.
//
// Differences from the reference, by design:
//   * at a domain face inside a tile the pull is clamped exactly as in the
//     plain step (the reference wraps periodically inside the tile there), so
//     every blocked policy is bitwise equal to the plain pull for any flag field;
//   * pulls from outside the tile (halo garbage) read 0 instead of wrapping;
//   * in-place tiles use the AA pattern with the same clamp side buffer as the
//     whole-domain in-place step, instead of the esoteric twist;
//   * cell flags are not re-tiled in memory: the op byte comes from the global
//     array and the valid box is compared in registers.
#pragma once

#include "stream_kernels.cuh"

namespace culbm {

// Device-resident round state, so that one captured graph serves every round.
struct RoundState {
    int sel;        // double buffer: index of the buffer holding the newest state
    int src_offz;   // ring buffer: z offset of the current state
    int dst_offz;   // ring buffer: z offset the round writes to
    uint32_t step;  // time steps done before this round (seeds stochastic rounding)
};

template <typename S>
struct GlobalPops {
    S* base[2];          // buffer 0 and 1 (ring: base[0] only)
    long long stride;    // elements per direction (N, or nx*ny*ring_nz)
    int ring_nz;         // 0: plain double buffer
    int ring_step;       // ring: offset decrement per round
};

template <typename S, typename R>
struct TileArgs {
    Domain dom;
    int bx, by, bz, bxy;    // tile extent
    int ox, oy, oz;         // tile origin (global)
    int sx, sy, sz;         // origin of this launch's box inside the tile (tile coordinates)
    int vlo[3], vhi[3];     // valid box [vlo, vhi) (global)
    const uint8_t* ops;
    const float* rho;
    const float* vx;
    const float* vy;
    const float* vz;
    R inv_tau;
    GlobalPops<S> g;
    Pops<S> t0, t1;         // tile buffers (t1: pull ping-pong only)
    S* edge;                // domain-clamp side buffer (in-place tiles)
    EdgeLayout el;
    const RoundState* rs;
    int j;                  // step of the round this launch performs (0 = first)
};

template <typename S>
__device__ __forceinline__ long long gaddr(const GlobalPops<S>& g, const Domain& D, int offz, int x, int y, int z)
{
    int pz = z;
    if (g.ring_nz) {
        pz += offz;
        if (pz >= g.ring_nz) pz -= g.ring_nz;
    }
    return (long long)pz * D.nxy + (long long)y * D.nx + x;
}

// The tile steps work on raw values 2^E f (E = ScaleExp<S>; the scale is
// folded into the cell update, as in the plain steps), loaded with ld_raw
// and stored with put_raw / put27_raw: the same bits as loading f and
// storing it with put.
template <typename S, typename R, bool HINT>
__device__ __forceinline__ R gload(const S* p)
{
    if constexpr (HINT) {
        return ld_raw_cs<S, R>(p);
    } else {
        return ld_raw<S, R>(p);
    }
}

// Per-cell stochastic-rounding hash of the step this launch performs.
template <typename S, typename R>
__device__ __forceinline__ uint32_t tile_hash(const TileArgs<S, R>& a, int gi)
{
    return cell_hash(static_cast<uint32_t>(gi), step_seed(a.rs->step + static_cast<uint32_t>(a.j)));
}

struct TileCell {
    int px, py, pz, t;        // tile coordinates and tile index
    int gx, gy, gz, gi;       // global coordinates and index
    bool active;              // inside the tile launch and inside the domain
    bool correct;             // inside the valid box
};

template <typename S, typename R>
__device__ __forceinline__ TileCell tile_cell(const TileArgs<S, R>& a)
{
    TileCell c;
    c.px = a.sx + static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    c.py = a.sy + static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    c.pz = a.sz + static_cast<int>(blockIdx.z);
    c.t = c.px + a.bx * (c.py + a.by * c.pz);
    c.gx = a.ox + c.px;
    c.gy = a.oy + c.py;
    c.gz = a.oz + c.pz;
    c.active = c.px < a.bx && c.py < a.by && c.gx < a.dom.nx && c.gy < a.dom.ny && c.gz < a.dom.nz;
    c.gi = c.gx + a.dom.nx * (c.gy + a.dom.ny * c.gz);
    c.correct = c.gx >= a.vlo[0] && c.gx < a.vhi[0] && c.gy >= a.vlo[1] && c.gy < a.vhi[1] && c.gz >= a.vlo[2] &&
                c.gz < a.vhi[2];
    return c;
}

__device__ __forceinline__ bool in_tile(int px, int py, int pz, int bx, int by, int bz)
{
    return (unsigned)px < (unsigned)bx && (unsigned)py < (unsigned)by && (unsigned)pz < (unsigned)bz;
}

// Resident blocks per SM the tile step kernels are compiled for: four
// blocks of 256 (at most 64 registers; the first-step kernels spill 8-24
// bytes).  Left free, the first-step kernels took 75-80 registers (three
// blocks) and the 16-bit steps ran a quarter slower; five blocks (48
// registers) spill 36-140 bytes.
constexpr int kTileMinBlocks = 4;

// Programmatic dependent launch: the tile steps of a round are launched
// with programmatic stream serialisation, so the next step's blocks may start
// while this grid's last blocks run.  Each step lets its dependents start at
// once and waits for the previous grid (complete, its memory visible) before
// touching memory; the wait is the hardware's own and always ends.
__device__ __forceinline__ void tile_step_enter()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Pull of all 27 populations from the global state with the domain clamp.
template <typename S, typename R, bool HINT>
__device__ __forceinline__ void tile_pull_global(const TileArgs<S, R>& a, const TileCell& c, int sel, int offz, R* f)
{
    const Domain& D = a.dom;
    const S* base = a.g.base[sel];
    // the three clamped source columns, rows and planes (x - c for c = -1, 0, 1
    // at index 1 - c), the planes through the ring mapping when there is one
    const int xs[3] = {c.gx == 0 ? c.gx : c.gx - 1, c.gx, c.gx == D.nx - 1 ? c.gx : c.gx + 1};
    const int ys[3] = {(c.gy == 0 ? c.gy : c.gy - 1) * D.nx, c.gy * D.nx,
                       (c.gy == D.ny - 1 ? c.gy : c.gy + 1) * D.nx};
    const long long zs[3] = {gaddr(a.g, D, offz, 0, 0, c.gz == 0 ? c.gz : c.gz - 1), gaddr(a.g, D, offz, 0, 0, c.gz),
                             gaddr(a.g, D, offz, 0, 0, c.gz == D.nz - 1 ? c.gz : c.gz + 1)};
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = gload<S, R, HINT>(base + d * a.g.stride + zs[1 - cz_of(d)] + (ys[1 - cy_of(d)] + xs[1 - cx_of(d)]));
}

template <typename S, typename R, bool HINT>
__device__ __forceinline__ void tile_store_global(const TileArgs<S, R>& a, const TileCell& c, int sel, int offz,
                                                  const R* f)
{
    S* base = a.g.base[sel];
    const long long off = gaddr(a.g, a.dom, offz, c.gx, c.gy, c.gz);
    put27_raw<S, HINT>(f, tile_hash(a, c.gi), [&](int d) { return base + d * a.g.stride + off; });
}

// Selected buffers of the current round.
__device__ __forceinline__ int round_src_sel(const RoundState* rs, int ring) { return ring ? 0 : rs->sel; }
__device__ __forceinline__ int round_dst_sel(const RoundState* rs, int ring) { return ring ? 0 : 1 - rs->sel; }

// ----------------------------------------------------- in-place (AA) tiles ---

// Loads of an in-place tile step.  LAYOUT_AA_A: from x - c_d's reversed slot,
// clamped values from the edge buffer, 0 outside the tile.  LAYOUT_AA_B: own slots.
template <int LAYOUT, typename S, typename R>
__device__ __forceinline__ void tile_load_aa(const TileArgs<S, R>& a, const TileCell& c, bool edge, R* f)
{
    const Domain& D = a.dom;
    if (LAYOUT == LAYOUT_AA_B) {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = ld_raw<S, R>(a.t0.p[d] + c.t);
        return;
    }
    if (!edge) {
        // off the domain faces only the tile's own faces cut pulls off; the
        // masks are per lane (predicated loads), so warps do not diverge
        const bool lx = c.px > 0, hx = c.px < a.bx - 1, ly = c.py > 0, hy = c.py < a.by - 1, lz = c.pz > 0,
                   hz = c.pz < a.bz - 1;
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            const bool ok = (cx == 1 ? lx : cx == -1 ? hx : true) && (cy == 1 ? ly : cy == -1 ? hy : true) &&
                            (cz == 1 ? lz : cz == -1 ? hz : true);
            f[d] = ok ? ld_raw<S, R>(a.t0.p[26 - d] + (c.t - (cx + cy * a.bx + cz * a.bxy))) : R(0);
        }
        return;
    }
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
        if (!inside(D, c.gx - cx, c.gy - cy, c.gz - cz))
            f[d] = ld_raw<S, R>(a.edge + edge_slot(D, a.el, c.gx, c.gy, c.gz, d));
        else if (in_tile(c.px - cx, c.py - cy, c.pz - cz, a.bx, a.by, a.bz))
            f[d] = ld_raw<S, R>(a.t0.p[26 - d] + (c.t - (cx + cy * a.bx + cz * a.bxy)));
        else
            f[d] = R(0);
    }
}

// A boundary cell files its post-collision populations into the edge-buffer
// slots of the boundary cells whose clamped pull reads it (layout A start).
// Slots of readers outside the tile are written too; those readers are halo
// cells of this tile and their own tile rewrites the slots before use.
template <typename S, typename R>
__device__ __forceinline__ void tile_file_clamp_sources(const TileArgs<S, R>& a, const TileCell& c, const R* f)
{
    const uint32_t hc = tile_hash(a, c.gi);
    for_dirs([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        for_each_clamp_reader<d>(a.dom, c.gx, c.gy, c.gz, [&](int yx, int yy, int yz) {
            put_raw(a.edge + edge_slot(a.dom, a.el, yx, yy, yz, d), f[d], hc, d);
        });
    });
}

// First step: global pull -> tile (layout A), or -> global when I == 1.
template <typename S, typename R, bool ONE, bool HINT>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_aa_first(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active) return;
    const int ring = a.g.ring_nz;
    const uint8_t op = a.ops[c.gi];
    R f[27];
    if (op & OP_LOAD) {
        tile_pull_global<S, R, HINT>(a, c, round_src_sel(a.rs, ring), a.rs->src_offz, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (!(op & OP_STORE)) return;
    if constexpr (ONE) {
        if (c.correct) tile_store_global<S, R, HINT>(a, c, round_dst_sel(a.rs, ring), a.rs->dst_offz, f);
    } else {
#pragma unroll
        put27_raw<S>(f, tile_hash(a, c.gi), [&](int d) { return a.t0.p[26 - d] + c.t; });
        if (op & OP_EDGE) tile_file_clamp_sources(a, c, f);
    }
}

// Middle odd step inside the tile (layout A -> B).
template <typename S, typename R>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_aa_odd(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active) return;
    const Domain& D = a.dom;
    const uint8_t op = a.ops[c.gi];
    const bool edge = (op & OP_EDGE) != 0;
    R f[27];
    if (op & OP_LOAD) {
        tile_load_aa<LAYOUT_AA_A>(a, c, edge, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (!(op & OP_STORE)) return;
    if (!edge) {
        // off the domain faces a push only has to stay inside the tile
        // (predicated stores, no divergence)
        const bool lx = c.px > 0, hx = c.px < a.bx - 1, ly = c.py > 0, hy = c.py < a.by - 1, lz = c.pz > 0,
                   hz = c.pz < a.bz - 1;
        const uint32_t hc = tile_hash(a, c.gi);
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            const bool ok = (cx == 1 ? hx : cx == -1 ? lx : true) && (cy == 1 ? hy : cy == -1 ? ly : true) &&
                            (cz == 1 ? hz : cz == -1 ? lz : true);
            if (ok) put_raw(a.t0.p[d] + (c.t + cx + cy * a.bx + cz * a.bxy), f[d], hc, d);
        }
        return;
    }
    for_dirs([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        constexpr int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
        if (inside(D, c.gx + cx, c.gy + cy, c.gz + cz) && in_tile(c.px + cx, c.py + cy, c.pz + cz, a.bx, a.by, a.bz))
            put_raw(a.t0.p[d] + (c.t + cx + cy * a.bx + cz * a.bxy), f[d], tile_hash(a, c.gi), d);
        if (edge) {
            // slot d of each boundary cell whose clamped pull reads this cell
            for_each_clamp_reader<d>(D, c.gx, c.gy, c.gz, [&](int yx, int yy, int yz) {
                const int qx = yx - a.ox, qy = yy - a.oy, qz = yz - a.oz;
                if (in_tile(qx, qy, qz, a.bx, a.by, a.bz))
                    put_raw(a.t0.p[d] + (qx + a.bx * (qy + a.by * qz)), f[d], tile_hash(a, c.gi), d);
            });
        }
    });
}

// Middle even step inside the tile (layout B -> A).
template <typename S, typename R>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_aa_even(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active) return;
    const uint8_t op = a.ops[c.gi];
    R f[27];
    if (op & OP_LOAD) {
        tile_load_aa<LAYOUT_AA_B>(a, c, false, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (!(op & OP_STORE)) return;
    put27_raw<S>(f, tile_hash(a, c.gi), [&](int d) { return a.t0.p[26 - d] + c.t; });
    if (op & OP_EDGE) tile_file_clamp_sources(a, c, f);
}

// Last step: tile (layout A or B) -> global result, valid cells only.
template <int LAYOUT, typename S, typename R, bool HINT>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_aa_last(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active || !c.correct) return;
    const uint8_t op = a.ops[c.gi];
    R f[27];
    if (op & OP_LOAD) {
        tile_load_aa<LAYOUT>(a, c, (op & OP_EDGE) != 0, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (op & OP_STORE) tile_store_global<S, R, HINT>(a, c, round_dst_sel(a.rs, a.g.ring_nz), a.rs->dst_offz, f);
}

// ------------------------------------------------------ pull (ping-pong) ---

// Pull inside the tile from buffer `src`: domain clamp reads the own slot,
// sources outside the tile read 0 (halo).
template <typename S, typename R>
__device__ __forceinline__ void tile_pull(const TileArgs<S, R>& a, const Pops<S>& src, const TileCell& c, bool edge,
                                          R* f)
{
    if (!edge) {
        // off the domain faces only the tile's own faces cut pulls off
        // (per-lane predicated loads, no divergence)
        const bool lx = c.px > 0, hx = c.px < a.bx - 1, ly = c.py > 0, hy = c.py < a.by - 1, lz = c.pz > 0,
                   hz = c.pz < a.bz - 1;
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
            const bool ok = (cx == 1 ? lx : cx == -1 ? hx : true) && (cy == 1 ? ly : cy == -1 ? hy : true) &&
                            (cz == 1 ? lz : cz == -1 ? hz : true);
            f[d] = ok ? ld_raw<S, R>(src.p[d] + (c.t - (cx + cy * a.bx + cz * a.bxy))) : R(0);
        }
        return;
    }
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        int cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
        if ((unsigned)(c.gx - cx) >= (unsigned)a.dom.nx) cx = 0;
        if ((unsigned)(c.gy - cy) >= (unsigned)a.dom.ny) cy = 0;
        if ((unsigned)(c.gz - cz) >= (unsigned)a.dom.nz) cz = 0;
        if (in_tile(c.px - cx, c.py - cy, c.pz - cz, a.bx, a.by, a.bz))
            f[d] = ld_raw<S, R>(src.p[d] + (c.t - (cx + cy * a.bx + cz * a.bxy)));
        else
            f[d] = R(0);
    }
}

template <typename S, typename R, bool ONE, bool HINT>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_pull_first(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active) return;
    const int ring = a.g.ring_nz;
    const uint8_t op = a.ops[c.gi];
    R f[27];
    if (op & OP_LOAD) {
        tile_pull_global<S, R, HINT>(a, c, round_src_sel(a.rs, ring), a.rs->src_offz, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (!(op & OP_STORE)) return;
    if constexpr (ONE) {
        if (c.correct) tile_store_global<S, R, HINT>(a, c, round_dst_sel(a.rs, ring), a.rs->dst_offz, f);
    } else {
        put27_raw<S>(f, tile_hash(a, c.gi), [&](int d) { return a.t0.p[d] + c.t; });
    }
}

// Middle step t0 -> t1 (the host swaps t0/t1 between launches).
template <typename S, typename R>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_pull_mid(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active) return;
    const uint8_t op = a.ops[c.gi];
    R f[27];
    if (op & OP_LOAD) {
        tile_pull(a, a.t0, c, (op & OP_EDGE) != 0, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (!(op & OP_STORE)) return;
    put27_raw<S>(f, tile_hash(a, c.gi), [&](int d) { return a.t1.p[d] + c.t; });
}

template <typename S, typename R, bool HINT>
__global__ void __launch_bounds__(256, kTileMinBlocks) k_tile_pull_last(const __grid_constant__ TileArgs<S, R> a)
{
    tile_step_enter();
    const TileCell c = tile_cell(a);
    if (!c.active || !c.correct) return;
    const uint8_t op = a.ops[c.gi];
    R f[27];
    if (op & OP_LOAD) {
        tile_pull(a, a.t0, c, (op & OP_EDGE) != 0, f);
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, c.gi, f);
    if (op & OP_STORE) tile_store_global<S, R, HINT>(a, c, round_dst_sel(a.rs, a.g.ring_nz), a.rs->dst_offz, f);
}

// Advances the round state after all tiles of a round.
__global__ void k_tile_advance(RoundState* rs, int ring_nz, int ring_step, int steps)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        rs->step += static_cast<uint32_t>(steps);
        if (ring_nz) {
            rs->src_offz = rs->dst_offz;
            int o = rs->dst_offz - ring_step;
            if (o < 0) o += ring_nz;
            rs->dst_offz = o;
        } else {
            rs->sel = 1 - rs->sel;
        }
    }
}

}  // namespace culbm
