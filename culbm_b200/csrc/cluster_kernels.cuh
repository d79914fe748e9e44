// optPolicy 2 (L1/L2 mixed blocking) with pull streaming: one thread-block
// cluster per tile, the populations of every cell held in registers across
// the innerLoop steps of a round, and streaming between the cells of a tile
// through shared memory -- the CTA's own and, across CTA faces, the other
// CTAs' through distributed shared memory (DSMEM).
//
// The reference's HaloBlockingL1L2D3Q27PullKernel
// (src/simulator/single_dev_expt/kernel.cu:138-329, streaming in
// L1L2StreamCore.cuh:45-690) runs one tile per cooperative launch over the
// whole GPU: registers per cell, shared memory inside a CTA, warp shuffles
// for +-x, an L2 swap buffer for CTA faces and a grid-wide barrier per step.
// Here a tile is small enough for one cluster (at most 16 CTAs of 512
// threads, one thread per cell), so:
//   * the CTA-face exchange goes through DSMEM instead of an L2 buffer, and
//     the per-step barrier is the cluster's hardware barrier instead of a
//     grid-wide one (no spin-wait of our own);
//   * every tile of a round runs in ONE launch (a grid of clusters), so no
//     tile waits for another and the SMs stay busy across tiles;
//   * the geometry (tile extent, halo innerLoop-1, valid boxes from
//     calcValidPrev, blocking_alogrithm.hpp:7-41) is the reference's, as in
//     the L2 tile engine, and the results are the plain pull step's bit for
//     bit (per-axis domain clamp; pulls from outside the tile read 0 and only
//     reach cells outside the valid box).
#pragma once

#include <cooperative_groups.h>
#include <cstring>

#include "tile_kernels.cuh"

namespace culbm {

namespace cg = cooperative_groups;

// Most CTAs in one cluster (B200 allows 16 with the non-portable attribute).
constexpr int kClusterMaxCtas = 16;
// Most threads (cells) per CTA.  The kernel needs 128 registers per thread
// to keep 27 populations, the exchange and the cell update free of spills;
// capped at 64 (1024-thread CTAs) it spilled about 200 bytes per thread, and
// the spill stores went out to L2 and stalled every cluster barrier's release
// fence (ncu: 22.8M local store sectors per launch, membar and barrier the
// top stall reasons, 6.8k MLUPS).
constexpr int kClusterMaxThreads = 512;

template <typename S, typename R>
struct ClusterTileArgs {
    Domain dom;
    int B[3];          // tile extent (cells)
    int nt[3];         // tiles per axis
    int I;             // innerLoop of the geometry (halo depth I - 1)
    int k;             // steps of this round (1..I)
    int cdim[3];       // CTAs per tile per axis (the cluster's shape)
    const uint8_t* ops;
    const float* rho;
    const float* vx;
    const float* vy;
    const float* vz;
    R inv_tau;
    GlobalPops<S> g;   // double-buffered global state (no ring buffer)
    const RoundState* rs;
};

// Warp shuffle of a stored population (any storage format) from the lane
// `delta` below (UP) or above this one.
template <bool UP, typename S>
__device__ __forceinline__ S shfl_pop(S v, int delta)
{
    if constexpr (sizeof(S) == 2) {
        unsigned short b;
        memcpy(&b, &v, 2);
        unsigned w = b;
        w = UP ? __shfl_up_sync(0xFFFFFFFFu, w, delta) : __shfl_down_sync(0xFFFFFFFFu, w, delta);
        b = static_cast<unsigned short>(w);
        S r;
        memcpy(&r, &b, 2);
        return r;
    } else {
        return UP ? __shfl_up_sync(0xFFFFFFFFu, v, delta) : __shfl_down_sync(0xFFFFFFFFu, v, delta);
    }
}

// First valid index of tile `idx` along one axis: calcValidPrev
// (blocking_alogrithm.hpp:34-41), as valid_prev in tile_runtime.cu.
__device__ __forceinline__ int cluster_valid_start(int idx, int blk, int num, int it, int dom)
{
    if (idx == num) return dom;
    if (idx == 0) return 0;
    return (blk + 1 - it) + (idx - 1) * (blk + 2 - 2 * it);
}

// The round's k steps over one tile per cluster.  Shared memory: two slots
// of 27 directions x (threads of the CTA) populations in storage format S,
// one per exchange, alternating; one cluster barrier per exchange.  A slot is
// rewritten two exchanges later, after the barrier of the exchange between,
// which every thread of the cluster reaches only once it has read the slot.
// (Three barriers per exchange, over groups of 9 directions in smaller
// slots, measured slower.)
template <typename S, typename R, bool HINT>
__global__ void __launch_bounds__(kClusterMaxThreads, 1) k_tile_cluster_pull(const __grid_constant__ ClusterTileArgs<S, R> a)
{
    extern __shared__ __align__(16) unsigned char cluster_smem[];
    S* slots = reinterpret_cast<S*>(cluster_smem);
    cg::cluster_group cl = cg::this_cluster();

    const Domain& D = a.dom;
    const int nthr = static_cast<int>(blockDim.x * blockDim.y * blockDim.z);
    const int lt = static_cast<int>(threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z));
    const int bdim[3] = {static_cast<int>(blockDim.x), static_cast<int>(blockDim.y), static_cast<int>(blockDim.z)};
    const int bidx[3] = {static_cast<int>(blockIdx.x), static_cast<int>(blockIdx.y), static_cast<int>(blockIdx.z)};
    const int tidx[3] = {static_cast<int>(threadIdx.x), static_cast<int>(threadIdx.y), static_cast<int>(threadIdx.z)};
    const int dn[3] = {D.nx, D.ny, D.nz};

    // this thread's cell: tile coordinates p, global coordinates gc
    int p[3], gc[3];
    bool active = true, correct = true;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int kt = bidx[q] / a.cdim[q];
        p[q] = (bidx[q] - kt * a.cdim[q]) * bdim[q] + tidx[q];
        const int vlo = cluster_valid_start(kt, a.B[q], a.nt[q], a.I, dn[q]);
        const int vhi = cluster_valid_start(kt + 1, a.B[q], a.nt[q], a.I, dn[q]);
        gc[q] = max(vlo - (a.I - 1), 0) + p[q];
        active = active && p[q] < a.B[q] && gc[q] < dn[q];
        correct = correct && gc[q] >= vlo && gc[q] < vhi;
    }
    const int gi = active ? gc[0] + D.nx * (gc[1] + D.ny * gc[2]) : 0;
    const uint8_t op = active ? a.ops[gi] : uint8_t(0);
    const int sel_src = a.rs->sel, sel_dst = 1 - a.rs->sel;
    const uint32_t step0 = a.rs->step;

    R f[27];
    if (op & OP_LOAD) {
        // first step: pull from the global state with the domain clamp
        const S* base = a.g.base[sel_src];
        const int xs[3] = {gc[0] == 0 ? gc[0] : gc[0] - 1, gc[0], gc[0] == D.nx - 1 ? gc[0] : gc[0] + 1};
        const int ys[3] = {(gc[1] == 0 ? gc[1] : gc[1] - 1) * D.nx, gc[1] * D.nx,
                           (gc[1] == D.ny - 1 ? gc[1] : gc[1] + 1) * D.nx};
        const long long zs[3] = {(long long)(gc[2] == 0 ? gc[2] : gc[2] - 1) * D.nxy, (long long)gc[2] * D.nxy,
                                 (long long)(gc[2] == D.nz - 1 ? gc[2] : gc[2] + 1) * D.nxy};
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = gload<S, R, HINT>(base + d * a.g.stride + zs[1 - cz_of(d)] + (ys[1 - cy_of(d)] + xs[1 - cx_of(d)]));
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) f[d] = R(0);
    }
    cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, gi, f);

    // Where the pull of this cell reads, per axis, for the source offsets
    // c = +1 and -1 (source p - c, or p where the domain clamp applies): the
    // step of the source's CTA rank and of its cell index inside that CTA,
    // relative to this cell and packed as (rank step << 16) + index step, and
    // whether the source lies in the tile.  A direction's source is this
    // cell's packed (rank, index) plus the sum over its axes; rank steps and
    // index steps may be negative, the resulting index lies in [0, 512).
    const int me = static_cast<int>(cl.block_rank());
    int dl[3][2];           // [axis][c == -1]
    unsigned inmask = 0;    // bit 3*axis + (1 - c): the source lies in the tile
    {
        const int rstride[3] = {1, a.cdim[0], a.cdim[0] * a.cdim[1]};
        const int lstride[3] = {1, bdim[0], bdim[0] * bdim[1]};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            inmask |= 1u << (3 * ax + 1);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                int c = j == 0 ? 1 : -1;
                if ((unsigned)(gc[ax] - c) >= (unsigned)dn[ax]) c = 0;   // domain clamp
                const int t = tidx[ax] - c;
                const int step = t < 0 ? -1 : (t >= bdim[ax] ? 1 : 0);
                dl[ax][j] = step * rstride[ax] * 65536 + (step * -bdim[ax] - c) * lstride[ax];
                if ((unsigned)(p[ax] - c) < (unsigned)a.B[ax]) inmask |= 1u << (3 * ax + (j == 0 ? 0 : 2));
            }
        }
    }
    const int own = me * 65536 + lt;
    // warp shuffles for d = 14 / 12: a warp is one row of the CTA, and the
    // source (x - 1 / x + 1, unclamped) is in the same warp
    const bool row_warp = bdim[0] == 32;
    const bool xlo_shfl = tidx[0] > 0 && gc[0] > 0;
    const bool xhi_shfl = tidx[0] < 31 && gc[0] < D.nx - 1;
    for (int m = 1; m < a.k; ++m) {
        // post-collision populations of step m - 1 in storage format S
        // (the same rounding as a stored step, stochastic bits included)
        S q[27];
        put27_raw<S>(f, cell_hash(static_cast<uint32_t>(gi), step_seed(step0 + static_cast<uint32_t>(m - 1))),
                     [&](int d) { return &q[d]; });
        // The pure +-x directions (d = 14: source x - 1; d = 12: source x + 1)
        // come from the neighbouring lane by a warp shuffle where a warp is
        // one 32-cell row of the CTA and the source lane lies in the warp (the
        // reference's L1/L2 kernel shuffles the same two directions); their
        // edge lanes and clamped cells read shared memory like the rest.  The
        // shuffle runs only where every warp is a full row (a CTA-uniform
        // test), so no partial warp executes the full-mask shuffle.
        S from_lo = q[14], from_hi = q[12];
        if (row_warp) {
            from_lo = shfl_pop<true>(q[14], 1);
            from_hi = shfl_pop<false>(q[12], 1);
        }
        S* slot = slots + (m & 1) * 27 * nthr;
#pragma unroll
        for (int d = 0; d < 27; ++d) slot[d * nthr + lt] = q[d];
        cl.sync();   // barrier.cluster arrive (release) + wait (acquire)
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int jx = 1 - cx_of(d), jy = 1 - cy_of(d), jz = 1 - cz_of(d);
            const unsigned need = (1u << jx) | (1u << (3 + jy)) | (1u << (6 + jz));
            R v = R(0);
            if ((d == 12 || d == 14) && row_warp && (op & OP_LOAD) && (inmask & need) == need &&
                (d == 14 ? xlo_shfl : xhi_shfl)) {
                const S w = d == 14 ? from_lo : from_hi;
                v = ld_raw<S, R>(&w);
            } else if ((op & OP_LOAD) && (inmask & need) == need) {
                int packed = own;
                if (jx != 1) packed += dl[0][jx >> 1];
                if (jy != 1) packed += dl[1][jy >> 1];
                if (jz != 1) packed += dl[2][jz >> 1];
                const int r = packed >> 16;
                // own CTA: plain shared-memory load; another CTA: DSMEM
                const S* src = slot + d * nthr + (packed & 0xFFFF);
                v = r == me ? ld_raw<S, R>(src) : ld_raw<S, R>(cl.map_shared_rank(src, r));
            }
            f[d] = v;
        }
        cell_update_for<S, true>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, gi, f);
    }

    if (active && correct && (op & OP_STORE)) {
        S* base = a.g.base[sel_dst];
        const long long off = gi;
        put27_raw<S>(f, cell_hash(static_cast<uint32_t>(gi), step_seed(step0 + static_cast<uint32_t>(a.k - 1))),
                     [&](int d) { return base + d * a.g.stride + off; });
    }
    // no CTA leaves while another may still read its shared memory
    if (a.k > 1) cl.sync();
}

}  // namespace culbm
