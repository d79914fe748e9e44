// Warp-staged pull step for the 16-bit population formats, with TMA tensor
// copies.
//
// The population buffer is described to the TMA unit as a 4-D tensor
// (x, y, z, d) of 16-bit values.  Each warp walks over 32-cell segments of
// x-rows on its own (no block-level synchronisation).  For a segment
// [x0, x0 + 32) of row (y, z) lanes 0..8 issue one tensor load each
// (cp.async.bulk.tensor): lane k = (cy + 1) + 3 (cz + 1) copies a 48 x 3 box,
// the windows of the three directions d = 3k, 3k + 1, 3k + 2 (cx = -1, 0, +1),
// which share the source row (clamp(y - cy), clamp(z - cz)) of the
// reference's per-axis clamp (kernel.cu:2506-2511), into the warp's shared
// memory, completing on the warp's mbarrier.  Each lane then reads its cell's
// 27 populations from shared memory at fixed offsets (x, x - 1 or x + 1, the x
// clamp in the element index), applies the cell update, writes its 27
// results into the warp's 27 x 32 output box, and lane 0 writes the box to the
// destination with one tensor store (values past nx are not written).  NB
// window buffers per warp keep the copies of the next NB - 1 segments in
// flight while a segment is computed.
//
// Requirements (checked on the host): 16-bit storage and nx a multiple of 8
// (16-byte aligned tensor rows and x coordinates).  Cells without STORE keep
// the destination's old bits.  Every mbarrier wait is bounded
// (kWarpWaitLimitNs of %globaltimer); on expiry the warp records
// CULBM_ERR_DEVICE_TIMEOUT in the error word, lets its copies land and stops.
#pragma once

#include <cuda.h>

#include <cstdint>
#include <type_traits>

#include "culbm.h"
#include "row_kernels.cuh"
#include "stream_kernels.cuh"

namespace culbm {

constexpr int kWarpWin = 48;      // window values per direction: x0 - 8 .. x0 + 40 (16-byte aligned)
constexpr int kWarpWarps = 8;     // warps per block
constexpr int kWarpBoxPitch = 384;                     // slot of one tensor load (3 x 48 values, 288 B), 128-byte aligned
constexpr int kWarpWinBytes = 9 * kWarpBoxPitch;       // one window buffer (27 directions)
constexpr int kWarpOutPitch = 1792;                    // output box 27 x 32 values (1728 B), 128-byte aligned
constexpr unsigned long long kWarpWaitLimitNs = 1000000000ull;

// Bytes of shared memory per warp with NB window buffers (the mbarriers in
// the last 128 bytes).
__host__ __device__ constexpr int warp_smem_per_warp(int nb) { return nb * kWarpWinBytes + kWarpOutPitch + 128; }

struct WarpArgs16 {
    int nseg_row;      // segments per row: ceil(nx / 32)
    int nseg;          // segments of the domain: nseg_row * ny * nz
    int* err;          // error word (mapped host memory)
    int debug_extra_tx;
};

// The tensor maps of a step: window loads from the source buffer (box 48 x 1
// x 1 x 3) and the output store to the destination buffer (box 32 x 1 x 1 x 27).
struct WarpMaps {
    CUtensorMap src;
    CUtensorMap dst;
};

// First value of the window of a segment starting at x0 (whole rows when nx <= 48).
__host__ __device__ __forceinline__ int warp_window_start(int x0, int nx)
{
    return nx <= kWarpWin ? 0 : (x0 - 8 < 0 ? 0 : (x0 - 8 > nx - kWarpWin ? nx - kWarpWin : x0 - 8));
}

// Lanes 0..8 load the 27 windows of the segment (x0, y, z) into window
// buffer `wbuf`; lane 0 first announces the byte count.
__device__ __forceinline__ void warp_issue_windows(const CUtensorMap* map, const Domain& D, const WarpArgs16& w,
                                                   uint32_t wbuf, uint64_t* bar, int x0, int y, int z, int lane)
{
    const int ws = warp_window_start(x0, D.nx);
    // every box is 3 x 48 values, zero-filled past nx on rows narrower than 48
    if (lane == 0) mbar_arrive_expect_tx(bar, 9u * 3u * 2u * kWarpWin + static_cast<uint32_t>(w.debug_extra_tx));
    __syncwarp();
    if (lane < 9) {
        const int cy = lane % 3 - 1, cz = lane / 3 - 1;
        int sy = y - cy, sz = z - cz;
        if ((unsigned)sy >= (unsigned)D.ny) sy = y;
        if ((unsigned)sz >= (unsigned)D.nz) sz = z;
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(wbuf + static_cast<uint32_t>(lane * kWarpBoxPitch)),
            "l"(map), "r"(ws), "r"(sy), "r"(sz), "r"(3 * lane), "r"(smem_addr(bar))
            : "memory");
    }
}

// Waits for the phase of `bar` with parity `parity`, at most kWarpWaitLimitNs.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kWarpWaitLimitNs) return false;
    }
}

template <typename S, int NB>
__global__ void __launch_bounds__(kWarpWarps * 32, NB == 2 ? 4 : 3) k_pull16_warp(const __grid_constant__ StepArgs<S, float> a,
                                                                 const __grid_constant__ WarpMaps maps,
                                                                 const WarpArgs16 w)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const Domain& D = a.dom;
    const int nx = D.nx;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* mine = smem + warp * warp_smem_per_warp(NB);
    const uint32_t win0 = smem_addr(mine), outb = win0 + NB * kWarpWinBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(mine + NB * kWarpWinBytes + kWarpOutPitch);
    const int gw = static_cast<int>(blockIdx.x) * kWarpWarps + warp;
    const int W = static_cast<int>(gridDim.x) * kWarpWarps;
    if (gw >= w.nseg) return;

    if (lane == 0) {
        for (int b = 0; b < NB; ++b) mbar_init(bars + b, 1);
        mbar_init_fence();
    }
    __syncwarp();

    // Segment s = seg + nseg_row * (y + ny * z); the walk over s, s + W, ...
    // advances (seg, y, z) without dividing per segment.
    struct SegWalk {
        int seg, y, z, dseg, dy, dz, nsr, ny;
        __device__ __forceinline__ void advance()
        {
            seg += dseg;
            int carry = 0;
            if (seg >= nsr) {
                seg -= nsr;
                carry = 1;
            }
            y += dy + carry;
            if (y >= ny) {
                y -= ny;
                z += 1;
            }
            z += dz;
        }
    };
    SegWalk cur;
    cur.nsr = w.nseg_row;
    cur.ny = D.ny;
    {
        const int row = gw / w.nseg_row;
        cur.seg = gw - row * w.nseg_row;
        cur.y = row % D.ny;
        cur.z = row / D.ny;
        const int drow = W / w.nseg_row;
        cur.dseg = W - drow * w.nseg_row;
        cur.dy = drow % D.ny;
        cur.dz = drow / D.ny;
    }
    // stage the first NB - 1 segments
    SegWalk ahead = cur;
    int sa = gw;
    for (int b = 0; b < NB - 1; ++b) {
        if (sa < w.nseg)
            warp_issue_windows(&maps.src, D, w, win0 + b * kWarpWinBytes, bars + b, ahead.seg * 32, ahead.y, ahead.z,
                               lane);
        sa += W;
        ahead.advance();
    }
    constexpr int E = ScaleExp<S>::value;
    bool ok = true;
    int k = 0;
    for (int s = gw; s < w.nseg; s += W, ++k, cur.advance()) {
        const int b = k % NB;
        // stage segment k + NB - 1 into the buffer read in iteration k - 1
        // (every lane's reads of it preceded that iteration's last __syncwarp)
        if (sa < w.nseg) {
            const int bn = (k + NB - 1) % NB;
            warp_issue_windows(&maps.src, D, w, win0 + bn * kWarpWinBytes, bars + bn, ahead.seg * 32, ahead.y,
                               ahead.z, lane);
        }
        sa += W;
        ahead.advance();
        // the op byte of this segment's cell, read before waiting for its windows
        const int x0p = cur.seg * 32 + lane;
        const int ip = (x0p < nx ? x0p : nx - 1) + nx * (cur.y + D.ny * cur.z);
        const uint8_t op_pre = a.ops[ip];
        if (!__all_sync(0xffffffffu, warp_wait(bars + b, static_cast<uint32_t>(k / NB) & 1u))) {
            ok = false;
            break;
        }
        const int x0 = cur.seg * 32, y = cur.y, z = cur.z;
        const int x = x0 + lane;
        const bool cell = x < nx;
        const int xc = cell ? x : nx - 1;
        const int ws = warp_window_start(x0, nx);
        const uint32_t wb = win0 + b * kWarpWinBytes;
        // the window element of cell x for cx = 0, +1 (x - 1), -1 (x + 1), clamped at the x faces
        const uint32_t e0 = wb + 2u * static_cast<uint32_t>(xc - ws);
        const uint32_t em = wb + 2u * static_cast<uint32_t>((xc > 0 ? xc - 1 : xc) - ws);
        const uint32_t ep = wb + 2u * static_cast<uint32_t>((xc < nx - 1 ? xc + 1 : xc) - ws);
        const int i = xc + nx * (y + D.ny * z);
        const uint8_t op = cell ? op_pre : uint8_t(0);
        float f[27];
        if (op & OP_LOAD) {
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const int cx = cx_of(d);
                const uint32_t base = cx == 1 ? em : cx == -1 ? ep : e0;
                // direction d = 3 k + j sits in box k, row j
                const uint32_t off = static_cast<uint32_t>((d / 3) * kWarpBoxPitch + (d % 3) * kWarpWin * 2);
                unsigned short v;
                asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(base + off));
                f[d] = raw16_to_float<S>(v);
            }
        } else {
#pragma unroll
            for (int d = 0; d < 27; ++d) f[d] = 0.0f;
        }
        const uint32_t hc = cell_hash(static_cast<uint32_t>(i), a.seed);
        cell_update_fast<E>(op, a.inv_tau, a.rho, a.vx, a.vy, a.vz, i, f);
        // the previous segment's store has read the output box
        if (lane == 0) bulk_wait_read_all();
        __syncwarp();
        const uint32_t ob = outb + 2u * static_cast<uint32_t>(lane);
        if (op & OP_STORE) {
#pragma unroll
            for (int k2 = 0; k2 < 13; ++k2) {
                const uint32_t wd = Pack2<S>::cvt(f[26 - k2], f[k2], IsSR<S>::value ? sr_word_pair(hc, k2) : 0u);
                sts16(ob + static_cast<uint32_t>(k2 * 64), static_cast<unsigned short>(wd));
                sts16(ob + static_cast<uint32_t>((26 - k2) * 64), static_cast<unsigned short>(wd >> 16));
            }
            sts16(ob + 13u * 64u, enc16_raw<S>(f[13], hc, 13));
        } else if (cell) {
            // no STORE: the destination keeps its bits
#pragma unroll
            for (int d = 0; d < 27; ++d)
                sts16(ob + static_cast<uint32_t>(d * 64), reinterpret_cast<const unsigned short*>(a.dst.p[d])[i]);
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
            asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                             &maps.dst),
                         "r"(x0), "r"(y), "r"(z), "r"(0), "r"(outb)
                         : "memory");
            bulk_commit();
        }
    }
    if (!ok) {
        if (lane == 0) atomicExch_system(w.err, static_cast<int>(CULBM_ERR_DEVICE_TIMEOUT));
        // let the windows of this and the later staged segments land (each wait bounded)
        for (int j = k; j < k + NB; ++j)
            if (gw + j * W < w.nseg) warp_wait(bars + j % NB, static_cast<uint32_t>(j / NB) & 1u);
    }
    if (lane == 0) bulk_wait_all();
}

}  // namespace culbm
