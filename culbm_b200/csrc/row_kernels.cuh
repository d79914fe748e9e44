// Row-staged step kernels for the 16-bit population formats (pull and the
// two in-place steps).
//
// One thread block owns one x-row (y, z) of the domain at a time, one
// consumer thread per cell of the row, and walks over rows with a stride of
// the grid size.  A producer warp stages, in shared memory, the 27 whole
// x-rows of the population planes that a row reads (one bulk asynchronous
// copy, cp.async.bulk, per plane row, completing on the stage's "full"
// mbarrier) plus the row's op bytes, up to STAGES rows ahead.  The consumer
// warps read their 27 populations from shared memory at x, x - 1 or x + 1,
// release the stage (its "empty" mbarrier), write their 27 results into a
// shared output row per plane and signal it ("ofull"); the producer writes
// those 27 rows back with one bulk store each and hands the output buffer
// back ("oempty") once the store has read it.  Consumer warps never wait for
// each other, only for data and buffers.  Per population this replaces a
// global address computation, a 2-byte global load and a 2-byte global store
// by two shared-memory accesses; the global traffic is whole 16-byte aligned
// rows.
//
// Rows and planes (x fastest, cell i = x + nx (y + ny z)):
//   pull      window d = plane d of the source buffer at row
//             (clamp(y - cy), clamp(z - cz)), read at clamp(x - cx): the
//             reference's per-axis clamp (kernel.cu:2506-2511) with the y and z
//             parts in the row choice and the x part in the element index.
//             Output d = plane d of the destination buffer at row (y, z).
//   AA even   window d = plane d at row (y, z), read at x; output 26 - d at
//             row (y, z) (the reversed own slots).
//   AA odd    window d = plane 26 - d at row (y - cy, z - cz), read at x - cx;
//             output d = plane d at row (y + cy, z + cz), written at x + cx.
//             The rows an in-place step reads are exactly the rows it writes
//             (plane d at row (y + cy, z + cz) is window 26 - d), and the row
//             sets of different rows are disjoint, so whole-row stores race
//             with nothing.
// The in-place kernels cover the inner rows (0 < y < ny-1, 0 < z < nz-1);
// the face rows keep the per-cell kernels (stream_kernels.cuh), whose clamp
// slots live in the edge buffer.  At the x faces of inner rows the odd step
// reads its clamped populations from the edge buffer and writes each face
// cell's clamp slot (its own x in the pushed row); the even step files the
// face cells' clamp sources into the edge buffer, as the per-cell kernels do.
//
// Requirements (checked on the host): 16-bit storage, nx a multiple of 16
// (16-byte aligned rows for the bulk copies), nx <= 992 (one block of nx
// consumer threads and a producer warp per row).
// Cells without STORE keep their stored bits: their output slots are filled
// with the bits just read (in place) or the destination's old bits (pull).
//
// Every mbarrier wait is bounded (kRowWaitLimitNs of %globaltimer).  On
// expiry the warp raises the block's abort flag and records
// CULBM_ERR_DEVICE_TIMEOUT in the error word; every warp then leaves its
// loop, the producer lets its bulk copies land, and the host reports the
// status at its next synchronisation.
#pragma once

#include <cstdint>
#include <type_traits>

#include "culbm.h"
#include "stream_kernels.cuh"

namespace culbm {

enum RowMode : int { ROWS_PULL = 0, ROWS_AA_ODD = 1, ROWS_AA_EVEN = 2 };

constexpr int kRowStages = 2;                                  // row windows in flight per block
constexpr unsigned long long kRowWaitLimitNs = 1000000000ull;  // 1 s

template <typename S>
struct RowArgs {
    StepArgs<S, float> s;   // domain, op bytes, EQU inputs, invTau, planes, edge buffer, SR seed
    int y0, z0;             // first row of the covered box
    int ry, rz;             // rows of the box in y and z (row q: y = y0 + q % ry, z = z0 + q / ry)
    int nrows;              // ry * rz
    int* err;               // error word (mapped host memory), 0 while no wait expired
    int debug_extra_tx;     // > 0: expect that many bytes more than arrive (tests of the bounded wait)
};

// Shared-memory layout of a block (byte offsets; every part 128-byte aligned).
struct RowSmem {
    int bars;       // mbarriers: full[STAGES], empty[STAGES], ofull[OUTB], oempty[OUTB]; then the abort flag
    int win;        // STAGES x 27 plane rows of nx values
    int ops;        // STAGES x nx op bytes
    int out;        // OUTB x 27 plane rows of nx values (output buffers)
    int stage_bytes;
    int total;
};

__host__ __device__ constexpr int align128(int v) { return (v + 127) & ~127; }

template <typename S, int STAGES, int OUTB>
__host__ __device__ inline RowSmem row_smem_layout(int nx)
{
    RowSmem L{};
    const int plane_row = nx * static_cast<int>(sizeof(S));
    L.bars = 0;
    L.win = align128((2 * STAGES + 4) * 8 + 8);
    L.stage_bytes = 27 * plane_row;
    L.ops = L.win + align128(STAGES * 27 * plane_row);
    L.out = L.ops + align128(STAGES * nx);
    L.total = L.out + align128(OUTB * 27 * plane_row);
    return L;
}

// Consumer warps of a row of nx cells; the producer is the warp after them.
__host__ __device__ constexpr int row_consumer_warps(int nx) { return (nx + 31) / 32; }

// ---- PTX helpers (sm_90+ bulk asynchronous copies and mbarriers) ----------

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-bit shared-memory store at a 32-bit shared address.
__device__ __forceinline__ void sts16(uint32_t addr, unsigned short v)
{
    asm volatile("st.shared.u16 [%0], %1;" ::"r"(addr), "h"(v));
}

// Raw value 2^E f of a stored 16-bit pattern (the ld_raw of storage.cuh).
template <typename S>
__device__ __forceinline__ float raw16_to_float(unsigned short b)
{
    if constexpr (std::is_same<S, __half>::value || std::is_same<S, Half16SR>::value)
        return __half2float(__ushort_as_half(b));
    else
        return __uint_as_float(static_cast<uint32_t>(b) << 16);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of `bar` with parity `parity`; false if it did not
// complete within kRowWaitLimitNs or the block's abort flag went up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int* abort_flag)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag != 0 || global_ns() - t0 > kRowWaitLimitNs) return false;
    }
}

// Global -> shared bulk copy completing on `bar` (non-multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Shared -> global bulk copy in the thread's bulk async-group.
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
}

// Global -> L2 prefetch of a byte range (no shared memory involved).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Earlier bulk stores of this thread have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Earlier bulk stores of this thread are complete (writes performed).
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's shared-memory writes before later async-proxy reads.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- the kernel -----------------------------------------------------------

// A walk over the rows q, q + G, q + 2G, ... of the box [y0, y0 + ry) x
// [z0, z0 + rz), y fastest, without a division per row.
struct RowWalk {
    int y, z;        // coordinates of the current row
    int dy, dz;      // G = dz * ry + dy, 0 <= dy < ry
    int y0, yend;    // y0 + ry
    __device__ __forceinline__ void init(int q, int G, int y0_, int z0, int ry)
    {
        y0 = y0_;
        yend = y0_ + ry;
        z = z0 + q / ry;
        y = y0_ + q % ry;
        dz = G / ry;
        dy = G % ry;
    }
    __device__ __forceinline__ void advance()
    {
        y += dy;
        z += dz;
        if (y >= yend) {
            y -= yend - y0;
            z += 1;
        }
    }
};

// Global row start of plane pointer p at row (y, z).
template <typename S>
__device__ __forceinline__ S* row_ptr(S* p, const Domain& D, int y, int z)
{
    return p + (static_cast<long long>(z) * D.nxy + static_cast<long long>(y) * D.nx);
}

// Source row of window d for the row (y, z) of mode MODE.
template <int MODE, typename S>
__device__ __forceinline__ const S* window_src(const RowArgs<S>& a, int d, int y, int z)
{
    const Domain& D = a.s.dom;
    const int cy = cy_of(d), cz = cz_of(d);
    if (MODE == ROWS_PULL) {
        int sy = y - cy, sz = z - cz;
        if ((unsigned)sy >= (unsigned)D.ny) sy = y;
        if ((unsigned)sz >= (unsigned)D.nz) sz = z;
        return row_ptr(a.s.src.p[d], D, sy, sz);
    } else if (MODE == ROWS_AA_EVEN) {
        return row_ptr(a.s.src.p[d], D, y, z);
    } else {
        return row_ptr(a.s.src.p[26 - d], D, y - cy, z - cz);
    }
}

// Destination row of output d for the row (y, z).
template <int MODE, typename S>
__device__ __forceinline__ S* output_dst(const RowArgs<S>& a, int d, int y, int z)
{
    const Domain& D = a.s.dom;
    if (MODE == ROWS_AA_ODD) return row_ptr(a.s.dst.p[d], D, y + cy_of(d), z + cz_of(d));
    return row_ptr(a.s.dst.p[d], D, y, z);
}

// The producer warp stages row (y, z) into stage st: lane l < 27 copies
// window l, lane 27 the op bytes; lane 0 first announces the byte count.
// The producer warp prefetches the 27 window rows of row (y, z) into L2.
template <int MODE, typename S>
__device__ __forceinline__ void prefetch_row(const RowArgs<S>& a, int y, int z, int lane)
{
    if (lane < 27) bulk_prefetch_l2(window_src<MODE>(a, lane, y, z), static_cast<uint32_t>(a.s.dom.nx * sizeof(S)));
}

template <int MODE, int STAGES, typename S>
__device__ __forceinline__ void issue_row_loads(const RowArgs<S>& a, unsigned char* smem, const RowSmem& L, int y,
                                                int z, int st, int lane)
{
    const int nx = a.s.dom.nx;
    const uint32_t row_bytes = static_cast<uint32_t>(nx * sizeof(S));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars) + st;
    if (lane == 0)
        mbar_arrive_expect_tx(full, 27u * row_bytes + static_cast<uint32_t>(nx) + static_cast<uint32_t>(a.debug_extra_tx));
    __syncwarp();
    if (lane < 27) {
        S* win = reinterpret_cast<S*>(smem + L.win + st * L.stage_bytes) + lane * nx;
        bulk_load(win, window_src<MODE>(a, lane, y, z), row_bytes, full);
    } else if (lane == 27) {
        bulk_load(smem + L.ops + st * nx,
                  a.s.ops + (static_cast<long long>(z) * a.s.dom.nxy + static_cast<long long>(y) * nx),
                  static_cast<uint32_t>(nx), full);
    }
}

// The 27 populations of cell x of the staged row into f (raw values), the
// clamped pulls of the x-face cells of the odd step from the edge buffer.
template <int MODE, typename S>
__device__ __forceinline__ void row_load(const RowArgs<S>& a, const S* win, int nx, int x, int y, int z, float* f)
{
    const int e_of[3] = {x < nx - 1 ? x + 1 : x, x, x > 0 ? x - 1 : 0};   // element for cx = -1, 0, +1
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = ld_raw<S, float>(win + d * nx + (MODE == ROWS_AA_EVEN ? x : e_of[cx_of(d) + 1]));
    if (MODE == ROWS_AA_ODD && (x == 0 || x == nx - 1)) {
        const Domain& D = a.s.dom;
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            if (cx_of(d) == 1 && x == 0) f[d] = ld_raw<S, float>(xface_edge_ptr(a.s.edge, D, a.s.el, 0, d, y, z));
            if (cx_of(d) == -1 && x == nx - 1) f[d] = ld_raw<S, float>(xface_edge_ptr(a.s.edge, D, a.s.el, 1, d, y, z));
        }
    }
}

// Output of cell x into the shared output rows `out` (STORE cells), or the
// bits its slots already hold (cells without STORE).
template <int MODE, typename S>
__device__ __forceinline__ void row_store(const RowArgs<S>& a, const S* win, S* out, int nx, int x, int y, int z,
                                          int i, uint8_t op, uint32_t hc, const float* f)
{
    const Domain& D = a.s.dom;
    if (op & OP_STORE) {
        if (MODE == ROWS_PULL) {
            put27_raw<S>(f, hc, [&](int d) { return out + d * nx + x; });
        } else if (MODE == ROWS_AA_EVEN) {
            put27_raw<S>(f, hc, [&](int d) { return out + (26 - d) * nx + x; });
            if (x == 0 || x == nx - 1) {
#pragma unroll
                for (int d = 0; d < 27; ++d) {
                    if (cx_of(d) == 1 && x == 0)
                        put_raw(const_cast<S*>(xface_edge_ptr(a.s.edge, D, a.s.el, 0, d, y + cy_of(d), z + cz_of(d))),
                                f[d], hc, d);
                    if (cx_of(d) == -1 && x == nx - 1)
                        put_raw(const_cast<S*>(xface_edge_ptr(a.s.edge, D, a.s.el, 1, d, y + cy_of(d), z + cz_of(d))),
                                f[d], hc, d);
                }
            }
        } else if (x > 0 && x < nx - 1) {
            put27_raw<S>(f, hc, [&](int d) { return out + d * nx + (x + cx_of(d)); });
        } else {
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const int cx = cx_of(d);
                // the pushed slot x + cx when inside the row; a face cell
                // also writes its own clamp slot at x
                if (x + cx >= 0 && x + cx < nx) put_raw(out + d * nx + (x + cx), f[d], hc, d);
                if ((cx == 1 && x == 0) || (cx == -1 && x == nx - 1)) put_raw(out + d * nx + x, f[d], hc, d);
            }
        }
    } else {
        unsigned short* o16 = reinterpret_cast<unsigned short*>(out);
        const unsigned short* w16 = reinterpret_cast<const unsigned short*>(win);
        if (MODE == ROWS_PULL) {
#pragma unroll
            for (int d = 0; d < 27; ++d) o16[d * nx + x] = reinterpret_cast<const unsigned short*>(a.s.dst.p[d])[i];
        } else if (MODE == ROWS_AA_EVEN) {
#pragma unroll
            for (int d = 0; d < 27; ++d) o16[d * nx + x] = w16[d * nx + x];
        } else {
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const int cx = cx_of(d);
                if (x + cx >= 0 && x + cx < nx) o16[d * nx + (x + cx)] = w16[(26 - d) * nx + (x + cx)];
                if ((cx == 1 && x == 0) || (cx == -1 && x == nx - 1)) o16[d * nx + x] = w16[(26 - d) * nx + x];
            }
        }
    }
}

template <typename S, int MODE, int STAGES, int OUTB, int PF>
__global__ void __launch_bounds__(1024) k_rows16(const __grid_constant__ RowArgs<S> a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const Domain& D = a.s.dom;
    const int nx = D.nx;
    const RowSmem L = row_smem_layout<S, STAGES, OUTB>(nx);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);
    uint64_t* empty = full + STAGES;
    uint64_t* ofull = empty + STAGES;
    uint64_t* oempty = ofull + OUTB;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(oempty + OUTB);
    const int NW = row_consumer_warps(nx);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = gridDim.x;
    if (static_cast<int>(blockIdx.x) >= a.nrows) return;

    if (threadIdx.x == 0) {
        for (int st = 0; st < STAGES; ++st) {
            mbar_init(full + st, 1);
            mbar_init(empty + st, NW);
        }
        for (int b = 0; b < OUTB; ++b) {
            mbar_init(ofull + b, NW);
            mbar_init(oempty + b, 1);
        }
        *abort_flag = 0;
        mbar_init_fence();
    }
    __syncthreads();
    bool ok = true;

    if (warp == NW) {
        // ---- producer: loads STAGES rows ahead (and prefetches PF more into
        // L2), stores each row once written
        RowWalk ld, st_row, pf;
        ld.init(blockIdx.x, G, a.y0, a.z0, a.ry);
        st_row = ld;
        int kl = 0;   // rows staged so far
        for (int q = blockIdx.x; q < a.nrows && kl < STAGES; q += G, ++kl, ld.advance())
            issue_row_loads<MODE, STAGES>(a, smem, L, ld.y, ld.z, kl, lane);
        pf = ld;
        int qp = blockIdx.x + STAGES * G;   // next row to prefetch
        for (int j = 0; j < PF && qp < a.nrows; ++j, qp += G, pf.advance()) prefetch_row<MODE>(a, pf.y, pf.z, lane);
        int ks = 0;
        for (int q = blockIdx.x; q < a.nrows && ok; q += G, ++ks, st_row.advance()) {
            // refill the stage of row ks with row ks + STAGES once every consumer warp has read it
            const int sl = ks % STAGES;
            if (q + STAGES * G < a.nrows) {
                ok = __all_sync(0xffffffffu, mbar_wait_bounded(empty + sl, static_cast<uint32_t>(ks / STAGES) & 1u,
                                                                abort_flag));
                if (!ok) break;
                issue_row_loads<MODE, STAGES>(a, smem, L, ld.y, ld.z, sl, lane);
                ++kl;
                ld.advance();
                if (PF > 0 && qp < a.nrows) {
                    prefetch_row<MODE>(a, pf.y, pf.z, lane);
                    qp += G;
                    pf.advance();
                }
            }
            // write row ks back once every consumer warp has written it
            const int b = ks % OUTB;
            ok = __all_sync(0xffffffffu,
                            mbar_wait_bounded(ofull + b, static_cast<uint32_t>(ks / OUTB) & 1u, abort_flag));
            if (!ok) break;
            if (lane < 27) {
                S* o = reinterpret_cast<S*>(smem + L.out) + (b * 27 + lane) * nx;
                bulk_store(output_dst<MODE>(a, lane, st_row.y, st_row.z), o, static_cast<uint32_t>(nx * sizeof(S)));
                bulk_commit();
                // OUTB == 2: the previous row's stores have read their buffer;
                // OUTB == 1: this row's stores have read the buffer
                if (OUTB == 2)
                    asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                else
                    bulk_wait_read_all();
            }
            __syncwarp();
            if (lane == 0) {
                if (OUTB == 1)
                    mbar_arrive(oempty);
                else if (ks >= 1)
                    mbar_arrive(oempty + ((ks - 1) % OUTB));
            }
        }
        if (lane < 27) bulk_wait_all();
        if (!ok) {
            if (lane == 0) {
                *abort_flag = 1;
                atomicExch_system(a.err, static_cast<int>(CULBM_ERR_DEVICE_TIMEOUT));
            }
            // let the last row staged into each stage land (each wait bounded)
            for (int j = (kl > STAGES ? kl - STAGES : 0); j < kl; ++j) {
                volatile int none = 0;
                mbar_wait_bounded(full + j % STAGES, static_cast<uint32_t>(j / STAGES) & 1u, &none);
            }
        }
        return;
    }

    // ---- consumers: one thread per cell of the row
    constexpr int E = ScaleExp<S>::value;
    const int x = threadIdx.x;
    const bool cell = x < nx;
    RowWalk cur;
    cur.init(blockIdx.x, G, a.y0, a.z0, a.ry);
    int k = 0;
    for (int q = blockIdx.x; q < a.nrows; q += G, ++k, cur.advance()) {
        const int st = k % STAGES;
        const int b = k % OUTB;
        ok = __all_sync(0xffffffffu, mbar_wait_bounded(full + st, static_cast<uint32_t>(k / STAGES) & 1u, abort_flag));
        if (!ok) break;
        const int y = cur.y, z = cur.z;
        const int i = x + nx * (y + D.ny * z);
        const S* win = reinterpret_cast<const S*>(smem + L.win + st * L.stage_bytes);
        float f[27];
        uint8_t op = 0;
        if (cell) {
            op = smem[L.ops + st * nx + x];
            if (op & OP_LOAD) {
                row_load<MODE>(a, win, nx, x, y, z, f);
            } else {
#pragma unroll
                for (int d = 0; d < 27; ++d) f[d] = 0.0f;
            }
        }
        // cells without STORE copy window bits in place: release the stage after the output
        const bool keep_win = MODE != ROWS_PULL && cell && !(op & OP_STORE);
        if (!__any_sync(0xffffffffu, keep_win)) {
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + st);
        }
        if (cell) {
            const uint32_t hc = cell_hash(static_cast<uint32_t>(i), a.s.seed);
            cell_update_fast<E>(op, a.s.inv_tau, a.s.rho, a.s.vx, a.s.vy, a.s.vz, i, f);
            if (k >= OUTB) ok = mbar_wait_bounded(oempty + b, static_cast<uint32_t>(k / OUTB - 1) & 1u, abort_flag);
            if (ok) row_store<MODE>(a, win, reinterpret_cast<S*>(smem + L.out) + b * 27 * nx, nx, x, y, z, i, op, hc, f);
            fence_proxy_async_smem();
        } else if (k >= OUTB) {
            ok = mbar_wait_bounded(oempty + b, static_cast<uint32_t>(k / OUTB - 1) & 1u, abort_flag);
        }
        if (__any_sync(0xffffffffu, keep_win)) {
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + st);
        }
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(ofull + b);
    }
    if (!ok && lane == 0) {
        *abort_flag = 1;
        atomicExch_system(a.err, static_cast<int>(CULBM_ERR_DEVICE_TIMEOUT));
    }
}

}  // namespace culbm
