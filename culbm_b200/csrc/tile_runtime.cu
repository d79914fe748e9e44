// Host side of the blocked policies (optPolicy 1, 2, 3): tile geometry, tile
// buffers per lane (tiles of a round run on two streams), the optional
// persisting-L2 access-policy window over them, the per-round launch
// sequence (replayed as one CUDA graph), and the ring-buffer option.
//
// Replaces the reference's haloBlocking*Run lambdas and initBlockingFlag /
// initRingDDFBuf / mapGlobalMem2PersistL2
// (src/simulator/single_dev_expt/simulator_expt_platform.cu:120-305, 608-942).
// optPolicy 1 (static L2) runs on the same L2 tile engine as 3 (dynamic L2).
// optPolicy 2 (L1/L2 mixed) with pull streaming runs on the cluster engine
// (cluster_kernels.cuh: one thread-block cluster per tile, populations in
// registers, streaming through shared memory and DSMEM, one launch per
// round) whenever the tile fits one cluster; larger tiles, and in-place
// streaming, run on the L2 tile engine.  Every engine gives the plain step's
// results bit for bit, so they differ only in speed.
#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "sim_internal.cuh"
#include "cluster_kernels.cuh"
#include "tile_kernels.cuh"

namespace culbm {

// Blocking geometry, restating blocking_core::validBlkAxisConfig,
// calcBlkNum and calcValidPrev (src/blocking_core/blocking_alogrithm.hpp:7-41)
// with the unsigned arithmetic the reference instantiates them with.
bool valid_blk_axis(uint32_t dom, uint32_t blk, uint32_t it)
{
    if (blk < dom && blk + 1 <= it) return false;
    if (2 * (blk + 1 - it) < dom && blk + 2 <= it) return false;
    return true;
}

uint32_t blk_num(uint32_t dom, uint32_t blk, uint32_t it)
{
    if (dom <= blk) return 1;
    if (dom <= 2 * (blk + 1 - it)) return 2;
    const uint32_t num = dom - 2 * (blk + 1 - it), den = blk + 2 - 2 * it;
    return 2 + (num + den - 1) / den;
}

int32_t valid_prev(int32_t idx, int32_t blk, int32_t num, int32_t it, int32_t dom)
{
    if (idx == num) return dom;
    if (idx == 0) return 0;
    return (blk + 1 - it) + (idx - 1) * (blk + 2 - 2 * it);
}

// Streams over which the tiles of one round are spread (double-buffered
// global state only).
constexpr int kTileLanes = 2;

namespace {

struct TileGeom {
    int org[3];
    int vlo[3], vhi[3];
};

}  // namespace

struct TileState {
    int B[3] = {0, 0, 0};
    int nt[3] = {1, 1, 1};
    int I = 1;
    long long tile_n = 0;
    std::vector<TileGeom> tiles;
    // Tiles of a round run on `lanes` streams at once (tile i on lane i mod
    // lanes), each lane with its own tile buffers and, in place, its own
    // edge buffer (scratch of one tile's round).  Concurrent tiles let one
    // tile's DRAM-bound first and last steps overlap other tiles' L2-bound
    // middle steps.  Not with the ring buffer, whose in-place result writes
    // are placed for tiles taken in order; under a persisting-L2 window only
    // when all lanes' tile buffers fit in 70 % of L2 (the window's set-aside
    // otherwise makes the lanes evict each other's tiles).
    int lanes = 1;
    cudaStream_t side[kTileLanes] = {};      // streams of lanes 1.. (lane 0: the simulation's)
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[kTileLanes] = {};
    void* d_edge_lane[kTileLanes] = {};      // edge buffers of lanes 1.. (lane 0: the simulation's)
    size_t lane_bytes = 0;                   // tile buffers of one lane
    void* d_tile = nullptr;      // lanes x (tile buffer 0, and 1 for pull)
    RoundState* d_rs = nullptr;
    RoundState h_rs{};
    int ring_nz = 0, ring_step = 0;
    long long gstride = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_I = 0;
    uint64_t graph_launches = 0;     // kernel launches in the captured round
    bool window = false;
    cudaAccessPolicyWindow apw{};
    size_t persist_bytes = 0;
    // cluster engine (optPolicy 2, pull): CTA shape, CTAs per tile per axis
    // (the cluster's shape) and dynamic shared memory per CTA
    bool cluster = false;
    int cta[3] = {0, 0, 0};
    int cdim[3] = {0, 0, 0};
    size_t cluster_smem = 0;
};

bool is_blocked(const culbm_config& cfg) { return cfg.opt_policy != CULBM_OPT_NONE; }

namespace {

template <typename S>
struct TileLauncher {
    using R = typename ArithOf<S>::type;
    culbm_sim* s;
    TileState* ts;

    TileArgs<S, R> base_args() const
    {
        TileArgs<S, R> a{};
        a.dom = s->dom;
        a.bx = ts->B[0];
        a.by = ts->B[1];
        a.bz = ts->B[2];
        a.bxy = ts->B[0] * ts->B[1];
        a.ops = s->d_ops;
        a.rho = s->d_mac[0];
        a.vx = s->d_mac[1];
        a.vy = s->d_mac[2];
        a.vz = s->d_mac[3];
        a.inv_tau = static_cast<R>(s->cfg.inv_tau);
        a.g.base[0] = static_cast<S*>(s->d_pop[0]);
        a.g.base[1] = static_cast<S*>(s->d_pop[ts->ring_nz ? 0 : 1]);
        a.g.stride = ts->gstride;
        a.g.ring_nz = ts->ring_nz;
        a.g.ring_step = ts->ring_step;
        S* t = static_cast<S*>(ts->d_tile);
        a.t0.set(t, ts->tile_n);
        a.t1.set(t + 27 * ts->tile_n, ts->tile_n);
        a.edge = static_cast<S*>(s->d_edge);
        a.el = s->el;
        a.rs = ts->d_rs;
        return a;
    }

    // Launch of one step of the round on the part of the tile that later
    // steps still read: the valid box grown by e = (steps left after this
    // one), clipped to the tile and the domain.  A cell outside it only
    // feeds cells farther than e from the valid box, whose values are never
    // used, so the valid cells get the same bits as with whole-tile steps.
    template <typename K>
    culbm_status launch(K kernel, TileArgs<S, R> a, const TileGeom& g, int e, cudaStream_t stream)
    {
        int lo[3], n[3];
        for (int q = 0; q < 3; ++q) {
            const int dom_q = q == 0 ? s->dom.nx : q == 1 ? s->dom.ny : s->dom.nz;
            lo[q] = std::max(0, g.vlo[q] - g.org[q] - e);
            const int hi = std::min(std::min(ts->B[q], dom_q - g.org[q]), g.vhi[q] - g.org[q] + e);
            n[q] = hi - lo[q];
            if (n[q] <= 0) return CULBM_OK;
        }
        a.sx = lo[0];
        a.sy = lo[1];
        a.sz = lo[2];
        cudaLaunchConfig_t lc{};
        lc.gridDim = dim3((n[0] + 31) / 32, (n[1] + 7) / 8, n[2]);
        lc.blockDim = dim3(32, 8, 1);
        lc.stream = stream;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        if (ts->window) {
            attr[1].id = cudaLaunchAttributeAccessPolicyWindow;
            attr[1].val.accessPolicyWindow = ts->apw;
            lc.numAttrs = 2;
        }
        CULBM_CUDA(cudaLaunchKernelEx(&lc, kernel, a));
        s->launches += 1;
        return CULBM_OK;
    }

    // Every tile of a round of k steps in one launch of the cluster engine.
    template <bool HINT>
    culbm_status cluster_round(int k)
    {
        ClusterTileArgs<S, R> a{};
        a.dom = s->dom;
        for (int q = 0; q < 3; ++q) {
            a.B[q] = ts->B[q];
            a.nt[q] = ts->nt[q];
            a.cdim[q] = ts->cdim[q];
        }
        a.I = ts->I;
        a.k = k;
        a.ops = s->d_ops;
        a.rho = s->d_mac[0];
        a.vx = s->d_mac[1];
        a.vy = s->d_mac[2];
        a.vz = s->d_mac[3];
        a.inv_tau = static_cast<R>(s->cfg.inv_tau);
        a.g.base[0] = static_cast<S*>(s->d_pop[0]);
        a.g.base[1] = static_cast<S*>(s->d_pop[1]);
        a.g.stride = ts->gstride;
        a.rs = ts->d_rs;
        cudaLaunchConfig_t lc{};
        lc.gridDim = dim3(ts->cdim[0] * ts->nt[0], ts->cdim[1] * ts->nt[1], ts->cdim[2] * ts->nt[2]);
        lc.blockDim = dim3(ts->cta[0], ts->cta[1], ts->cta[2]);
        lc.dynamicSmemBytes = ts->cluster_smem;
        lc.stream = s->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = ts->cdim[0];
        attr[0].val.clusterDim.y = ts->cdim[1];
        attr[0].val.clusterDim.z = ts->cdim[2];
        lc.attrs = attr;
        lc.numAttrs = 1;
        CULBM_CUDA(cudaLaunchKernelEx(&lc, k_tile_cluster_pull<S, R, HINT>, a));
        s->launches += 1;
        return CULBM_OK;
    }

    // All tiles for one round of k <= I steps, then the round-state advance.
    // Step j of a tile (0-based) covers the valid box grown by k - 1 - j.
    // With two lanes, lane 1 forks from and joins the simulation's stream
    // (recorded into the round's graph when captured).
    culbm_status round(int k)
    {
        const bool hint = s->cfg.cache_hints != 0;
        const bool inplace = s->cfg.stream_policy == CULBM_STREAM_INPLACE;
        if (ts->cluster) {
            CULBM_TRY(hint ? cluster_round<true>(k) : cluster_round<false>(k));
            k_tile_advance<<<1, 32, 0, s->stream>>>(ts->d_rs, ts->ring_nz, ts->ring_step, k);
            CULBM_CUDA(cudaGetLastError());
            s->launches += 1;
            return CULBM_OK;
        }
        const TileArgs<S, R> base = base_args();
        if (ts->lanes > 1) {
            CULBM_CUDA(cudaEventRecord(ts->ev_fork, s->stream));
            for (int l = 1; l < ts->lanes; ++l) CULBM_CUDA(cudaStreamWaitEvent(ts->side[l], ts->ev_fork, 0));
        }
        for (size_t ti = 0; ti < ts->tiles.size(); ++ti) {
            const TileGeom& g = ts->tiles[ti];
            const int lane = static_cast<int>(ti % static_cast<size_t>(ts->lanes));
            const cudaStream_t st = lane ? ts->side[lane] : s->stream;
            TileArgs<S, R> a = base;
            if (lane) {
                S* t = reinterpret_cast<S*>(static_cast<char*>(ts->d_tile) + lane * ts->lane_bytes);
                a.t0.set(t, ts->tile_n);
                a.t1.set(t + 27 * ts->tile_n, ts->tile_n);
                a.edge = static_cast<S*>(ts->d_edge_lane[lane]);
            }
            a.ox = g.org[0];
            a.oy = g.org[1];
            a.oz = g.org[2];
            for (int q = 0; q < 3; ++q) {
                a.vlo[q] = g.vlo[q];
                a.vhi[q] = g.vhi[q];
            }
            a.j = 0;
            if (inplace) {
                if (k == 1) {
                    CULBM_TRY(hint ? launch(k_tile_aa_first<S, R, true, true>, a, g, 0, st)
                                   : launch(k_tile_aa_first<S, R, true, false>, a, g, 0, st));
                    continue;
                }
                CULBM_TRY(hint ? launch(k_tile_aa_first<S, R, false, true>, a, g, k - 1, st)
                               : launch(k_tile_aa_first<S, R, false, false>, a, g, k - 1, st));
                for (int j = 2; j < k; ++j) {
                    a.j = j - 1;
                    if (j % 2 == 0) CULBM_TRY(launch(k_tile_aa_odd<S, R>, a, g, k - j, st));
                    else CULBM_TRY(launch(k_tile_aa_even<S, R>, a, g, k - j, st));
                }
                a.j = k - 1;
                if (k % 2 == 0)
                    CULBM_TRY(hint ? launch(k_tile_aa_last<LAYOUT_AA_A, S, R, true>, a, g, 0, st)
                                   : launch(k_tile_aa_last<LAYOUT_AA_A, S, R, false>, a, g, 0, st));
                else
                    CULBM_TRY(hint ? launch(k_tile_aa_last<LAYOUT_AA_B, S, R, true>, a, g, 0, st)
                                   : launch(k_tile_aa_last<LAYOUT_AA_B, S, R, false>, a, g, 0, st));
            } else {
                if (k == 1) {
                    CULBM_TRY(hint ? launch(k_tile_pull_first<S, R, true, true>, a, g, 0, st)
                                   : launch(k_tile_pull_first<S, R, true, false>, a, g, 0, st));
                    continue;
                }
                CULBM_TRY(hint ? launch(k_tile_pull_first<S, R, false, true>, a, g, k - 1, st)
                               : launch(k_tile_pull_first<S, R, false, false>, a, g, k - 1, st));
                for (int j = 2; j < k; ++j) {
                    a.j = j - 1;
                    CULBM_TRY(launch(k_tile_pull_mid<S, R>, a, g, k - j, st));
                    std::swap(a.t0, a.t1);
                }
                a.j = k - 1;
                CULBM_TRY(hint ? launch(k_tile_pull_last<S, R, true>, a, g, 0, st)
                               : launch(k_tile_pull_last<S, R, false>, a, g, 0, st));
            }
        }
        for (int l = 1; l < ts->lanes; ++l) {
            CULBM_CUDA(cudaEventRecord(ts->ev_join[l], ts->side[l]));
            CULBM_CUDA(cudaStreamWaitEvent(s->stream, ts->ev_join[l], 0));
        }
        k_tile_advance<<<1, 32, 0, s->stream>>>(ts->d_rs, ts->ring_nz, ts->ring_step, k);
        CULBM_CUDA(cudaGetLastError());
        s->launches += 1;
        return CULBM_OK;
    }
};

void host_advance(TileState* ts, int steps)
{
    ts->h_rs.step += static_cast<uint32_t>(steps);
    if (ts->ring_nz) {
        ts->h_rs.src_offz = ts->h_rs.dst_offz;
        int o = ts->h_rs.dst_offz - ts->ring_step;
        if (o < 0) o += ts->ring_nz;
        ts->h_rs.dst_offz = o;
    } else {
        ts->h_rs.sel = 1 - ts->h_rs.sel;
    }
}

template <typename S>
culbm_status tiles_step_typed(culbm_sim* s, uint32_t nsteps)
{
    TileState* ts = s->tiles;
    TileLauncher<S> L{s, ts};
    const uint32_t I = static_cast<uint32_t>(ts->I);
    uint32_t full = nsteps / I;
    const uint32_t rem = nsteps % I;
    if (full > 0 && s->cfg.use_graphs) {
        if (ts->graph == nullptr || ts->graph_I != ts->I) {
            if (ts->graph) cudaGraphExecDestroy(ts->graph);
            ts->graph = nullptr;
            cudaGraph_t g = nullptr;
            const uint64_t launches0 = s->launches;
            CULBM_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            const culbm_status st = L.round(ts->I);
            const cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
            if (st != CULBM_OK) {
                if (g) cudaGraphDestroy(g);
                return st;
            }
            if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
            const cudaError_t ie = cudaGraphInstantiate(&ts->graph, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
            ts->graph_I = ts->I;
            ts->graph_launches = s->launches - launches0;
            s->launches = launches0;
        }
        const uint64_t per_round = ts->graph_launches;
        for (uint32_t r = 0; r < full; ++r) {
            CULBM_CUDA(cudaGraphLaunch(ts->graph, s->stream));
            s->launches += per_round;
            host_advance(ts, ts->I);
        }
        full = 0;
    }
    for (uint32_t r = 0; r < full; ++r) {
        CULBM_TRY(L.round(ts->I));
        host_advance(ts, ts->I);
    }
    if (rem) {
        CULBM_TRY(L.round(static_cast<int>(rem)));
        host_advance(ts, static_cast<int>(rem));
    }
    s->cur = ts->h_rs.sel;
    return CULBM_OK;
}

template <typename S>
__global__ void k_fill_dirs(S* base, long long stride, typename ArithOf<S>::type rho)
{
    using R = typename ArithOf<S>::type;
    R f[27];
    equilibrium<R>(rho, R(0), R(0), R(0), f);
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < stride;
         j += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int d = 0; d < 27; ++d) Cvt<S, R>::st(base + d * stride + j, f[d]);
}

// CTA shape and cluster shape for the cluster engine: one thread per tile
// cell, at most kClusterMaxThreads threads per CTA and kClusterMaxCtas CTAs
// per tile; CTA widths are multiples of 32 or the tile's own width.
// Preferred: portable clusters (at most 8 CTAs), then the fewest idle
// threads, then the fewest CTAs.  False if no shape covers the tile.
bool cluster_shape(const int B[3], int cta[3], int cdim[3])
{
    const long long cells = 1ll * B[0] * B[1] * B[2];
    long long best = LLONG_MAX;
    std::vector<int> widths;
    for (int tx = 32; tx <= kClusterMaxThreads && tx - 32 < B[0]; tx += 32) widths.push_back(tx);
    if (B[0] % 32 != 0 && B[0] <= kClusterMaxThreads) widths.push_back(B[0]);
    for (const int tx : widths)
        for (int ty = 1; tx * ty <= kClusterMaxThreads && ty <= B[1]; ++ty)
            for (int tz = 1; tx * ty * tz <= kClusterMaxThreads && tz <= B[2]; ++tz) {
                const int n[3] = {(B[0] + tx - 1) / tx, (B[1] + ty - 1) / ty, (B[2] + tz - 1) / tz};
                const long long ctas = 1ll * n[0] * n[1] * n[2];
                if (ctas > kClusterMaxCtas) continue;
                const long long idle = ctas * tx * ty * tz - cells;
                const long long key = (ctas > 8 ? (1ll << 40) : 0) + idle * 64 + ctas;
                if (key < best) {
                    best = key;
                    cta[0] = tx;
                    cta[1] = ty;
                    cta[2] = tz;
                    for (int q = 0; q < 3; ++q) cdim[q] = n[q];
                }
            }
    return best != LLONG_MAX;
}

// Selects the cluster engine for optPolicy 2 with pull streaming when the
// tile fits one cluster and the GPU can hold such a cluster; otherwise the
// tile engine stays in charge (ts->cluster false).
template <typename S>
culbm_status cluster_plan(culbm_sim* s, TileState* ts)
{
    using R = typename ArithOf<S>::type;
    // The reference's split when it fits (blockDim is the CTA, gridDim the
    // tile's CTAs: HaloBlockingL1L2D3Q27PullKernel's launch,
    // simulator_expt_platform.cu:608-650), else a shape of our own.
    const culbm_config& c = s->cfg;
    int cta[3], cdim[3];
    const unsigned long long user_threads = 1ull * c.block_dim[0] * c.block_dim[1] * c.block_dim[2];
    const unsigned long long user_ctas = 1ull * c.grid_dim[0] * c.grid_dim[1] * c.grid_dim[2];
    if (user_threads >= 32 && user_threads <= kClusterMaxThreads && user_ctas <= kClusterMaxCtas) {
        for (int q = 0; q < 3; ++q) {
            cta[q] = static_cast<int>(c.block_dim[q]);
            cdim[q] = static_cast<int>(c.grid_dim[q]);
        }
    } else if (!cluster_shape(ts->B, cta, cdim)) {
        return CULBM_OK;
    }
    for (int q = 0; q < 3; ++q)
        if (1ll * cdim[q] * ts->nt[q] > (q == 0 ? INT_MAX : 65535)) return CULBM_OK;
    const int nthr = cta[0] * cta[1] * cta[2];
    const int ctas = cdim[0] * cdim[1] * cdim[2];
    const size_t smem = 2ull * 27 * nthr * sizeof(S);
    void (*kernels[2])(ClusterTileArgs<S, R>) = {k_tile_cluster_pull<S, R, true>, k_tile_cluster_pull<S, R, false>};
    for (auto kern : kernels) {
        CULBM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        if (ctas > 8) CULBM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(cdim[0] * ts->nt[0], cdim[1] * ts->nt[1], cdim[2] * ts->nt[2]);
    lc.blockDim = dim3(cta[0], cta[1], cta[2]);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cdim[0];
    attr[0].val.clusterDim.y = cdim[1];
    attr[0].val.clusterDim.z = cdim[2];
    lc.attrs = attr;
    lc.numAttrs = 1;
    int resident = 0;
    if (cudaOccupancyMaxActiveClusters(&resident, kernels[0], &lc) != cudaSuccess) {
        (void)cudaGetLastError();   // not a sticky error: this shape just cannot run
        return CULBM_OK;
    }
    if (resident < 1) return CULBM_OK;
    ts->cluster = true;
    for (int q = 0; q < 3; ++q) {
        ts->cta[q] = cta[q];
        ts->cdim[q] = cdim[q];
    }
    ts->cluster_smem = smem;
    return CULBM_OK;
}

}  // namespace

// One axis of a blocked geometry: tile extent b (blockDim*gridDim) over
// domain extent dom with innerLoop I >= 1.
static culbm_status validate_axis(uint32_t dom, unsigned long long b, uint32_t I)
{
    if (b > 65535) return fail(CULBM_ERR_INVALID_ARGUMENT, "tile extent blockDim*gridDim above 65535");
    const uint32_t B = static_cast<uint32_t>(b);
    if (!valid_blk_axis(dom, B, I))
        return fail(CULBM_ERR_INVALID_ARGUMENT, "<Domain Dimension, Blocking Dimension and InnerLoop> don't match!");
    // The reference's check lets B + 2 - 2I <= 0 through when more than
    // two tiles are needed, and calcBlkNum then divides by it.
    if (dom > B && dom > 2 * (B + 1 - I) && static_cast<long long>(B) + 2 - 2ll * I <= 0)
        return fail(CULBM_ERR_INVALID_ARGUMENT,
                    "<Domain Dimension, Blocking Dimension and InnerLoop> don't match! (tile too small for innerLoop)");
    return CULBM_OK;
}

culbm_status validate_blocking(const culbm_config& c)
{
    if (c.inner_loop < 1) return fail(CULBM_ERR_INVALID_ARGUMENT, "innerLoop must be at least 1");
    const uint32_t I = static_cast<uint32_t>(c.inner_loop);
    for (int k = 0; k < 3; ++k)
        CULBM_TRY(validate_axis(c.domain_dim[k], 1ull * c.block_dim[k] * c.grid_dim[k], I));
    if (c.use_ring_ddf_buf && 1ull * c.block_dim[2] * c.grid_dim[2] < I)
        return fail(CULBM_ERR_INVALID_ARGUMENT, "ring buffer needs blockDim.z*gridDim.z >= innerLoop");
    return CULBM_OK;
}

culbm_status tiles_create(culbm_sim* s)
{
    const culbm_config& c = s->cfg;
    CULBM_TRY(validate_blocking(c));
    TileState* ts = new TileState();
    s->tiles = ts;
    ts->I = c.inner_loop;
    for (int k = 0; k < 3; ++k) ts->B[k] = static_cast<int>(c.block_dim[k] * c.grid_dim[k]);
    const uint32_t I = static_cast<uint32_t>(ts->I);
    for (int k = 0; k < 3; ++k) ts->nt[k] = static_cast<int>(blk_num(c.domain_dim[k], static_cast<uint32_t>(ts->B[k]), I));
    for (int kz = 0; kz < ts->nt[2]; ++kz)
        for (int ky = 0; ky < ts->nt[1]; ++ky)
            for (int kx = 0; kx < ts->nt[0]; ++kx) {
                TileGeom g{};
                const int kk[3] = {kx, ky, kz};
                for (int q = 0; q < 3; ++q) {
                    const int dom = static_cast<int>(c.domain_dim[q]);
                    g.vlo[q] = valid_prev(kk[q], ts->B[q], ts->nt[q], ts->I, dom);
                    g.vhi[q] = valid_prev(kk[q] + 1, ts->B[q], ts->nt[q], ts->I, dom);
                    g.org[q] = std::max(g.vlo[q] - (ts->I - 1), 0);
                }
                ts->tiles.push_back(g);
            }
    ts->tile_n = 1ll * ts->B[0] * ts->B[1] * ts->B[2];
    const bool inplace = c.stream_policy == CULBM_STREAM_INPLACE;
    if (!inplace && c.opt_policy == CULBM_OPT_L1L2) {
        CULBM_TRY(with_storage(s, [&](auto tag) { return cluster_plan<typename decltype(tag)::type>(s, ts); }));
        if (ts->cluster) {
            // no tile buffers: the tile lives in registers and shared memory
            void* p = nullptr;
            CULBM_TRY(dev_alloc(s, &p, sizeof(RoundState), "round state"));
            ts->d_rs = static_cast<RoundState*>(p);
            ts->gstride = s->n;
            return CULBM_OK;
        }
    }
    ts->lane_bytes = ((inplace ? 1 : 2) * 27ull * ts->tile_n * s->esize + 255) / 256 * 256;
    {
        int l2 = 0;
        CULBM_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, s->dev));
        const int want = static_cast<int>(std::min<size_t>(kTileLanes, ts->tiles.size()));
        const bool fits = want * ts->lane_bytes <= static_cast<size_t>(0.7 * static_cast<double>(l2));
        ts->lanes = (!c.use_ring_ddf_buf && (!c.persist_l2 || fits)) ? std::max(want, 1) : 1;
    }
    const size_t tile_bytes = ts->lanes * ts->lane_bytes;
    void* p = nullptr;
    CULBM_TRY(dev_alloc(s, &p, tile_bytes, "tile buffers"));
    ts->d_tile = p;
    if (ts->lanes > 1) {
        CULBM_CUDA(cudaEventCreateWithFlags(&ts->ev_fork, cudaEventDisableTiming));
        for (int l = 1; l < ts->lanes; ++l) {
            CULBM_CUDA(cudaStreamCreateWithFlags(&ts->side[l], cudaStreamNonBlocking));
            CULBM_CUDA(cudaEventCreateWithFlags(&ts->ev_join[l], cudaEventDisableTiming));
        }
    }
    CULBM_TRY(dev_alloc(s, &p, sizeof(RoundState), "round state"));
    ts->d_rs = static_cast<RoundState*>(p);

    if (c.use_ring_ddf_buf) {
        // One global buffer of nz + step planes; each round writes its result
        // `step` planes below its source, modulo the ring
        // (simulator_expt_platform.cu:252-277, 749-846).  A z-slab k of tiles
        // writes its valid planes [vp(k), vp(k+1)); the tiles still to come
        // read from plane vp(k) - innerLoop upwards, so the shifted writes stay
        // clear of them iff step >= extent(k) + innerLoop for k >= 1, and
        // step >= extent(0) for the first slab.  The reference's fixed
        // Bz - (I-1) + 1 meets this for middle slabs only; a longer last slab
        // (or a single slab) would overwrite planes that later tiles read.
        int step = 0;
        const int nz = s->dom.nz;
        for (int kz = 0; kz < ts->nt[2]; ++kz) {
            const int lo = valid_prev(kz, ts->B[2], ts->nt[2], ts->I, nz);
            const int hi = valid_prev(kz + 1, ts->B[2], ts->nt[2], ts->I, nz);
            step = std::max(step, (hi - lo) + (kz > 0 ? ts->I : 0));
        }
        step = std::max(step, ts->B[2] - (ts->I - 1) + 1);
        ts->ring_step = step;
        ts->ring_nz = s->dom.nz + ts->ring_step;
        ts->gstride = 1ll * s->dom.nxy * ts->ring_nz;
        CULBM_TRY(dev_alloc(s, &s->d_pop[0], 27ull * ts->gstride * s->esize, "ring population buffer"));
        s->npop = 1;
    } else {
        ts->gstride = s->n;
    }
    if (inplace) {
        const long long fx = 9ll * s->dom.ny * s->dom.nz, fy = 9ll * s->dom.nx * s->dom.nz, fz = 9ll * s->dom.nx * s->dom.ny;
        s->el.off[0] = 0;
        s->el.off[1] = fx;
        s->el.off[2] = 2 * fx;
        s->el.off[3] = 2 * fx + fy;
        s->el.off[4] = 2 * fx + 2 * fy;
        s->el.off[5] = 2 * fx + 2 * fy + fz;
        s->edge_elems = 2 * (fx + fy + fz);
        CULBM_TRY(dev_alloc(s, &s->d_edge, s->edge_elems * s->esize, "edge buffer"));
        for (int l = 1; l < ts->lanes; ++l)
            CULBM_TRY(dev_alloc(s, &ts->d_edge_lane[l], s->edge_elems * s->esize, "lane edge buffer"));
    }

    // Keep the tile buffers resident: persisting set-aside + access-policy
    // window (the reference's mapGlobalMem2PersistL2, which queries device 0;
    // here the selected device).
    if (c.persist_l2) {
        cudaDeviceProp prop{};
        CULBM_CUDA(cudaGetDeviceProperties(&prop, s->dev));
        if (prop.persistingL2CacheMaxSize > 0 && prop.accessPolicyMaxWindowSize > 0) {
            const size_t setaside = std::min<size_t>(tile_bytes, static_cast<size_t>(prop.persistingL2CacheMaxSize));
            const size_t win = std::min<size_t>(tile_bytes, static_cast<size_t>(prop.accessPolicyMaxWindowSize));
            CULBM_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, setaside));
            ts->apw.base_ptr = ts->d_tile;
            ts->apw.num_bytes = win;
            ts->apw.hitRatio = static_cast<float>(std::min(1.0, static_cast<double>(setaside) / static_cast<double>(win)));
            ts->apw.hitProp = cudaAccessPropertyPersisting;
            ts->apw.missProp = cudaAccessPropertyStreaming;
            ts->window = true;
            ts->persist_bytes = setaside;
        }
    }
    return CULBM_OK;
}

void tiles_destroy(culbm_sim* s)
{
    TileState* ts = s->tiles;
    if (ts == nullptr) return;
    if (ts->graph) cudaGraphExecDestroy(ts->graph);
    cudaFree(ts->d_tile);
    cudaFree(ts->d_rs);
    for (int l = 1; l < kTileLanes; ++l) {
        cudaFree(ts->d_edge_lane[l]);
        if (ts->side[l]) cudaStreamDestroy(ts->side[l]);
        if (ts->ev_join[l]) cudaEventDestroy(ts->ev_join[l]);
    }
    if (ts->ev_fork) cudaEventDestroy(ts->ev_fork);
    if (ts->window) {
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    }
    delete ts;
    s->tiles = nullptr;
}

culbm_status tiles_upload_flags(culbm_sim*, const uint32_t*) { return CULBM_OK; }

// Resets the round state and fills the global state with rest equilibrium.
culbm_status tiles_reset(culbm_sim* s)
{
    TileState* ts = s->tiles;
    ts->h_rs = RoundState{0, 0, ts->ring_nz ? s->dom.nz : 0, 0u};
    CULBM_CUDA(cudaMemcpyAsync(ts->d_rs, &ts->h_rs, sizeof(RoundState), cudaMemcpyHostToDevice, s->stream));
    auto fill = [&](auto tag) -> culbm_status {
        using S = typename decltype(tag)::type;
        using R = typename ArithOf<S>::type;
        for (int k = 0; k < s->npop; ++k) {
            k_fill_dirs<S><<<1184, 256, 0, s->stream>>>(static_cast<S*>(s->d_pop[k]), ts->gstride, R(1));
            CULBM_CUDA(cudaGetLastError());
        }
        return CULBM_OK;
    };
    CULBM_TRY(with_storage(s, fill));
    s->cur = 0;
    return CULBM_OK;
}

culbm_status tiles_step(culbm_sim* s, uint32_t nsteps)
{
    return with_storage(s, [&](auto tag) { return tiles_step_typed<typename decltype(tag)::type>(s, nsteps); });
}

void tiles_view(const culbm_sim* s, int* ring_nz, int* offz, long long* stride)
{
    const TileState* ts = s->tiles;
    *ring_nz = ts ? ts->ring_nz : 0;
    *offz = ts ? ts->h_rs.src_offz : 0;
    *stride = ts ? ts->gstride : s->n;
}

void tiles_info(const culbm_sim* s, culbm_info* info)
{
    const TileState* ts = s->tiles;
    if (ts == nullptr) return;
    for (int k = 0; k < 3; ++k) {
        info->blocking_num[k] = static_cast<uint32_t>(ts->nt[k]);
        info->blocking_dim[k] = static_cast<uint32_t>(ts->B[k]);
    }
    info->persisting_l2_bytes = ts->persist_bytes;
}

}  // namespace culbm

extern "C" culbm_status culbm_blocking_axis(uint32_t domain, uint32_t tile, int32_t inner_loop, uint32_t* num_tiles,
                                            int32_t* valid_starts, uint32_t capacity)
{
    using namespace culbm;
    if (num_tiles == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (inner_loop < 1) return fail(CULBM_ERR_INVALID_ARGUMENT, "innerLoop must be at least 1");
    if (domain < 1 || domain > 0x7FFFFFFFu || tile < 1)
        return fail(CULBM_ERR_INVALID_ARGUMENT, "domain and tile extents must be in [1, 2^31)");
    const uint32_t I = static_cast<uint32_t>(inner_loop);
    CULBM_TRY(validate_axis(domain, tile, I));
    const uint32_t num = blk_num(domain, tile, I);
    *num_tiles = num;
    if (valid_starts == nullptr) return CULBM_OK;
    if (capacity < num + 1ull)
        return fail(CULBM_ERR_INVALID_ARGUMENT, "valid_starts needs " + std::to_string(num + 1ull) + " entries");
    for (uint32_t k = 0; k <= num; ++k)
        valid_starts[k] = valid_prev(static_cast<int32_t>(k), static_cast<int32_t>(tile), static_cast<int32_t>(num),
                                     inner_loop, static_cast<int32_t>(domain));
    return CULBM_OK;
}
