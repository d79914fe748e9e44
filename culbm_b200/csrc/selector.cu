// Tile / innerLoop selection for the L2-blocked policies, and the two memory
// constants its model needs, measured on the current device.
//
// Model (the speed-up over plain streaming of one tile of B = (Bx, By, Bz)
// cells advanced I steps per round in L2; the reference's
// analysis/selector.py:15-69, restated here):
//   h(B, I)  = prod_k (1 - 2 (I-1) / B_k)                 valid fraction of a tile
//   alpha    = 1 + lambda (beta_sec - 1) + p (2 gamma - (1 + lambda)) beta_edge
//              beta_sec:  32-byte sectors per 8 useful floats of the valid x-rows,
//              beta_edge: partial (edge) sectors per useful float, both averaged over
//                         the alignments a row start can take;
//              p = 1 - exp(-V / (L2 - V)), V = tile bytes (0 once V >= L2)
//   S(B, I)  = h / ((1 + alpha h) / (2 I) + lambda (1 - 1/I))
//              (with a compute floor for issue-bound storage formats, below)
// lambda = DRAM bandwidth / L2 bandwidth (copy kernels; 16-byte accesses,
// which B200 needs to reach its HBM bandwidth), gamma = cost of a
// partial sector relative to a full one in a streaming store.  The search
// keeps tiles with Bx a multiple of 32 up to 160, By >= Bz, 2 (I-1) < Bz,
// V within the persisting-L2 limit, 2 <= I <= 20, and (added here) only
// geometries the blocking engine accepts for the given domain, plus
// whole-row tiles (Bx = nx, no x halo between tiles) on domains wider than 160.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sim_internal.cuh"

namespace culbm {
bool valid_blk_axis(uint32_t dom, uint32_t blk, uint32_t inner);   // tile_runtime.cu
}

namespace {

using namespace culbm;

constexpr int kMeasureThreads = 256;
constexpr int kMeasureBlocksPerSm = 8;

// Copy of count float4 values, `passes` times, through L2 (cache-global
// loads and stores), two 16-byte values per thread in flight: the 4-byte
// copies of a plain grid-stride loop leave B200's HBM far from saturated.
__global__ void __launch_bounds__(kMeasureThreads) k_copy_cg(float4* dst, const float4* src, long long count,
                                                             int passes)
{
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (int p = 0; p < passes; ++p) {
        long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        for (; i + stride < count; i += 2 * stride) {
            const float4 u = __ldcg(src + i), v = __ldcg(src + i + stride);
            __stcg(dst + i, u);
            __stcg(dst + i + stride, v);
        }
        if (i < count) __stcg(dst + i, __ldcg(src + i));
    }
}

// One streaming store per lane for `units` 128-byte units; with PARTIAL the
// first 7 floats of each unit are skipped (one partial sector, three full).
template <bool PARTIAL>
__global__ void __launch_bounds__(kMeasureThreads) k_store_units(float* dst, long long units)
{
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5;
    const long long warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
    for (long long u = warp; u < units; u += warps) {
        if (!PARTIAL || lane >= 7) __stcs(dst + u * 32 + lane, 0.0f);
    }
}

template <class F>
culbm_status median_ms(cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, int samples, F&& launch, float* out)
{
    std::vector<float> t(samples);
    launch();   // warm-up
    for (int k = 0; k < samples; ++k) {
        CULBM_CUDA(cudaEventRecord(e0, s));
        launch();
        CULBM_CUDA(cudaEventRecord(e1, s));
        CULBM_CUDA(cudaEventSynchronize(e1));
        CULBM_CUDA(cudaEventElapsedTime(&t[k], e0, e1));
    }
    CULBM_CUDA(cudaGetLastError());
    std::sort(t.begin(), t.end());
    *out = t[samples / 2];
    return CULBM_OK;
}

// (beta_sec, beta_edge) of the valid x-rows of a tile of width bx advanced
// i steps: warps of 32 cells cover x in [r, bx - r), r = i - 1; a row start
// takes the alignments (mod 8 floats) that rows of its length reach.  The
// reference counts the warps of x < 160, its widest tile; wider tiles (the
// whole-row tiles below) count all of theirs, which changes nothing up to 160.
void beta(int bx, int i, double* sec, double* edge)
{
    const int r = i - 1, len = bx - 2 * r;
    *sec = 1.0;
    *edge = 0.0;
    if (len <= 0) return;
    int g = len, b = 8;
    while (b) {
        const int t = g % b;
        g = b;
        b = t;
    }
    const int period = 8 / g;
    long long n_sec = 0, n_edge = 0;
    for (int ph = 0; ph < 8; ++ph) {
        if (ph % g) continue;
        for (int w = 0; w < std::max(160, bx); w += 32) {
            const int lo = std::max(r, w), hi = std::min(bx - r, w + 32);
            if (hi > lo) n_sec += (ph + hi - 1) / 8 + 1 - (ph + lo) / 8;
        }
        n_edge += ((ph + r) % 8 != 0) + ((ph + bx - r) % 8 != 0);
    }
    *sec = 8.0 * n_sec / (static_cast<double>(period) * len);
    *edge = 4.0 * n_edge / (static_cast<double>(period) * len);
}

// S of the model, with a compute floor added here: `compute` is the plain
// step's time per update over its DRAM streaming time (0: memory-bound, the
// reference's model unchanged).  A round's time per valid update is then the
// larger of its memory time D / h and its compute time compute / h (the
// halo cells are computed too), against max(1, compute) for plain streaming:
//   S = h max(1, compute) / max(D, compute),  D = (1 + alpha h) / (2 I) + lambda (1 - 1/I).
double speedup(int bx, int by, int bz, int i, double lambda, double gamma, double l2, double cell_bytes,
               bool with_alpha, double compute, double tile_cost = -1)
{
    const double r = i - 1;
    const double h = (1 - 2 * r / bx) * (1 - 2 * r / by) * (1 - 2 * r / bz);
    double alpha = 1.0;
    if (with_alpha) {
        double bs, be;
        beta(bx, i, &bs, &be);
        const double v = cell_bytes * bx * by * bz;
        const double p = v < l2 ? 1.0 - std::exp(-v / (l2 - v)) : 0.0;
        alpha = 1 + lambda * (bs - 1) + p * (2 * gamma - (1 + lambda)) * be;
    }
    const double D = (1 + alpha * h) / (2.0 * i) + lambda * (1 - 1.0 / i);
    // tile_cost >= 0: a tile step's own cost per computed cell, apart from
    // the plain step's (predicted_speedup_b200)
    return h * std::max(1.0, compute) / std::max(D, tile_cost >= 0 ? tile_cost : compute);
}

// The measured plain and tile step costs of a storage format on B200 (FP64:
// none measured, the model as it is).
void b200_costs(int32_t storage, double* plain, double* tile)
{
    const bool is16 = storage == CULBM_STORAGE_F16 || storage == CULBM_STORAGE_BF16 ||
                      storage == CULBM_STORAGE_F16_SR || storage == CULBM_STORAGE_BF16_SR;
    *plain = is16 ? CULBM_B200_COMPUTE_16 : storage == CULBM_STORAGE_F32 ? CULBM_B200_PLAIN_32 : 0.0;
    *tile = is16 ? CULBM_B200_TILE_16 : storage == CULBM_STORAGE_F32 ? CULBM_B200_TILE_32 : 0.0;
}

// The compute floor of a storage format on B200: 16-bit steps are bound by
// instruction issue (CULBM_B200_COMPUTE_16), FP32 and FP64 by memory.
double compute_of(int32_t storage)
{
    return (storage == CULBM_STORAGE_F16 || storage == CULBM_STORAGE_BF16 || storage == CULBM_STORAGE_F16_SR ||
            storage == CULBM_STORAGE_BF16_SR)
               ? CULBM_B200_COMPUTE_16
               : 0.0;
}

culbm_status resolve_constants(double& lambda, double& gamma)
{
    if (!(lambda > 0)) lambda = CULBM_B200_LAMBDA;
    if (!(gamma > 0)) gamma = CULBM_B200_GAMMA;
    if (!(lambda > 0) || !(gamma > 0)) return fail(CULBM_ERR_INVALID_ARGUMENT, "lambda and gamma must be positive");
    return CULBM_OK;
}

culbm_status resolve_l2(uint64_t& l2_bytes, uint64_t* persist_bytes)
{
    if (l2_bytes && (!persist_bytes || *persist_bytes)) return CULBM_OK;
    int dev = 0, v = 0;
    CULBM_CUDA(cudaGetDevice(&dev));
    if (l2_bytes == 0) {
        CULBM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, dev));
        l2_bytes = static_cast<uint64_t>(v);
    }
    if (persist_bytes && *persist_bytes == 0) {
        CULBM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxPersistingL2CacheSize, dev));
        *persist_bytes = static_cast<uint64_t>(v);
    }
    return CULBM_OK;
}

double cell_bytes_of(int32_t storage)
{
    const double esize = storage == CULBM_STORAGE_F64 ? 8 : storage == CULBM_STORAGE_F32 ? 4 : 2;
    return 27 * esize;
}

}  // namespace

extern "C" {

culbm_status culbm_measure_memory(int32_t dev, culbm_memory_constants* out)
{
    if (!out) return fail(CULBM_ERR_INVALID_ARGUMENT, "out is NULL");
    std::memset(out, 0, sizeof(*out));
    CULBM_CUDA(cudaSetDevice(dev));
    int l2 = 0, sms = 0;
    CULBM_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    CULBM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t dram_bytes = (3ull * l2) / 256 * 256, l2_bytes = (static_cast<size_t>(l2) / 4) / 256 * 256;
    const long long units = 1ll << 23;   // 1 GiB of 128-byte units
    float *a = nullptr, *b = nullptr, *c = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto body = [&]() -> culbm_status {
        CULBM_CUDA(cudaMalloc(&a, dram_bytes));
        CULBM_CUDA(cudaMalloc(&b, dram_bytes));
        CULBM_CUDA(cudaMalloc(&c, units * 128));
        CULBM_CUDA(cudaMemset(a, 0, dram_bytes));
        CULBM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CULBM_CUDA(cudaEventCreate(&e0));
        CULBM_CUDA(cudaEventCreate(&e1));
        const int blocks = sms * kMeasureBlocksPerSm;
        const double target = 8.0 * (1ull << 30);   // bytes moved per timed launch
        float ms = 0;
        for (int which = 0; which < 2; ++which) {
            const size_t bytes = which ? l2_bytes : dram_bytes;
            const int passes = std::max(1, static_cast<int>(target / (2.0 * bytes)));
            const long long count = static_cast<long long>(bytes / sizeof(float4));
            CULBM_TRY(median_ms(s, e0, e1, 11, [&] {
                k_copy_cg<<<blocks, kMeasureThreads, 0, s>>>(reinterpret_cast<float4*>(b),
                                                             reinterpret_cast<const float4*>(a), count, passes);
            }, &ms));
            (which ? out->l2_gbs : out->dram_gbs) = 2.0 * bytes * passes / (ms * 1e6);
        }
        out->lambda = out->dram_gbs / out->l2_gbs;
        CULBM_TRY(median_ms(s, e0, e1, 11, [&] { k_store_units<false><<<blocks, kMeasureThreads, 0, s>>>(c, units); },
                            &ms));
        out->full_store_ms = ms;
        CULBM_TRY(median_ms(s, e0, e1, 11, [&] { k_store_units<true><<<blocks, kMeasureThreads, 0, s>>>(c, units); },
                            &ms));
        out->partial_store_ms = ms;
        out->gamma = 4.0 * out->partial_store_ms / out->full_store_ms - 3.0;
        out->l2_bytes = static_cast<uint64_t>(l2);
        return CULBM_OK;
    };
    const culbm_status st = body();
    if (s) cudaStreamSynchronize(s);
    cudaFree(a);
    cudaFree(b);
    cudaFree(c);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    return st;
}

culbm_status culbm_select_tile(const uint32_t domain_dim[3], int32_t storage, double lambda, double gamma,
                               uint64_t l2_bytes, uint64_t persist_bytes, culbm_tile_choice* out)
{
    if (!domain_dim || !out) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    CULBM_TRY(resolve_constants(lambda, gamma));
    CULBM_TRY(resolve_l2(l2_bytes, &persist_bytes));
    const double cell_bytes = cell_bytes_of(storage);
    const double compute = compute_of(storage);
    const double l2 = static_cast<double>(l2_bytes);
    double best = -1;
    // tile widths: the reference's multiples of 32 up to 160, and whole rows
    // (Bx = nx) when the domain is wider
    std::vector<int> widths = {32, 64, 96, 128, 160};
    if (domain_dim[0] > 160) widths.push_back(static_cast<int>(domain_dim[0]));
    for (int i = 2; i <= 20; ++i)
        for (int bx : widths) {
            if (bx <= 2 * (i - 1)) continue;
            for (int bz = 2 * (i - 1) + 1; bz <= 160; ++bz)
                for (int by = bz; by <= 160; ++by) {
                    if (cell_bytes * bx * by * bz > static_cast<double>(persist_bytes)) break;
                    const uint32_t b[3] = {static_cast<uint32_t>(bx), static_cast<uint32_t>(by),
                                           static_cast<uint32_t>(bz)};
                    bool ok = true;
                    for (int k = 0; k < 3 && ok; ++k) ok = valid_blk_axis(domain_dim[k], b[k], static_cast<uint32_t>(i));
                    if (!ok) continue;
                    const double sp = speedup(bx, by, bz, i, lambda, gamma, l2, cell_bytes, true, compute);
                    if (sp > best) {
                        best = sp;
                        for (int k = 0; k < 3; ++k) out->tile[k] = b[k];
                        out->inner_loop = i;
                        out->predicted_speedup = sp;
                        out->predicted_speedup_no_alignment =
                            speedup(bx, by, bz, i, lambda, gamma, l2, cell_bytes, false, compute);
                    }
                }
        }
    if (best < 0) return fail(CULBM_ERR_INVALID_ARGUMENT, "no tile of the model's range fits this domain");
    double plain_cost, tile_cost;
    b200_costs(storage, &plain_cost, &tile_cost);
    out->predicted_speedup_b200 = speedup(static_cast<int>(out->tile[0]), static_cast<int>(out->tile[1]),
                                          static_cast<int>(out->tile[2]), out->inner_loop, lambda, gamma, l2,
                                          cell_bytes, true, plain_cost, tile_cost);
    return CULBM_OK;
}

culbm_status culbm_blocking_speedup(const uint32_t tile[3], int32_t inner_loop, int32_t storage, double lambda,
                                    double gamma, uint64_t l2_bytes, double* speedup_out, double* speedup_no_alignment)
{
    if (!tile || !speedup_out) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (inner_loop < 1 || tile[0] < 1 || tile[1] < 1 || tile[2] < 1)
        return fail(CULBM_ERR_INVALID_ARGUMENT, "tile and innerLoop must be positive");
    CULBM_TRY(resolve_constants(lambda, gamma));
    CULBM_TRY(resolve_l2(l2_bytes, nullptr));
    const int bx = static_cast<int>(tile[0]), by = static_cast<int>(tile[1]), bz = static_cast<int>(tile[2]);
    const double cb = cell_bytes_of(storage), l2 = static_cast<double>(l2_bytes), c = compute_of(storage);
    *speedup_out = speedup(bx, by, bz, inner_loop, lambda, gamma, l2, cb, true, c);
    if (speedup_no_alignment) *speedup_no_alignment = speedup(bx, by, bz, inner_loop, lambda, gamma, l2, cb, false, c);
    return CULBM_OK;
}

}  // extern "C"
