// culbm_mass_momentum_noalloc: the FP64 mass/momentum reduction of
// culbm_mass_momentum (sim.cu, k_mass_momentum + k_sum_partials) over a
// caller-owned FP32 population buffer, with its block partial sums in a
// fixed file-scope device array instead of memory from cudaMalloc.  No
// reference counterpart.  It is for callers that must not allocate device
// memory: a framework process (PyTorch, say) whose device memory belongs to
// its caching allocator, where cudaMalloc would take memory behind the
// allocator's back and cudaMalloc/cudaFree synchronise the device.
//
// Work split: thread block b covers cells [b * kCellsPerBlock, (b + 1) *
// kCellsPerBlock), thread t of it the cells b * kCellsPerBlock + t + 256 k.
// The block count therefore depends on n alone, so the summation order, and
// the result, are the same on every device.  Every partial slot that the sum
// kernel reads is written by the first kernel of the same call, and the sum
// kernel writes the four result slots: nothing has to start at zero.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "sim_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr long long kCellsPerThread = 256;
constexpr long long kCellsPerBlock = kThreads * kCellsPerThread;
constexpr int kMaxBlocks = 1184;
static_assert(kMaxBlocks * kCellsPerBlock == CULBM_NOALLOC_MAX_CELLS, "limit in culbm.h");

// 4 partial sums per block, then the 4 results: 37,920 bytes.
static __device__ __align__(256) double g_noalloc_scratch[4 * kMaxBlocks + 4];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kThreads) k_mass_momentum_noalloc(const float* ddf, long long n, double* partial)
{
    double acc[4] = {0, 0, 0, 0};
    const long long base = blockIdx.x * kCellsPerBlock + threadIdx.x;
    for (long long k = 0; k < kCellsPerThread; ++k) {
        const long long i = base + k * kThreads;
        if (i >= n) break;
        double r = 1.0, mx = 0, my = 0, mz = 0;
        for (int d = 0; d < 27; ++d) {
            const double v = static_cast<double>(ddf[d * n + i]);
            r += v;
            mx += culbm::cx_of(d) * v;
            my += culbm::cy_of(d) * v;
            mz += culbm::cz_of(d) * v;
        }
        acc[0] += r;
        acc[1] += mx;
        acc[2] += my;
        acc[3] += mz;
    }
    __shared__ double sh[4][kThreads];
    for (int c = 0; c < 4; ++c) sh[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 4; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 4; ++c) partial[4 * blockIdx.x + c] = sh[c][0];
}

__global__ void k_sum_partials_noalloc(const double* partial, int nblocks, double* out)
{
    if (threadIdx.x < 4) {
        double s = 0;
        for (int b = 0; b < nblocks; ++b) s += partial[4 * b + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached.
culbm_status scratch_on_current_device(double** out)
{
    int dev = 0;
    CULBM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return culbm::fail(CULBM_ERR_UNSUPPORTED, "device ordinal " + std::to_string(dev) + " above " +
                                                      std::to_string(kMaxDevices - 1));
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        CULBM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return CULBM_OK;
}

}  // namespace

extern "C" culbm_status culbm_mass_momentum_noalloc(const float* d_ddf, uint64_t n, void* stream, double out[4])
{
    if (d_ddf == nullptr || out == nullptr) return culbm::fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return culbm::fail(CULBM_ERR_INVALID_ARGUMENT, "n must be positive");
    if (n > CULBM_NOALLOC_MAX_CELLS)
        return culbm::fail(CULBM_ERR_INVALID_ARGUMENT,
                           "culbm_mass_momentum_noalloc: " + std::to_string(n) + " cells exceed its limit of " +
                               std::to_string(CULBM_NOALLOC_MAX_CELLS) +
                               " (the partial sums live in a fixed 37,920-byte device array)");
    double* scratch = nullptr;
    CULBM_TRY(scratch_on_current_device(&scratch));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = static_cast<int>((static_cast<long long>(n) + kCellsPerBlock - 1) / kCellsPerBlock);
    double* result = scratch + 4 * kMaxBlocks;
    k_mass_momentum_noalloc<<<blocks, kThreads, 0, s>>>(d_ddf, static_cast<long long>(n), scratch);
    CULBM_CUDA(cudaGetLastError());
    k_sum_partials_noalloc<<<1, 32, 0, s>>>(scratch, blocks, result);
    CULBM_CUDA(cudaGetLastError());
    CULBM_CUDA(cudaMemcpyAsync(out, result, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CULBM_CUDA(cudaStreamSynchronize(s));
    return CULBM_OK;
}
