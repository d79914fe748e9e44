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
#include <cuda.h>
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

// The scratch address is kept per device together with the unique ID of the
// context it was looked up in.  A context made after cudaDeviceReset, or one
// made with cuCtxCreate, may place the array elsewhere: its ID differs, so
// the address is looked up again in it before any launch.
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    double* ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points, so
// the library needs no link against libcuda.
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;

// ID of the context current on this thread; 0 when none is current yet.
culbm_status current_context_id(unsigned long long* id)
{
    if (g_ctx_get_current == nullptr || g_ctx_get_id == nullptr) {
        void* fc = nullptr;
        void* fi = nullptr;
        cudaDriverEntryPointQueryResult qc{}, qi{};
        CULBM_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fc, 12000, cudaEnableDefault, &qc));
        CULBM_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetId", &fi, 12000, cudaEnableDefault, &qi));
        if (qc != cudaDriverEntryPointSuccess || qi != cudaDriverEntryPointSuccess || !fc || !fi)
            return culbm::fail(CULBM_ERR_CUDA, "culbm_mass_momentum_noalloc: driver lacks cuCtxGetId");
        g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(fc);
        g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(fi);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS)
        return culbm::fail(CULBM_ERR_CUDA, "culbm_mass_momentum_noalloc: cuCtxGetCurrent failed");
    *id = 0;
    if (ctx != nullptr && g_ctx_get_id(ctx, id) != CUDA_SUCCESS)
        return culbm::fail(CULBM_ERR_CUDA, "culbm_mass_momentum_noalloc: cuCtxGetId failed");
    return CULBM_OK;
}

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

// Device address of the scratch array in the current context: looked up
// (cudaGetSymbolAddress, with the device current) on the first call in each
// context, then reused while that context stays current.
culbm_status scratch_on_current_device(double** out)
{
    int dev = 0;
    CULBM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return culbm::fail(CULBM_ERR_UNSUPPORTED, "device ordinal " + std::to_string(dev) + " above " +
                                                      std::to_string(kMaxDevices - 1));
    std::lock_guard<std::mutex> lock(g_mutex);
    unsigned long long id = 0;
    CULBM_TRY(current_context_id(&id));
    if (id == 0 || g_scratch[dev].ptr == nullptr || g_scratch[dev].ctx_id != id) {
        // Also makes the device's primary context current when none is yet.
        void* p = nullptr;
        CULBM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        CULBM_TRY(current_context_id(&id));
        g_scratch[dev].ctx_id = id;
        g_scratch[dev].ptr = static_cast<double*>(p);
    }
    *out = g_scratch[dev].ptr;
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
