// Host runtime behind include/culbm.h: configuration checks, device
// allocation, init-state loading, step dispatch, dumps and reductions.
//
// Replaces the reference's Simulator / Simulator::Data
// (src/simulator/single_dev_expt/simulator_expt_platform.cu) minus argv
// parsing, which single_dev_expt_main does on top of this ABI.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <string>
#include <type_traits>
#include <vector>

#include "row_kernels.cuh"
#include "warp_kernels.cuh"
#include "sim_internal.cuh"

namespace culbm {

namespace {
thread_local std::string t_last_error;
std::atomic<int> g_inject_skip{0};
std::atomic<int> g_inject_code{0};
std::atomic<int> g_row_extra_tx{0};
}  // namespace

void set_last_error(const std::string& msg) { t_last_error = msg; }

culbm_status fail(culbm_status s, const std::string& msg)
{
    t_last_error = msg;
    return s;
}

cudaError_t injection_gate()
{
    const int code = g_inject_code.load();
    if (code == 0) return cudaSuccess;
    const int left = g_inject_skip.fetch_sub(1);
    if (left > 0) return cudaSuccess;
    int expected = code;
    if (g_inject_code.compare_exchange_strong(expected, 0)) return static_cast<cudaError_t>(code);
    return cudaSuccess;
}

culbm_status cuda_fail(cudaError_t e, const char* what, const char* file, int line)
{
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %d (%s: %s) in %s at %s:%d", static_cast<int>(e),
                  cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
    t_last_error = buf;
    return e == cudaErrorMemoryAllocation ? CULBM_ERR_OUT_OF_MEMORY : CULBM_ERR_CUDA;
}

// ------------------------------------------------------------ utilities ---

template <typename S>
StepArgs<S, typename ArithOf<S>::type> make_args(const culbm_sim* s, int src, int dst)
{
    using R = typename ArithOf<S>::type;
    StepArgs<S, R> a{};
    long long stride = s->n;
    if (is_blocked(s->cfg)) tiles_view(s, &a.ring_nz, &a.ring_off, &stride);
    a.dom = s->dom;
    a.ops = s->d_ops;
    a.rho = s->d_mac[0];
    a.vx = s->d_mac[1];
    a.vy = s->d_mac[2];
    a.vz = s->d_mac[3];
    a.inv_tau = static_cast<R>(s->cfg.inv_tau);
    S* b0 = static_cast<S*>(s->d_pop[src]);
    S* b1 = static_cast<S*>(s->d_pop[dst]);
    a.src.set(b0, stride);
    a.dst.set(b1, stride);
    a.edge = static_cast<S*>(s->d_edge);
    a.el = s->el;
    a.seed = step_seed(static_cast<uint32_t>(s->step));
    return a;
}

// Layout of the newest state and the buffer holding it.
int current_layout(const culbm_sim* s)
{
    if (s->cfg.stream_policy == CULBM_STREAM_INPLACE && !is_blocked(s->cfg))
        return s->aa_phase == 0 ? LAYOUT_AA_A : LAYOUT_AA_B;
    if (is_blocked(s->cfg) && s->cfg.use_ring_ddf_buf) return LAYOUT_PULL_RING;
    return LAYOUT_PULL;
}

// Calls f(std::integral_constant<int, layout>{}).
template <class F>
void with_layout(int layout, F&& f)
{
    switch (layout) {
        case LAYOUT_AA_A: f(std::integral_constant<int, LAYOUT_AA_A>{}); break;
        case LAYOUT_AA_B: f(std::integral_constant<int, LAYOUT_AA_B>{}); break;
        case LAYOUT_PULL_RING: f(std::integral_constant<int, LAYOUT_PULL_RING>{}); break;
        default: f(std::integral_constant<int, LAYOUT_PULL>{}); break;
    }
}

size_t storage_bytes(int storage)
{
    switch (storage) {
        case CULBM_STORAGE_F16:
        case CULBM_STORAGE_BF16:
        case CULBM_STORAGE_F16_SR:
        case CULBM_STORAGE_BF16_SR: return 2;
        case CULBM_STORAGE_F64: return 8;
        default: return 4;
    }
}

culbm_status dev_alloc(culbm_sim* s, void** p, size_t bytes, const char* what)
{
    cudaError_t e = injection_gate();
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        char buf[256];
        std::snprintf(buf, sizeof(buf), "device allocation of %zu bytes for %s failed: %s", bytes, what,
                      cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? CULBM_ERR_OUT_OF_MEMORY : CULBM_ERR_CUDA, buf);
    }
    s->device_bytes += bytes;
    return CULBM_OK;
}

// Builds the compact op bytes from the flag words: step bits plus OP_EDGE on
// the domain boundary.
__global__ void k_build_ops(Domain D, const uint32_t* flag, uint8_t* ops, int z0)
{
    const CellCoord c = cell_of_thread(D, z0);
    if (!c.valid) return;
    const uint32_t fl = flag[c.i];
    uint8_t op = static_cast<uint8_t>(fl & 0x1Fu);
    if (c.x == 0 || c.x == D.nx - 1 || c.y == 0 || c.y == D.ny - 1 || c.z == 0 || c.z == D.nz - 1) op |= OP_EDGE;
    ops[c.i] = op;
}

__global__ void k_fill_u32(uint32_t* p, long long n, uint32_t v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void k_fill_f32(float* p, long long n, float v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

// FP64 mass/momentum partial sums, one set of 4 per block, fixed order.
template <int LAYOUT, typename S, typename R>
__global__ void __launch_bounds__(256) k_mass_momentum(const __grid_constant__ StepArgs<S, R> a, double* partial)
{
    const Domain& D = a.dom;
    double acc[4] = {0, 0, 0, 0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < D.n; t += (long long)gridDim.x * blockDim.x) {
        const int i = static_cast<int>(t);
        const uint8_t op = a.ops[i];
        if ((op & (OP_LOAD | OP_EQU)) == 0) continue;
        const int x = i % D.nx, y = (i / D.nx) % D.ny, z = i / D.nxy;
        R f[27];
        load_pulled<LAYOUT>(a, x, y, z, i, (op & OP_EDGE) != 0, f);
        double r = 1.0, mx = 0, my = 0, mz = 0;
        for (int d = 0; d < 27; ++d) {
            const double v = static_cast<double>(f[d]);
            r += v;
            mx += cx_of(d) * v;
            my += cy_of(d) * v;
            mz += cz_of(d) * v;
        }
        acc[0] += r;
        acc[1] += mx;
        acc[2] += my;
        acc[3] += mz;
    }
    __shared__ double sh[4][256];
    for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) partial[4 * blockIdx.x + k] = sh[k][0];
}

__global__ void k_sum_partials(const double* partial, int nblocks, double* out)
{
    if (threadIdx.x < 4) {
        double s = 0;
        for (int b = 0; b < nblocks; ++b) s += partial[4 * b + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

constexpr uint32_t kDefaultFlag =
    FLAG_LOAD | FLAG_COLLIDE | FLAG_STORE | FLAG_DUMP_RHO | FLAG_DUMP_VX | FLAG_DUMP_VY | FLAG_DUMP_VZ;

// Rest-equilibrium fill of the population state in its start layout.
template <typename S>
culbm_status fill_rest(culbm_sim* s)
{
    using R = typename ArithOf<S>::type;
    if (is_blocked(s->cfg)) return tiles_reset(s);
    const dim3 g = cell_grid(s->dom), b = cell_block();
    for (int k = 0; k < s->npop; ++k) {
        auto a = make_args<S>(s, k, k);
        if (s->cfg.stream_policy == CULBM_STREAM_INPLACE && !is_blocked(s->cfg))
            k_fill_equilibrium<LAYOUT_AA_A, S, R><<<g, b, 0, s->stream>>>(a, R(1), R(0), R(0), R(0));
        else
            k_fill_equilibrium<LAYOUT_PULL, S, R><<<g, b, 0, s->stream>>>(a, R(1), R(0), R(0), R(0));
        CULBM_CUDA(cudaGetLastError());
    }
    s->cur = 0;
    s->aa_phase = 0;
    return CULBM_OK;
}

culbm_status check_device_error(culbm_sim* s)
{
    if (s->err_host == nullptr) return CULBM_OK;
    const int e = *reinterpret_cast<volatile int*>(s->err_host);
    if (e == 0) return CULBM_OK;
    *reinterpret_cast<volatile int*>(s->err_host) = 0;
    return fail(CULBM_ERR_DEVICE_TIMEOUT,
                "a bounded wait of the row-staged step kernel gave up (its bulk copies did not complete); "
                "the state of that step is not valid");
}

// The row-staged kernels (kernel_variant 1 and 2) serve the plain policies
// with 16-bit storage when rows are 16-byte aligned (nx a multiple of 16),
// fit one block (nx <= 992) and, in place, the domain has inner rows.
// Variant 1 stages two rows per block with one output buffer, variant 2
// with two output buffers.
bool rows_applicable(const culbm_sim* s)
{
    const Domain& D = s->dom;
    if (is_blocked(s->cfg) || s->esize != 2) return false;
    if (s->cfg.kernel_variant != 1 && s->cfg.kernel_variant != 2) return false;
    if (D.nx % 16 != 0 || D.nx < 32 || D.nx > 992) return false;
    if (s->cfg.stream_policy == CULBM_STREAM_INPLACE && (D.ny < 3 || D.nz < 3)) return false;
    return true;
}

// Calls f(stages, output buffers, L2 prefetch rows as integral constants)
// for the sim's pipeline shape.
template <class F>
culbm_status with_row_shape(const culbm_sim* s, F&& f)
{
    using std::integral_constant;
    if (s->cfg.kernel_variant == 2)
        return f(integral_constant<int, 2>{}, integral_constant<int, 2>{}, integral_constant<int, 0>{});
    return f(integral_constant<int, 2>{}, integral_constant<int, 1>{}, integral_constant<int, 0>{});
}

template <typename S, int MODE, int NS, int OB, int PF>
culbm_status rows_prepare(culbm_sim* s)
{
    const RowSmem L = row_smem_layout<S, NS, OB>(s->dom.nx);
    const int threads = (row_consumer_warps(s->dom.nx) + 1) * 32;
    auto kern = k_rows16<S, MODE, NS, OB, PF>;
    CULBM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total));
    int per_sm = 0, sms = 0;
    CULBM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, L.total));
    CULBM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->dev));
    if (per_sm < 1) return fail(CULBM_ERR_UNSUPPORTED, "row-staged step kernel does not fit an SM");
    s->row_grid[MODE] = per_sm * sms;
    return CULBM_OK;
}

template <typename S>
culbm_status rows_setup(culbm_sim* s)
{
    if constexpr (Is16<S>::value) {
        CULBM_TRY(with_row_shape(s, [&](auto ns, auto ob, auto pf) -> culbm_status {
            constexpr int NS = decltype(ns)::value, OB = decltype(ob)::value, PF = decltype(pf)::value;
            if (s->cfg.stream_policy == CULBM_STREAM_PULL) {
                CULBM_TRY((rows_prepare<S, ROWS_PULL, NS, OB, PF>(s)));
            } else {
                CULBM_TRY((rows_prepare<S, ROWS_AA_ODD, NS, OB, PF>(s)));
                CULBM_TRY((rows_prepare<S, ROWS_AA_EVEN, NS, OB, PF>(s)));
            }
            return CULBM_OK;
        }));
        s->rows = true;
    }
    return CULBM_OK;
}

// One row-staged launch over the rows [y0, y0 + ry) x [z0, z0 + rz).
template <typename S, int MODE>
culbm_status rows_launch(culbm_sim* s, const StepArgs<S, float>& a, int y0, int z0, int ry, int rz)
{
    RowArgs<S> ra{};
    ra.s = a;
    ra.y0 = y0;
    ra.z0 = z0;
    ra.ry = ry;
    ra.rz = rz;
    ra.nrows = ry * rz;
    ra.err = s->err_dev;
    ra.debug_extra_tx = g_row_extra_tx.load();
    const int grid = std::min(ra.nrows, s->row_grid[MODE]);
    const int threads = (row_consumer_warps(s->dom.nx) + 1) * 32;
    return with_row_shape(s, [&](auto ns, auto ob, auto pf) -> culbm_status {
        constexpr int NS = decltype(ns)::value, OB = decltype(ob)::value, PF = decltype(pf)::value;
        const RowSmem L = row_smem_layout<S, NS, OB>(s->dom.nx);
        k_rows16<S, MODE, NS, OB, PF><<<grid, threads, L.total, s->stream>>>(ra);
        CULBM_CUDA(cudaGetLastError());
        return CULBM_OK;
    });
}

// The warp-staged 16-bit pull (warp_kernels.cuh, kernel_variant 3 with two
// window buffers per warp, 4 with three): plain pull with 16-bit storage and
// nx a multiple of 8.
bool warp_pull_applicable(const culbm_sim* s)
{
    return !is_blocked(s->cfg) && s->esize == 2 && (s->cfg.kernel_variant == 3 || s->cfg.kernel_variant == 4) &&
           s->cfg.stream_policy == CULBM_STREAM_PULL && s->dom.nx % 8 == 0;
}

using PfnEncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The population buffer `base` as the 4-D tensor (x, y, z, d) of 16-bit
// values with the given box.
culbm_status encode_pop_map(const culbm_sim* s, void* base, const cuuint32_t box[4], CUtensorMap* out)
{
    static PfnEncodeTiled encode = nullptr;
    if (encode == nullptr) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CULBM_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || fn == nullptr)
            return fail(CULBM_ERR_CUDA, "driver lacks cuTensorMapEncodeTiled");
        encode = reinterpret_cast<PfnEncodeTiled>(fn);
    }
    const Domain& D = s->dom;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(D.nx), static_cast<cuuint64_t>(D.ny),
                                static_cast<cuuint64_t>(D.nz), 27};
    const cuuint64_t strides[3] = {2ull * D.nx, 2ull * D.nxy, 2ull * s->n};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, base, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CULBM_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(r));
    return CULBM_OK;
}

template <typename S, int NB>
culbm_status warp_pull_prepare(culbm_sim* s)
{
    const int smem = kWarpWarps * warp_smem_per_warp(NB);
    CULBM_CUDA(cudaFuncSetAttribute(k_pull16_warp<S, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0, sms = 0;
    CULBM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pull16_warp<S, NB>, kWarpWarps * 32, smem));
    CULBM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->dev));
    if (per_sm < 1) return fail(CULBM_ERR_UNSUPPORTED, "warp-staged pull kernel does not fit an SM");
    s->row_grid[ROWS_PULL] = per_sm * sms;
    return CULBM_OK;
}

template <typename S>
culbm_status warp_pull_setup(culbm_sim* s)
{
    if constexpr (Is16<S>::value) {
        if (s->cfg.kernel_variant == 4) {
            CULBM_TRY((warp_pull_prepare<S, 3>(s)));
        } else {
            CULBM_TRY((warp_pull_prepare<S, 2>(s)));
        }
        const cuuint32_t load_box[4] = {kWarpWin, 1, 1, 3}, store_box[4] = {32, 1, 1, 27};
        for (int k = 0; k < 2; ++k) {
            CULBM_TRY(encode_pop_map(s, s->d_pop[k], load_box, &s->map_load[k]));
            CULBM_TRY(encode_pop_map(s, s->d_pop[k], store_box, &s->map_store[k]));
        }
        s->warp_pull = true;
    }
    return CULBM_OK;
}

template <typename S>
culbm_status plain_steps(culbm_sim* s, uint32_t nsteps)
{
    using R = typename ArithOf<S>::type;
    const dim3 g = cell_grid(s->dom), b = cell_block();
    for (uint32_t k = 0; k < nsteps; ++k) {
        const uint32_t seed = step_seed(static_cast<uint32_t>(s->step + k));
        if constexpr (Is16<S>::value) {
            if (s->warp_pull) {
                auto a = make_args<S>(s, s->cur, 1 - s->cur);
                a.seed = seed;
                WarpArgs16 w{};
                w.nseg_row = (s->dom.nx + 31) / 32;
                w.nseg = w.nseg_row * s->dom.ny * s->dom.nz;
                w.err = s->err_dev;
                w.debug_extra_tx = g_row_extra_tx.load();
                WarpMaps maps;
                maps.src = s->map_load[s->cur];
                maps.dst = s->map_store[1 - s->cur];
                const int blocks = (w.nseg + kWarpWarps - 1) / kWarpWarps;
                const int grid = std::min(blocks, s->row_grid[ROWS_PULL]);
                if (s->cfg.kernel_variant == 4)
                    k_pull16_warp<S, 3><<<grid, kWarpWarps * 32, kWarpWarps * warp_smem_per_warp(3), s->stream>>>(
                        a, maps, w);
                else
                    k_pull16_warp<S, 2><<<grid, kWarpWarps * 32, kWarpWarps * warp_smem_per_warp(2), s->stream>>>(
                        a, maps, w);
                CULBM_CUDA(cudaGetLastError());
                s->cur ^= 1;
                s->launches += 1;
                continue;
            }
            if (s->rows) {
                const Domain& D = s->dom;
                if (s->cfg.stream_policy == CULBM_STREAM_PULL) {
                    auto a = make_args<S>(s, s->cur, 1 - s->cur);
                    a.seed = seed;
                    CULBM_TRY((rows_launch<S, ROWS_PULL>(s, a, 0, 0, D.ny, D.nz)));
                    s->cur ^= 1;
                    s->launches += 1;
                } else {
                    // face rows with the per-cell kernel (the outer slices of
                    // split_grid), inner rows row-staged; disjoint locations
                    auto a = make_args<S>(s, 0, 0);
                    a.seed = seed;
                    const dim3 gs = split_grid(D, AaShape<S>::rows, AaShape<S>::cols);
                    const dim3 go(gs.x, gs.y, outer_slices(D, AaShape<S>::rows));
                    if (s->aa_phase == 0) {
                        k_aa_odd<S, R><<<go, aa_block<S>(), 0, s->stream>>>(a);
                        CULBM_CUDA(cudaGetLastError());
                        CULBM_TRY((rows_launch<S, ROWS_AA_ODD>(s, a, 1, 1, D.ny - 2, D.nz - 2)));
                    } else {
                        k_aa_even<S, R><<<go, aa_block<S>(), 0, s->stream>>>(a);
                        CULBM_CUDA(cudaGetLastError());
                        CULBM_TRY((rows_launch<S, ROWS_AA_EVEN>(s, a, 1, 1, D.ny - 2, D.nz - 2)));
                    }
                    s->aa_phase ^= 1;
                    s->launches += 2;
                }
                continue;
            }
        }
        if (s->cfg.stream_policy == CULBM_STREAM_PULL) {
            auto a = make_args<S>(s, s->cur, 1 - s->cur);
            a.seed = seed;
            k_pull_step<S, R><<<g, b, 0, s->stream>>>(a, 0);
            CULBM_CUDA(cudaGetLastError());
            s->cur ^= 1;
        } else {
            auto a = make_args<S>(s, 0, 0);
            a.seed = seed;
            const dim3 gs = split_grid(s->dom, AaShape<S>::rows, AaShape<S>::cols);
            if (s->aa_phase == 0)
                k_aa_odd<S, R><<<gs, aa_block<S>(), 0, s->stream>>>(a);
            else
                k_aa_even<S, R><<<gs, aa_block<S>(), 0, s->stream>>>(a);
            CULBM_CUDA(cudaGetLastError());
            s->aa_phase ^= 1;
        }
        s->launches += 1;
    }
    return CULBM_OK;
}

culbm_status check_sim(culbm_sim* s, bool need_loaded = false)
{
    if (s == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "culbm_sim is NULL");
    if (need_loaded && !s->loaded) return fail(CULBM_ERR_STATE, "no state loaded");
    CULBM_CUDA(cudaSetDevice(s->dev));
    return CULBM_OK;
}

culbm_status validate_config(const culbm_config& c)
{
    for (int k = 0; k < 3; ++k) {
        if (c.domain_dim[k] == 0) return fail(CULBM_ERR_INVALID_ARGUMENT, "domainDim must be positive");
        if (c.block_dim[k] == 0 || c.grid_dim[k] == 0)
            return fail(CULBM_ERR_INVALID_ARGUMENT, "blockDim and gridDim must be positive");
    }
    const unsigned long long n = 1ull * c.domain_dim[0] * c.domain_dim[1] * c.domain_dim[2];
    if (n >= (1ull << 31)) return fail(CULBM_ERR_INVALID_ARGUMENT, "domain has 2^31 cells or more");
    if (c.domain_dim[2] > 65535) return fail(CULBM_ERR_INVALID_ARGUMENT, "domainDim z above 65535");
    if (c.stream_policy == CULBM_STREAM_INPLACE) {
        Domain d{};
        d.nx = static_cast<int>(c.domain_dim[0]);
        d.ny = static_cast<int>(c.domain_dim[1]);
        d.nz = static_cast<int>(c.domain_dim[2]);
        const bool s16 = c.storage == CULBM_STORAGE_F16 || c.storage == CULBM_STORAGE_BF16 ||
                         c.storage == CULBM_STORAGE_F16_SR || c.storage == CULBM_STORAGE_BF16_SR;
        const dim3 g = s16 ? split_grid(d, AaShape<__half>::rows, AaShape<__half>::cols)
                           : split_grid(d, AaShape<float>::rows, AaShape<float>::cols);
        if (g.z > 65535)
            return fail(CULBM_ERR_INVALID_ARGUMENT, "domainDim z too large for in-place streaming (grid z above 65535)");
        if (g.y > 65535)
            return fail(CULBM_ERR_INVALID_ARGUMENT, "domainDim y too large for in-place streaming (grid y above 65535)");
    }
    if (c.vel_set != 0) return fail(CULBM_ERR_INVALID_ARGUMENT, "Unsupport Velocity Set: " + std::to_string(c.vel_set));
    if (c.stream_policy != CULBM_STREAM_PULL && c.stream_policy != CULBM_STREAM_INPLACE)
        return fail(CULBM_ERR_INVALID_ARGUMENT, "streamPolicy must be 0 or 1");
    if (c.opt_policy < 0 || c.opt_policy > 3) return fail(CULBM_ERR_INVALID_ARGUMENT, "optPolicy must be 0..3");
    if (c.storage < 0 || c.storage > 5) return fail(CULBM_ERR_INVALID_ARGUMENT, "storage must be 0..5");
    if (c.run_slabs < 0) return fail(CULBM_ERR_INVALID_ARGUMENT, "run_slabs must be 0 (automatic) or positive");
    if (!(c.inv_tau > 0.0f && c.inv_tau < 2.0f))
        return fail(CULBM_ERR_INVALID_ARGUMENT, "invTau must lie in (0, 2)");
    // The reference rejects the ring buffer outside in-place dynamic L2
    // blocking (simulator_expt_platform.cu:365-368).
    if (c.use_ring_ddf_buf && !(c.stream_policy == CULBM_STREAM_INPLACE && c.opt_policy == CULBM_OPT_DYNAMIC_L2))
        return fail(CULBM_ERR_INVALID_ARGUMENT, "--useRingDDFBuf is unimplemented unless --streamPolicy 1 --optPolicy 3.");
    // The reference's plain pull launches one thread per cell with the user's
    // grid and requires it to cover the domain exactly (simulator_expt_platform.cu:962-967).
    if (c.stream_policy == CULBM_STREAM_PULL && c.opt_policy == CULBM_OPT_NONE)
        for (int k = 0; k < 3; ++k)
            if (1ull * c.block_dim[k] * c.grid_dim[k] != c.domain_dim[k])
                return fail(CULBM_ERR_INVALID_ARGUMENT, "Dimension of domain doesn't match computation grid!");
    if (is_blocked(c)) return validate_blocking(c);
    return CULBM_OK;
}

void release(culbm_sim* s)
{
    if (s == nullptr) return;
    cudaSetDevice(s->dev);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& st : s->slab_st)
        if (st) cudaStreamSynchronize(st);
    for (auto& st : s->copy_st)
        if (st) cudaStreamSynchronize(st);
    tiles_destroy(s);
    cudaFree(s->d_flag);
    cudaFree(s->d_ops);
    for (auto& p : s->d_mac) cudaFree(p);
    for (auto& p : s->d_pop) cudaFree(p);
    cudaFree(s->d_edge);
    cudaFree(s->d_red);
    for (auto& e : s->slab_ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : s->run_ev)
        if (e) cudaEventDestroy(e);
    for (auto& st : s->slab_st)
        if (st) cudaStreamDestroy(st);
    for (auto& st : s->copy_st)
        if (st) cudaStreamDestroy(st);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->err_host) cudaFreeHost(s->err_host);
    delete s;
}

culbm_status upload_state(culbm_sim* s, const uint32_t* flag, const float* const mac[4])
{
    const long long n = s->n;
    const dim3 g1(1184), b1(256);
    if (flag != nullptr) {
        CULBM_CUDA(cudaMemcpyAsync(s->d_flag, flag, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    } else {
        k_fill_u32<<<g1, b1, 0, s->stream>>>(s->d_flag, n, kDefaultFlag);
        CULBM_CUDA(cudaGetLastError());
    }
    const float dflt[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < 4; ++k) {
        if (mac[k] != nullptr) {
            CULBM_CUDA(cudaMemcpyAsync(s->d_mac[k], mac[k], n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        } else {
            k_fill_f32<<<g1, b1, 0, s->stream>>>(s->d_mac[k], n, dflt[k]);
            CULBM_CUDA(cudaGetLastError());
        }
    }
    k_build_ops<<<cell_grid(s->dom), cell_block(), 0, s->stream>>>(s->dom, s->d_flag, s->d_ops, 0);
    CULBM_CUDA(cudaGetLastError());
    if (is_blocked(s->cfg)) {
        std::vector<uint32_t> host;
        const uint32_t* hf = flag;
        if (hf == nullptr) {
            host.assign(static_cast<size_t>(n), kDefaultFlag);
            hf = host.data();
        }
        CULBM_TRY(tiles_upload_flags(s, hf));
    }
    CULBM_TRY(with_storage(s, [&](auto tag) { return fill_rest<typename decltype(tag)::type>(s); }));
    s->step = 0;
    s->loaded = true;
    return CULBM_OK;
}

// ------------------------------------------------- overlapped host run ---
//
// culbm_run_host cuts the domain into slabs of z-planes a_0 = 0 < a_1 < ...
// < a_m = nz, at least two planes each, and skews them in time: step t of
// slab j updates the planes [a_j - t', a_{j+1} - t') (clamped to the domain;
// t' counts the steps of the skewed phase; slab 0 starts at 0 and the last
// ends at nz).  A cell of a plain step reads and writes only locations
// within one plane of itself, so
//   step t of slab j reads what step t-1 wrote on its own region and on
//   slab j-1's (which holds the two planes below it): it waits for nothing
//   above, so slab 0 can take all its steps as soon as its inputs are in;
//   steps of one t on different slabs touch disjoint locations (each
//   location belongs to one cell per step), and so do step t on slab j and
//   step t-1 on slab j+1: in pull mode the write sets of t and the read sets
//   of t-1 above a_{j+1} - t' are disjoint, and in place one of the two
//   steps touches only its own planes;
//   the dump of slab j, on the region of the step after the last, waits for
//   the last step on slabs j and j-1.
// Events carry the dependencies.  One copy stream brings the slabs in, in
// slab order; the other takes each dump region out as it finishes, so the
// fields of low slabs leave while high slabs still step.  Only the first and
// the last steps of a long run go slab by slab; the steps in between are
// whole-domain launches.  The population start does not depend on the
// inputs (rest equilibrium, as culbm_load_state), so it runs on the
// simulation's stream while the first slab arrives.
//
// Order of submission.  A device runs the streams of a process on a few
// hardware queues (8 by default), and work that shares a queue starts in the
// order it was submitted.  The slabs' work is therefore spread over
// kRunStreams streams (slab j on stream j mod kRunStreams) and submitted by
// anti-diagonal d = j + t', then t': everything a task waits for has a
// smaller d.  Each slab's four step events are a ring: step t's event is
// waited on by step t+1 of slab j+1 (d + 2) before step t+4 records it again
// (d + 4).

constexpr int kSlabEvents = 6;   // per slab: a ring of 4 step events, inputs copied in, dump done
constexpr int kSlabIn = 4, kSlabDump = 5;
constexpr int kRunStreams = 4;

// Slab count: culbm_config.run_slabs, or automatic: runs of up to 40 steps
// (all skewed) take up to 64 slabs of at least 2^18 cells, so that the first
// slabs arrive early; longer runs up to 32 slabs of at least 2^19 cells,
// which keeps their two skewed phases short.  At most nz / 2 either way.
// (288x272x280, in place: 20 steps 19.9 ms with 64 slabs against 20.5 ms
// with 32; 100 steps 87.1 ms with 32 against 89.0 ms with 64.)
int run_slabs(const culbm_sim* s, uint32_t nsteps)
{
    const Domain& D = s->dom;
    long long want = s->cfg.run_slabs;
    if (want <= 0) want = nsteps <= 40 ? std::min<long long>(64, D.n >> 18) : std::min<long long>(32, D.n >> 19);
    return static_cast<int>(std::max<long long>(1, std::min<long long>(want, D.nz / 2)));
}

// First plane of slab j of nslab balanced slabs (slab_z0(nslab) = nz).
int slab_z0(const Domain& D, int nslab, int j)
{
    return static_cast<int>(static_cast<long long>(j) * D.nz / nslab);
}

// First plane of slab j's region `shift` steps into a skewed phase.
int slab_lo(const Domain& D, int nslab, int j, int shift)
{
    if (j <= 0) return 0;
    if (j >= nslab) return D.nz;
    return std::max(0, slab_z0(D, nslab, j) - shift);
}

culbm_status ensure_run_streams(culbm_sim* s, int nstream, int nslab)
{
    for (auto& st : s->copy_st)
        if (!st) CULBM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& e : s->run_ev)
        if (!e) CULBM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    while (static_cast<int>(s->slab_st.size()) < nstream) {
        cudaStream_t st = nullptr;
        CULBM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        s->slab_st.push_back(st);
    }
    while (static_cast<int>(s->slab_ev.size()) < nslab * kSlabEvents) {
        cudaEvent_t e = nullptr;
        CULBM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s->slab_ev.push_back(e);
    }
    return CULBM_OK;
}

// Submits the skewed steps t0 .. t1-1 slab by slab, with the op bytes of
// each slab's planes first when `build` and the dump of each slab's region
// after step t1 - 1 last when `dump`.  The first step waits for nothing from
// the neighbours: it follows the population start or a join of all slabs.
template <typename S>
culbm_status run_slab_steps(culbm_sim* s, int nslab, int nstream, int t0, int t1, bool build, bool dump)
{
    using R = typename ArithOf<S>::type;
    const Domain& D = s->dom;
    auto ev = [&](int j, int k) { return s->slab_ev[static_cast<size_t>(j) * kSlabEvents + k]; };
    auto planes = [&](int za, int zb) { return dim3((D.nx + 31) / 32, (D.ny + 7) / 8, zb - za); };
    const dim3 b = cell_block();
    const bool pull = s->cfg.stream_policy == CULBM_STREAM_PULL;

    struct Task {
        int d, t, j;   // t = t0 - 1: op bytes; t1: dump
    };
    std::vector<Task> tasks;
    tasks.reserve(static_cast<size_t>(nslab) * (t1 - t0 + 2));
    for (int j = 0; j < nslab; ++j)
        for (int t = build ? t0 - 1 : t0; t <= (dump ? t1 : t1 - 1); ++t) tasks.push_back({j + std::max(t - t0, 0), t, j});
    std::sort(tasks.begin(), tasks.end(), [](const Task& x, const Task& y) { return x.d != y.d ? x.d < y.d : x.t < y.t; });

    for (const Task& k : tasks) {
        const int j = k.j, t = k.t;
        cudaStream_t st = s->slab_st[j % nstream];
        if (t < t0) {
            const int za = slab_z0(D, nslab, j), zb = slab_z0(D, nslab, j + 1);
            CULBM_CUDA(cudaStreamWaitEvent(st, ev(j, kSlabIn), 0));
            k_build_ops<<<planes(za, zb), b, 0, st>>>(D, s->d_flag, s->d_ops, za);
            CULBM_CUDA(cudaGetLastError());
            continue;
        }
        // Step t - 1 on slab j - 1 (on slab j it is earlier on the same stream).
        if (t > t0 && j > 0 && (j - 1) % nstream != j % nstream)
            CULBM_CUDA(cudaStreamWaitEvent(st, ev(j - 1, (t - 1) & 3), 0));
        const int za = slab_lo(D, nslab, j, t - t0), zb = slab_lo(D, nslab, j + 1, t - t0);
        if (t == t1) {
            // Dump of the state after step t1 - 1, as culbm_moments.
            if (zb > za) {
                const int cur = pull ? t1 & 1 : 0;
                const int layout = pull ? LAYOUT_PULL : ((t1 & 1) == 0 ? LAYOUT_AA_A : LAYOUT_AA_B);
                auto a = make_args<S>(s, cur, cur);
                float* const* m = s->d_mac;
                with_layout(layout, [&](auto L) {
                    k_moments<decltype(L)::value, S, R><<<planes(za, zb), b, 0, st>>>(a, s->d_flag, m[0], m[1], m[2],
                                                                                    m[3], za);
                });
                CULBM_CUDA(cudaGetLastError());
            }
            CULBM_CUDA(cudaEventRecord(ev(j, kSlabDump), st));
            continue;
        }
        if (zb > za) {
            if (pull) {
                auto a = make_args<S>(s, t & 1, 1 - (t & 1));
                a.seed = step_seed(static_cast<uint32_t>(t));
                k_pull_step<S, R><<<planes(za, zb), b, 0, st>>>(a, za);
            } else {
                auto a = make_args<S>(s, 0, 0);
                a.seed = step_seed(static_cast<uint32_t>(t));
                constexpr int ar = AaShape<S>::rows, ac = AaShape<S>::cols;
                const SlabSplit q = slab_split(D, za, zb, ar);
                if ((t & 1) == 0)
                    k_aa_odd_slab<S, R><<<slab_split_grid(D, q, ar, ac), aa_block<S>(), 0, st>>>(a, q);
                else
                    k_aa_even_slab<S, R><<<slab_split_grid(D, q, ar, ac), aa_block<S>(), 0, st>>>(a, q);
            }
            CULBM_CUDA(cudaGetLastError());
            s->launches += 1;
        }
        CULBM_CUDA(cudaEventRecord(ev(j, t & 3), st));
    }
    return CULBM_OK;
}

// The simulation's stream waits for every slab stream (join), or every slab
// stream for the simulation's stream (fork).
culbm_status join_slabs(culbm_sim* s, int nstream)
{
    for (int k = 0; k < nstream; ++k) {
        CULBM_CUDA(cudaEventRecord(s->slab_ev[k * kSlabEvents + kSlabDump], s->slab_st[k]));
        CULBM_CUDA(cudaStreamWaitEvent(s->stream, s->slab_ev[k * kSlabEvents + kSlabDump], 0));
    }
    return CULBM_OK;
}

culbm_status fork_slabs(culbm_sim* s, int nstream, cudaEvent_t e)
{
    CULBM_CUDA(cudaEventRecord(e, s->stream));
    for (int k = 0; k < nstream; ++k) CULBM_CUDA(cudaStreamWaitEvent(s->slab_st[k], e, 0));
    return CULBM_OK;
}

template <typename S>
culbm_status run_host_overlapped(culbm_sim* s, const uint32_t* flag, const float* const mac[4], uint32_t nsteps,
                                 float* const out[4])
{
    const Domain& D = s->dom;
    const int nslab = run_slabs(s, nsteps);
    const int nstream = std::min(nslab, kRunStreams);
    CULBM_TRY(ensure_run_streams(s, nstream, nslab));
    auto ev = [&](int j, int k) { return s->slab_ev[static_cast<size_t>(j) * kSlabEvents + k]; };
    cudaStream_t h2d = s->copy_st[0], d2h = s->copy_st[1];
    const int T = static_cast<int>(nsteps);

    // Everything follows the simulation's earlier work.
    CULBM_CUDA(cudaEventRecord(s->run_ev[0], s->stream));
    CULBM_CUDA(cudaStreamWaitEvent(h2d, s->run_ev[0], 0));
    CULBM_CUDA(cudaStreamWaitEvent(d2h, s->run_ev[0], 0));
    // Defaults of NULL inputs and the population start, on the simulation's stream.
    const dim3 g1(1184), b1(256);
    if (flag == nullptr) k_fill_u32<<<g1, b1, 0, s->stream>>>(s->d_flag, s->n, kDefaultFlag);
    const float dflt[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < 4; ++k)
        if (mac[k] == nullptr) k_fill_f32<<<g1, b1, 0, s->stream>>>(s->d_mac[k], s->n, dflt[k]);
    CULBM_CUDA(cudaGetLastError());
    CULBM_TRY(fill_rest<S>(s));
    CULBM_TRY(fork_slabs(s, nstream, s->run_ev[1]));

    // Slabs in, in slab order.
    auto span = [&](int j, long long* off, long long* cnt) {
        const int z0 = slab_z0(D, nslab, j), z1 = slab_z0(D, nslab, j + 1);
        *off = static_cast<long long>(z0) * D.nxy;
        *cnt = static_cast<long long>(z1 - z0) * D.nxy;
    };
    for (int j = 0; j < nslab; ++j) {
        long long off, cnt;
        span(j, &off, &cnt);
        if (flag != nullptr)
            CULBM_CUDA(cudaMemcpyAsync(s->d_flag + off, flag + off, cnt * sizeof(uint32_t), cudaMemcpyHostToDevice, h2d));
        for (int k = 0; k < 4; ++k)
            if (mac[k] != nullptr)
                CULBM_CUDA(cudaMemcpyAsync(s->d_mac[k] + off, mac[k] + off, cnt * sizeof(float), cudaMemcpyHostToDevice,
                                           h2d));
        CULBM_CUDA(cudaEventRecord(ev(j, kSlabIn), h2d));
    }

    // Slab by slab for the first and the last nslab steps, which the copies
    // overlap; whole-domain launches in between.  fill_rest left cur = 0 and
    // aa_phase = 0.
    const bool pull = s->cfg.stream_policy == CULBM_STREAM_PULL;
    int shift_end = T;   // steps into the skewed phase that ends with the dumps
    if (T <= 2 * nslab) {
        CULBM_TRY(run_slab_steps<S>(s, nslab, nstream, 0, T, true, true));
    } else {
        const int ta = nslab, tb = T - nslab;
        shift_end = T - tb;
        CULBM_TRY(run_slab_steps<S>(s, nslab, nstream, 0, ta, true, false));
        CULBM_TRY(join_slabs(s, nstream));
        s->step = static_cast<uint64_t>(ta);
        s->cur = pull ? ta & 1 : 0;
        s->aa_phase = pull ? 0 : ta & 1;
        CULBM_TRY(plain_steps<S>(s, static_cast<uint32_t>(tb - ta)));
        CULBM_TRY(fork_slabs(s, nstream, s->run_ev[1]));
        CULBM_TRY(run_slab_steps<S>(s, nslab, nstream, tb, T, false, true));
    }
    s->step = nsteps;
    s->launched_steps += nsteps;
    s->cur = pull ? T & 1 : 0;
    s->aa_phase = pull ? 0 : T & 1;
    s->loaded = true;

    // The fields out as each slab's dump finishes.
    for (int j = 0; j < nslab; ++j) {
        const int za = slab_lo(D, nslab, j, shift_end), zb = slab_lo(D, nslab, j + 1, shift_end);
        if (zb <= za) continue;
        const long long off = static_cast<long long>(za) * D.nxy, cnt = static_cast<long long>(zb - za) * D.nxy;
        CULBM_CUDA(cudaStreamWaitEvent(d2h, ev(j, kSlabDump), 0));
        for (int k = 0; k < 4; ++k)
            CULBM_CUDA(cudaMemcpyAsync(out[k] + off, s->d_mac[k] + off, cnt * sizeof(float), cudaMemcpyDeviceToHost, d2h));
    }
    // Every slab stream ends with dumps, which the copy-out stream waited for.
    CULBM_CUDA(cudaEventRecord(s->run_ev[2], d2h));
    CULBM_CUDA(cudaStreamWaitEvent(s->stream, s->run_ev[2], 0));
    CULBM_CUDA(cudaStreamSynchronize(s->stream));
    return check_device_error(s);
}

bool read_exact(const std::string& path, void* dst, size_t bytes, bool* present, std::string* err)
{
    std::ifstream f(path, std::ios::binary);
    *present = static_cast<bool>(f);
    if (!f) return false;
    f.read(static_cast<char*>(dst), static_cast<std::streamsize>(bytes));
    if (static_cast<size_t>(f.gcount()) != bytes) {
        *err = "File: " + path + " holds " + std::to_string(f.gcount()) + " bytes, expected " + std::to_string(bytes);
        return false;
    }
    return true;
}

}  // namespace culbm

using namespace culbm;

extern "C" {

culbm_status culbm_config_init(culbm_config* cfg)
{
    if (cfg == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "cfg is NULL");
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->dev_id = 0;
    cfg->block_dim[0] = 32;
    cfg->block_dim[1] = 16;
    cfg->block_dim[2] = 2;
    cfg->grid_dim[0] = 2;
    cfg->grid_dim[1] = 3;
    cfg->grid_dim[2] = 19;
    cfg->domain_dim[0] = cfg->domain_dim[1] = cfg->domain_dim[2] = 256;
    cfg->inner_loop = 5;
    cfg->stream_policy = CULBM_STREAM_PULL;
    cfg->opt_policy = CULBM_OPT_NONE;
    cfg->vel_set = 0;
    cfg->inv_tau = 0.5f;
    cfg->use_ring_ddf_buf = 0;
    cfg->storage = CULBM_STORAGE_F32;
    cfg->persist_l2 = 0;
    cfg->cache_hints = 1;
    cfg->use_graphs = 1;
    return CULBM_OK;
}

culbm_status culbm_create(const culbm_config* cfg, culbm_sim** out)
{
    if (cfg == nullptr || out == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "cfg or out is NULL");
    *out = nullptr;
    CULBM_TRY(validate_config(*cfg));
    culbm_sim* s = new culbm_sim();
    s->cfg = *cfg;
    s->dev = cfg->dev_id;
    s->dom.nx = static_cast<int>(cfg->domain_dim[0]);
    s->dom.ny = static_cast<int>(cfg->domain_dim[1]);
    s->dom.nz = static_cast<int>(cfg->domain_dim[2]);
    s->dom.nxy = s->dom.nx * s->dom.ny;
    s->n = 1ll * s->dom.nxy * s->dom.nz;
    s->dom.n = static_cast<int>(s->n);
    s->esize = storage_bytes(cfg->storage);

    auto body = [&]() -> culbm_status {
        CULBM_CUDA(cudaSetDevice(s->dev));
        CULBM_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        CULBM_CUDA(cudaEventCreate(&s->ev0));
        CULBM_CUDA(cudaEventCreate(&s->ev1));
        const long long n = s->n;
        const bool blocked = is_blocked(s->cfg);
        const bool inplace = s->cfg.stream_policy == CULBM_STREAM_INPLACE && !blocked;
        s->npop = (inplace || (blocked && s->cfg.use_ring_ddf_buf)) ? 1 : 2;

        // Capacity check before allocating: populations dominate.
        size_t free_b = 0, total_b = 0;
        CULBM_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const double need = static_cast<double>(s->npop) * 27.0 * n * s->esize + 9.0 * n;
        if (need > static_cast<double>(free_b))
            return fail(CULBM_ERR_OUT_OF_MEMORY, "domain needs " + std::to_string(need / 1e9) + " GB, " +
                                                     std::to_string(free_b / 1e9) + " GB free on the device");

        CULBM_TRY(dev_alloc(s, reinterpret_cast<void**>(&s->d_flag), n * sizeof(uint32_t), "flags"));
        CULBM_TRY(dev_alloc(s, reinterpret_cast<void**>(&s->d_ops), n, "op bytes"));
        for (int k = 0; k < 4; ++k)
            CULBM_TRY(dev_alloc(s, reinterpret_cast<void**>(&s->d_mac[k]), n * sizeof(float), "macroscopic buffer"));
        if (!blocked || !s->cfg.use_ring_ddf_buf) {
            for (int k = 0; k < s->npop; ++k)
                CULBM_TRY(dev_alloc(s, &s->d_pop[k], 27ull * n * s->esize, "populations"));
        }
        if (inplace) {
            const long long fx = 9ll * s->dom.ny * s->dom.nz, fy = 9ll * s->dom.nx * s->dom.nz,
                            fz = 9ll * s->dom.nx * s->dom.ny;
            s->el.off[0] = 0;
            s->el.off[1] = fx;
            s->el.off[2] = 2 * fx;
            s->el.off[3] = 2 * fx + fy;
            s->el.off[4] = 2 * fx + 2 * fy;
            s->el.off[5] = 2 * fx + 2 * fy + fz;
            s->edge_elems = 2 * (fx + fy + fz);
            CULBM_TRY(dev_alloc(s, &s->d_edge, s->edge_elems * s->esize, "edge buffer"));
        }
        s->red_blocks = 592;
        CULBM_TRY(dev_alloc(s, reinterpret_cast<void**>(&s->d_red), (4ull * s->red_blocks + 4) * sizeof(double),
                            "reduction scratch"));
        if (blocked) CULBM_TRY(tiles_create(s));
        CULBM_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s->err_host), sizeof(int), cudaHostAllocMapped));
        *s->err_host = 0;
        CULBM_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->err_dev), s->err_host, 0));
        if (rows_applicable(s))
            CULBM_TRY(with_storage(s, [&](auto tag) { return rows_setup<typename decltype(tag)::type>(s); }));
        if (warp_pull_applicable(s))
            CULBM_TRY(with_storage(s, [&](auto tag) { return warp_pull_setup<typename decltype(tag)::type>(s); }));
        const float* none[4] = {nullptr, nullptr, nullptr, nullptr};
        CULBM_TRY(upload_state(s, nullptr, none));
        s->loaded = false;   // defaults in place; a load call is still expected
        CULBM_CUDA(cudaStreamSynchronize(s->stream));
        return CULBM_OK;
    };
    const culbm_status st = body();
    if (st != CULBM_OK) {
        const std::string msg = t_last_error;
        release(s);
        cudaGetLastError();
        set_last_error(msg);
        return st;
    }
    s->loaded = true;
    *out = s;
    return CULBM_OK;
}

culbm_status culbm_destroy(culbm_sim* sim)
{
    if (sim == nullptr) return CULBM_OK;
    release(sim);
    return CULBM_OK;
}

culbm_status culbm_load_state(culbm_sim* sim, const uint32_t* flag, const float* rho, const float* vx,
                              const float* vy, const float* vz)
{
    CULBM_TRY(check_sim(sim));
    const float* mac[4] = {rho, vx, vy, vz};
    CULBM_TRY(upload_state(sim, flag, mac));
    CULBM_CUDA(cudaStreamSynchronize(sim->stream));
    CULBM_TRY(check_device_error(sim));
    return CULBM_OK;
}

culbm_status culbm_load_state_folder(culbm_sim* sim, const char* folder, uint32_t* loaded_mask)
{
    CULBM_TRY(check_sim(sim));
    if (loaded_mask) *loaded_mask = 0;
    if (folder == nullptr || folder[0] == '\0') return culbm_load_state(sim, nullptr, nullptr, nullptr, nullptr, nullptr);
    const std::string dir(folder);
    const size_t n = static_cast<size_t>(sim->n);
    std::vector<uint32_t> flag(n);
    bool present = false;
    std::string err;
    if (!read_exact(dir + "/flag.dat", flag.data(), n * 4, &present, &err)) {
        if (!present) return fail(CULBM_ERR_IO, "File: " + dir + "/flag.dat doesn't exist!");
        return fail(CULBM_ERR_IO, err);
    }
    uint32_t mask = 1;
    std::vector<float> mac[4];
    const char* names[4] = {"rho", "vx", "vy", "vz"};
    const float* ptr[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < 4; ++k) {
        mac[k].resize(n);
        if (read_exact(dir + "/" + names[k] + ".dat", mac[k].data(), n * 4, &present, &err)) {
            ptr[k] = mac[k].data();
            mask |= 1u << (k + 1);
        } else if (present) {
            return fail(CULBM_ERR_IO, err);
        }
    }
    CULBM_TRY(culbm_load_state(sim, flag.data(), ptr[0], ptr[1], ptr[2], ptr[3]));
    if (loaded_mask) *loaded_mask = mask;
    return CULBM_OK;
}

culbm_status culbm_step(culbm_sim* sim, uint32_t nsteps)
{
    CULBM_TRY(check_sim(sim, true));
    if (nsteps == 0) return CULBM_OK;
    if (is_blocked(sim->cfg)) {
        CULBM_TRY(tiles_step(sim, nsteps));
    } else {
        CULBM_TRY(with_storage(sim, [&](auto tag) { return plain_steps<typename decltype(tag)::type>(sim, nsteps); }));
    }
    sim->step += nsteps;
    sim->launched_steps += nsteps;
    return CULBM_OK;
}

culbm_status culbm_step_timed(culbm_sim* sim, uint32_t nsteps, float* elapsed_ms)
{
    CULBM_TRY(check_sim(sim, true));
    CULBM_CUDA(cudaEventRecord(sim->ev0, sim->stream));
    CULBM_TRY(culbm_step(sim, nsteps));
    CULBM_CUDA(cudaEventRecord(sim->ev1, sim->stream));
    CULBM_CUDA(cudaEventSynchronize(sim->ev1));
    CULBM_TRY(check_device_error(sim));
    float ms = 0.0f;
    CULBM_CUDA(cudaEventElapsedTime(&ms, sim->ev0, sim->ev1));
    if (elapsed_ms) *elapsed_ms = ms;
    return CULBM_OK;
}

culbm_status culbm_synchronize(culbm_sim* sim)
{
    CULBM_TRY(check_sim(sim));
    CULBM_CUDA(cudaStreamSynchronize(sim->stream));
    return check_device_error(sim);
}

culbm_status culbm_moments(culbm_sim* sim)
{
    CULBM_TRY(check_sim(sim, true));
    const int layout = current_layout(sim);
    return with_storage(sim, [&](auto tag) -> culbm_status {
        using S = typename decltype(tag)::type;
        using R = typename ArithOf<S>::type;
        auto a = make_args<S>(sim, sim->cur, sim->cur);
        const dim3 g = cell_grid(sim->dom), b = cell_block();
        float* const* m = sim->d_mac;
        with_layout(layout, [&](auto L) {
            k_moments<decltype(L)::value, S, R><<<g, b, 0, sim->stream>>>(a, sim->d_flag, m[0], m[1], m[2], m[3], 0);
        });
        CULBM_CUDA(cudaGetLastError());
        return CULBM_OK;
    });
}

culbm_status culbm_get_field(culbm_sim* sim, culbm_field field, float* host_out)
{
    CULBM_TRY(check_sim(sim));
    if (field < 0 || field > 3 || host_out == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "bad field or NULL output");
    CULBM_CUDA(cudaMemcpyAsync(host_out, sim->d_mac[field], sim->n * sizeof(float), cudaMemcpyDeviceToHost, sim->stream));
    CULBM_CUDA(cudaStreamSynchronize(sim->stream));
    CULBM_TRY(check_device_error(sim));
    return CULBM_OK;
}

culbm_status culbm_run_host(culbm_sim* sim, const uint32_t* flag, const float* rho, const float* vx,
                            const float* vy, const float* vz, uint32_t nsteps, float* out_rho, float* out_vx,
                            float* out_vy, float* out_vz)
{
    CULBM_TRY(check_sim(sim));
    float* const out[4] = {out_rho, out_vx, out_vy, out_vz};
    for (float* o : out)
        if (o == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "culbm_run_host: NULL output buffer");
    const float* mac[4] = {rho, vx, vy, vz};
    if (is_blocked(sim->cfg) || sim->rows || sim->warp_pull) {
        // The tile engine and the staged 16-bit kernels step the whole domain at once.
        CULBM_TRY(upload_state(sim, flag, mac));
        CULBM_TRY(culbm_step(sim, nsteps));
        CULBM_TRY(culbm_moments(sim));
        for (int k = 0; k < 4; ++k)
            CULBM_CUDA(cudaMemcpyAsync(out[k], sim->d_mac[k], sim->n * sizeof(float), cudaMemcpyDeviceToHost,
                                       sim->stream));
        CULBM_CUDA(cudaStreamSynchronize(sim->stream));
        return check_device_error(sim);
    }
    return with_storage(sim, [&](auto tag) {
        return run_host_overlapped<typename decltype(tag)::type>(sim, flag, mac, nsteps, out);
    });
}

culbm_status culbm_dump(culbm_sim* sim, const char* folder, uint32_t field_mask)
{
    CULBM_TRY(check_sim(sim));
    if (folder == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "folder is NULL");
    std::error_code ec;
    std::filesystem::create_directories(folder, ec);
    if (ec) return fail(CULBM_ERR_IO, std::string("cannot create dump folder ") + folder + ": " + ec.message());
    if ((field_mask & 0xFu) == 0) return CULBM_OK;
    std::vector<float> host(static_cast<size_t>(sim->n));
    const char* names[4] = {"rho", "vx", "vy", "vz"};
    for (int k = 0; k < 4; ++k) {
        if (!(field_mask & (1u << k))) continue;
        const std::string path = std::string(folder) + "/" + names[k] + "_" + std::to_string(sim->step) + ".dat";
        std::ofstream f(path, std::ios::binary);
        if (!f) return fail(CULBM_ERR_IO, "Could not open the file: " + path);
        CULBM_TRY(culbm_get_field(sim, static_cast<culbm_field>(k), host.data()));
        f.write(reinterpret_cast<const char*>(host.data()), static_cast<std::streamsize>(host.size() * sizeof(float)));
        if (!f) return fail(CULBM_ERR_IO, "short write to " + path);
    }
    return CULBM_OK;
}

culbm_status culbm_get_step(culbm_sim* sim, uint64_t* step)
{
    if (sim == nullptr || step == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    *step = sim->step;
    return CULBM_OK;
}

culbm_status culbm_get_pulled_ddf(culbm_sim* sim, void* host_out, int32_t out_type)
{
    CULBM_TRY(check_sim(sim, true));
    if (host_out == nullptr || (out_type != 0 && out_type != 1))
        return fail(CULBM_ERR_INVALID_ARGUMENT, "bad output buffer or type");
    const size_t tsize = out_type == 0 ? 4 : 8;
    const size_t bytes = 27ull * sim->n * tsize;
    void* d_out = nullptr;
    CULBM_CUDA(cudaMalloc(&d_out, bytes));
    const int layout = current_layout(sim);
    culbm_status st = with_storage(sim, [&](auto tag) -> culbm_status {
        using S = typename decltype(tag)::type;
        using R = typename ArithOf<S>::type;
        auto a = make_args<S>(sim, sim->cur, sim->cur);
        const dim3 g = cell_grid(sim->dom), b = cell_block();
        auto launch = [&](auto tt) {
            using T = typename decltype(tt)::type;
            T* o = static_cast<T*>(d_out);
            with_layout(layout, [&](auto L) {
                k_export_pulled<decltype(L)::value, S, R, T><<<g, b, 0, sim->stream>>>(a, o);
            });
        };
        if (out_type == 0) launch(Tag<float>{});
        else launch(Tag<double>{});
        CULBM_CUDA(cudaGetLastError());
        CULBM_CUDA(cudaMemcpyAsync(host_out, d_out, bytes, cudaMemcpyDeviceToHost, sim->stream));
        CULBM_CUDA(cudaStreamSynchronize(sim->stream));
        CULBM_TRY(check_device_error(sim));
        return CULBM_OK;
    });
    cudaFree(d_out);
    return st;
}

culbm_status culbm_set_ddf(culbm_sim* sim, const void* host_in, int32_t in_type)
{
    CULBM_TRY(check_sim(sim, true));
    if (host_in == nullptr || (in_type != 0 && in_type != 1))
        return fail(CULBM_ERR_INVALID_ARGUMENT, "bad input buffer or type");
    const size_t tsize = in_type == 0 ? 4 : 8;
    const size_t bytes = 27ull * sim->n * tsize;
    void* d_in = nullptr;
    CULBM_CUDA(cudaMalloc(&d_in, bytes));
    const int layout = current_layout(sim);
    const bool aa = layout == LAYOUT_AA_A || layout == LAYOUT_AA_B;
    culbm_status st = with_storage(sim, [&](auto tag) -> culbm_status {
        using S = typename decltype(tag)::type;
        using R = typename ArithOf<S>::type;
        CULBM_CUDA(cudaMemcpyAsync(d_in, host_in, bytes, cudaMemcpyHostToDevice, sim->stream));
        const int target = aa ? 0 : sim->cur;
        auto a = make_args<S>(sim, target, target);
        const dim3 g = cell_grid(sim->dom), b = cell_block();
        auto launch = [&](auto tt) {
            using T = typename decltype(tt)::type;
            const T* in = static_cast<const T*>(d_in);
            if (aa)
                k_import<LAYOUT_AA_A, S, R, T><<<g, b, 0, sim->stream>>>(a, in);
            else if (layout == LAYOUT_PULL_RING)
                k_import<LAYOUT_PULL_RING, S, R, T><<<g, b, 0, sim->stream>>>(a, in);
            else
                k_import<LAYOUT_PULL, S, R, T><<<g, b, 0, sim->stream>>>(a, in);
        };
        if (in_type == 0) launch(Tag<float>{});
        else launch(Tag<double>{});
        CULBM_CUDA(cudaGetLastError());
        CULBM_CUDA(cudaStreamSynchronize(sim->stream));
        CULBM_TRY(check_device_error(sim));
        if (aa) sim->aa_phase = 0;
        return CULBM_OK;
    });
    cudaFree(d_in);
    return st;
}

culbm_status culbm_mass_momentum(culbm_sim* sim, double out[4])
{
    CULBM_TRY(check_sim(sim, true));
    if (out == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "out is NULL");
    const int layout = current_layout(sim);
    return with_storage(sim, [&](auto tag) -> culbm_status {
        using S = typename decltype(tag)::type;
        using R = typename ArithOf<S>::type;
        auto a = make_args<S>(sim, sim->cur, sim->cur);
        double* part = sim->d_red;
        const int nb = sim->red_blocks;
        with_layout(layout, [&](auto L) {
            k_mass_momentum<decltype(L)::value, S, R><<<nb, 256, 0, sim->stream>>>(a, part);
        });
        CULBM_CUDA(cudaGetLastError());
        k_sum_partials<<<1, 32, 0, sim->stream>>>(part, nb, part + 4 * nb);
        CULBM_CUDA(cudaGetLastError());
        CULBM_CUDA(cudaMemcpyAsync(out, part + 4 * nb, 4 * sizeof(double), cudaMemcpyDeviceToHost, sim->stream));
        CULBM_CUDA(cudaStreamSynchronize(sim->stream));
        CULBM_TRY(check_device_error(sim));
        return CULBM_OK;
    });
}

const char* culbm_last_error(void) { return t_last_error.c_str(); }

const char* culbm_status_string(culbm_status s)
{
    switch (s) {
        case CULBM_OK: return "CULBM_OK";
        case CULBM_ERR_INVALID_ARGUMENT: return "CULBM_ERR_INVALID_ARGUMENT";
        case CULBM_ERR_CUDA: return "CULBM_ERR_CUDA";
        case CULBM_ERR_OUT_OF_MEMORY: return "CULBM_ERR_OUT_OF_MEMORY";
        case CULBM_ERR_IO: return "CULBM_ERR_IO";
        case CULBM_ERR_STATE: return "CULBM_ERR_STATE";
        case CULBM_ERR_UNSUPPORTED: return "CULBM_ERR_UNSUPPORTED";
        case CULBM_ERR_DEVICE_TIMEOUT: return "CULBM_ERR_DEVICE_TIMEOUT";
    }
    return "CULBM_ERR_UNKNOWN";
}

int32_t culbm_abi_version(void) { return CULBM_ABI_VERSION; }

void culbm_debug_row_wait_extra_bytes(int32_t bytes) { g_row_extra_tx.store(bytes > 0 ? bytes : 0); }

void culbm_debug_inject_cuda_error(int32_t skip, int32_t code)
{
    g_inject_skip.store(skip < 0 ? 0 : skip);
    g_inject_code.store(code);
}

}  // extern "C"

extern "C" culbm_status culbm_get_info(culbm_sim* sim, culbm_info* info)
{
    if (sim == nullptr || info == nullptr) return fail(CULBM_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->cells = static_cast<uint64_t>(sim->n);
    info->device_bytes = sim->device_bytes;
    for (int k = 0; k < 3; ++k) {
        info->blocking_num[k] = 1;
        info->blocking_dim[k] = sim->cfg.domain_dim[k];
    }
    info->storage = sim->cfg.storage;
    info->stream_policy = sim->cfg.stream_policy;
    info->opt_policy = sim->cfg.opt_policy;
    info->inner_loop = sim->cfg.inner_loop;
    info->kernel_launches_per_step_x1000 =
        sim->launched_steps ? static_cast<uint32_t>(1000ull * sim->launches / sim->launched_steps) : 0;
    tiles_info(sim, info);
    return CULBM_OK;
}
