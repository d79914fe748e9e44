// Internal state of a culbm_sim and the helpers shared by the host runtime
// translation units (error reporting with fault injection, launch shapes).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "culbm.h"
#include "stream_kernels.cuh"

namespace culbm {

// ---------------------------------------------------------------- errors ---
void set_last_error(const std::string& msg);
culbm_status fail(culbm_status s, const std::string& msg);
// Returns the injected error for this call, or cudaSuccess (no injection).
cudaError_t injection_gate();
culbm_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);

}  // namespace culbm

// Runs a CUDA runtime call through the injection gate; on failure records
// the message and returns CULBM_ERR_CUDA (or OUT_OF_MEMORY) from the caller.
#define CULBM_CUDA(expr)                                                          \
    do {                                                                          \
        cudaError_t culbm_e_ = ::culbm::injection_gate();                         \
        if (culbm_e_ == cudaSuccess) culbm_e_ = (expr);                           \
        if (culbm_e_ != cudaSuccess)                                              \
            return ::culbm::cuda_fail(culbm_e_, #expr, __FILE__, __LINE__);       \
    } while (0)

#define CULBM_TRY(expr)                                                           \
    do {                                                                          \
        culbm_status culbm_s_ = (expr);                                           \
        if (culbm_s_ != CULBM_OK) return culbm_s_;                                \
    } while (0)

namespace culbm {

struct TileState;   // blocked policies (tile_runtime.cu)

}  // namespace culbm

struct culbm_sim {
    culbm_config cfg{};
    culbm::Domain dom{};
    long long n = 0;
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    uint32_t* d_flag = nullptr;     // flag.dat words, N
    uint8_t* d_ops = nullptr;       // compact op bytes, N
    float* d_mac[4] = {};           // rho, vx, vy, vz, N each (EQU inputs and dump outputs)
    void* d_pop[2] = {};            // population buffers, 27*N elements each
    int npop = 0;                   // 1 (in-place) or 2 (double buffer)
    void* d_edge = nullptr;         // in-place clamp side buffer
    culbm::EdgeLayout el{};
    long long edge_elems = 0;
    size_t esize = 4;               // bytes per stored population
    double* d_red = nullptr;        // reduction partials
    int red_blocks = 0;

    int cur = 0;                    // double buffer: index of the buffer holding the newest state
    int aa_phase = 0;               // in-place: 0 = layout A, 1 = layout B
    uint64_t step = 0;
    uint64_t device_bytes = 0;
    uint64_t launches = 0;          // kernel launches issued by step calls
    uint64_t launched_steps = 0;
    bool loaded = false;

    culbm::TileState* tiles = nullptr;

    // Row-staged 16-bit step kernels (row_kernels.cuh), when the domain suits them.
    bool rows = false;
    bool warp_pull = false;         // warp-staged 16-bit pull (warp_kernels.cuh)
    CUtensorMap map_load[2];        // its tensor maps of population buffer 0 and 1: window loads
    CUtensorMap map_store[2];       // and output stores
    int row_grid[3] = {0, 0, 0};    // resident blocks per launch, by RowMode
    int* err_host = nullptr;        // mapped host word a bounded device-side wait writes on expiry
    int* err_dev = nullptr;         // its device address

    // Overlapped host run (culbm_run_host), created on first use.
    cudaStream_t copy_st[2] = {nullptr, nullptr};   // host-to-device, device-to-host copies
    std::vector<cudaStream_t> slab_st;              // one per slab of z-planes
    std::vector<cudaEvent_t> slab_ev;               // kSlabEvents per slab
    cudaEvent_t run_ev[3] = {nullptr, nullptr, nullptr};   // start, populations filled, copies out done
};

namespace culbm {

inline dim3 cell_block() { return dim3(32, 8, 1); }
// Blocks of the in-place step launches of storage format S (AaShape).
template <typename S>
inline dim3 aa_block() { return dim3(AaShape<S>::cols, AaShape<S>::rows, 1); }
inline dim3 cell_grid(const Domain& D)
{
    return dim3((D.nx + 31) / 32, (D.ny + 7) / 8, D.nz);
}

template <typename S>
struct Tag {
    using type = S;
};

culbm_status fail(culbm_status s, const std::string& msg);

// Calls f(Tag<S>{}) for the storage type of sim.
template <class F>
culbm_status with_storage(const culbm_sim* s, F&& f)
{
    switch (s->cfg.storage) {
        case CULBM_STORAGE_F32: return f(Tag<float>{});
        case CULBM_STORAGE_F16: return f(Tag<__half>{});
        case CULBM_STORAGE_BF16: return f(Tag<__nv_bfloat16>{});
        case CULBM_STORAGE_F64: return f(Tag<double>{});
        case CULBM_STORAGE_F16_SR: return f(Tag<Half16SR>{});
        case CULBM_STORAGE_BF16_SR: return f(Tag<BF16SR>{});
        default: return fail(CULBM_ERR_INVALID_ARGUMENT, "unknown storage format");
    }
}

// Reports and clears an expired bounded device-side wait (after a synchronisation).
culbm_status check_device_error(culbm_sim* s);

// Device allocation counted in sim->device_bytes (sim.cu).
culbm_status dev_alloc(culbm_sim* s, void** p, size_t bytes, const char* what);

// Blocked-policy entry points (tile_runtime.cu).
culbm_status validate_blocking(const culbm_config& cfg);
culbm_status tiles_create(culbm_sim* sim);
void tiles_destroy(culbm_sim* sim);
culbm_status tiles_upload_flags(culbm_sim* sim, const uint32_t* host_flag);
culbm_status tiles_reset(culbm_sim* sim);
culbm_status tiles_step(culbm_sim* sim, uint32_t nsteps);
// Where the newest global state lives: ring planes (0 = plain buffers), its
// z offset in the ring, and the per-direction stride in elements.
void tiles_view(const culbm_sim* sim, int* ring_nz, int* offz, long long* stride);
void tiles_info(const culbm_sim* sim, culbm_info* info);
bool is_blocked(const culbm_config& cfg);

}  // namespace culbm
