/*
 * culbm.h — C ABI of culbm_b200, a D3Q27 lattice Boltzmann (BGK) solver for
 * one NVIDIA B200 (sm_100a).
 *
 * The reference (cuLBM) has no C ABI: its boundary is the single_dev_expt_main
 * process (argv, init-state folder, dump files) over the C++ class
 * culbm::simulator::single_dev_expt::Simulator
 * (src/simulator/single_dev_expt/simulator_expt_platform.hpp:5-15).  Each entry
 * point below names the reference code whose job it takes over.  Plain C
 * types only: host pointers, sizes and status codes; no exceptions cross it.
 *
 * Threading: one culbm_sim is used by one host thread at a time.  All device
 * work of a culbm_sim runs on its own CUDA stream; calls that return host data
 * synchronise that stream.
 *
 * Ownership: the library owns every device buffer; host buffers passed in are
 * only read (or written) during the call.
 *
 * Errors: every call returns a culbm_status; culbm_last_error() returns the
 * message of the last failure on the calling thread.
 */
#ifndef CULBM_H
#define CULBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CULBM_ABI_VERSION 1

typedef enum culbm_status {
    CULBM_OK = 0,
    CULBM_ERR_INVALID_ARGUMENT = 1, /* bad size/policy/geometry (reference: std::invalid_argument, runtime_error) */
    CULBM_ERR_CUDA = 2,             /* a CUDA runtime call failed (reference: basic::cu::CudaRuntimeError) */
    CULBM_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed or would not fit */
    CULBM_ERR_IO = 4,               /* init-state file missing or short, dump file not writable */
    CULBM_ERR_STATE = 5,            /* call out of order */
    CULBM_ERR_UNSUPPORTED = 6,      /* policy/storage combination not built */
    CULBM_ERR_DEVICE_TIMEOUT = 7    /* a bounded device-side wait gave up */
} culbm_status;

/* --streamPolicy, simulator_expt_platform.cu:37-41 */
typedef enum culbm_stream_policy { CULBM_STREAM_PULL = 0, CULBM_STREAM_INPLACE = 1 } culbm_stream_policy;

/* --optPolicy, simulator_expt_platform.cu:43-49.  Every policy gives the
 * plain step's results bit for bit.  CULBM_OPT_L1L2 with pull streaming runs
 * each tile (blockDim*gridDim) as one thread-block cluster (blockDim as the
 * CTA and gridDim as the cluster's CTAs when they fit: at most 512 threads,
 * 16 CTAs); tiles no cluster holds, in-place streaming and the other blocked
 * policies run on the L2 tile engine. */
typedef enum culbm_opt_policy {
    CULBM_OPT_NONE = 0,
    CULBM_OPT_STATIC_L2 = 1,
    CULBM_OPT_L1L2 = 2,
    CULBM_OPT_DYNAMIC_L2 = 3
} culbm_opt_policy;

/* Population storage in HBM (no reference counterpart; the reference is FP32 only). */
typedef enum culbm_storage {
    CULBM_STORAGE_F32 = 0,  /* FP32, the reference's format */
    CULBM_STORAGE_F16 = 1,  /* FP16 deviations f_i - w_i (scaled by 2^15), FP32 arithmetic */
    CULBM_STORAGE_BF16 = 2, /* BF16 deviations f_i - w_i, FP32 arithmetic */
    CULBM_STORAGE_F64 = 3,  /* FP64 storage and arithmetic (the GPU oracle) */
    CULBM_STORAGE_F16_SR = 4,  /* as F16, stored with deterministic stochastic rounding */
    CULBM_STORAGE_BF16_SR = 5  /* as BF16, stored with deterministic stochastic rounding */
} culbm_storage;

typedef enum culbm_field {
    CULBM_FIELD_RHO = 0,
    CULBM_FIELD_VX = 1,
    CULBM_FIELD_VY = 2,
    CULBM_FIELD_VZ = 3
} culbm_field;

/* Flag bits of flag.dat, src/simulator/single_dev_expt/local_config.hpp:12-22. */
#define CULBM_FLAG_LOAD (1u << 0)
#define CULBM_FLAG_EQU (1u << 1)
#define CULBM_FLAG_COLLIDE (1u << 2)
#define CULBM_FLAG_BOUNCE_BACK (1u << 3)
#define CULBM_FLAG_STORE (1u << 4)
#define CULBM_FLAG_DUMP_RHO (1u << 27)
#define CULBM_FLAG_DUMP_VX (1u << 28)
#define CULBM_FLAG_DUMP_VY (1u << 29)
#define CULBM_FLAG_DUMP_VZ (1u << 30)

/*
 * Solver configuration.  The first block mirrors the single_dev_expt_main
 * options and their defaults (simulator_expt_platform.cu:312-354); the rest
 * are additions.
 */
typedef struct culbm_config {
    int32_t dev_id;            /* --devId, default 0 */
    uint32_t block_dim[3];     /* --blockDim, default [32,16,2] */
    uint32_t grid_dim[3];      /* --gridDim, default [2,3,19] */
    uint32_t domain_dim[3];    /* --domainDim, default [256,256,256] */
    int32_t inner_loop;        /* --innerLoop, default 5 */
    int32_t stream_policy;     /* --streamPolicy, culbm_stream_policy */
    int32_t opt_policy;        /* --optPolicy, culbm_opt_policy */
    int32_t vel_set;           /* --velSet, 0 = D3Q27 (the only one) */
    float inv_tau;             /* --invTau, default 0.5 */
    int32_t use_ring_ddf_buf;  /* --useRingDDFBuf */
    /* additions */
    int32_t storage;           /* culbm_storage, default F32 */
    int32_t persist_l2;        /* 1: L2 persisting window over tile buffers (reference build
                                  switch CULBM_EXPT_ENABLE_PERSISTENT_L2, on in its default
                                  build); 0 (default): none, which is faster on B200 */
    int32_t cache_hints;       /* 1 (default): evict-first/evict-last hints on global/tile traffic
                                  (reference build switch CULBM_EXPT_CACHE_HINT_POLICY) */
    int32_t use_graphs;        /* 1 (default): tile launch sequences replayed as CUDA graphs */
    int32_t kernel_variant;    /* step kernels of the plain policies with 16-bit storage: 0 (default)
                                  one thread per cell with direct global loads and stores; 1 and 2
                                  row-staged (whole x-rows of the 27 planes staged in shared memory
                                  by bulk asynchronous copies, one block per row; 1: one output
                                  buffer, 2: two), used where nx is a multiple of 16 and at most
                                  992; 3 and 4 (pull only) warp-staged (32-cell row segments
                                  through TMA tensor copies, two or three window buffers per
                                  warp), used where nx is a multiple of 8.  Same bits either way */
    int32_t run_slabs;         /* culbm_run_host: slabs of z-planes the overlapped run cuts the domain
                                  into; 0 (default) automatic: for runs of up to 40 steps at most 64
                                  slabs of at least 2^18 cells, else at most 32 of at least 2^19;
                                  always at most nz/2, so that every slab has two planes or more */
    uint32_t reserved[6];
} culbm_config;

/* Fills cfg with the reference's defaults plus the additions' defaults. */
culbm_status culbm_config_init(culbm_config* cfg);

typedef struct culbm_sim culbm_sim;

/*
 * Validates cfg, selects the device, allocates every device buffer and fills
 * the populations with rest equilibrium; flags default to fluid everywhere
 * and rho/u to 1/0 until culbm_load_state is called.
 * Replaces Simulator::Data::Data, simulator_expt_platform.cu:308-445
 * (minus argv parsing, which single_dev_expt_main does on top of this ABI).
 */
culbm_status culbm_create(const culbm_config* cfg, culbm_sim** out);

/* Frees every device resource.  Replaces Simulator::Data::~Data, simulator_expt_platform.cu:447-505. */
culbm_status culbm_destroy(culbm_sim* sim);

/*
 * Loads an init state from host arrays of domain_dim[0]*[1]*[2] values,
 * x fastest.  flag == NULL selects LOAD|COLLIDE|STORE|DUMP_* everywhere;
 * rho == NULL selects 1, vx/vy/vz == NULL select 0.  Resets the populations
 * to rest equilibrium and the step counter to 0.
 * Replaces initFlag / initBlockingFlag / initRhoU / initDoubleDDFBuf /
 * initRingDDFBuf, simulator_expt_platform.cu:95-277.
 */
culbm_status culbm_load_state(culbm_sim* sim, const uint32_t* flag, const float* rho, const float* vx,
                              const float* vy, const float* vz);

/*
 * Same from an init-state folder: <folder>/flag.dat is mandatory, rho.dat,
 * vx.dat, vy.dat, vz.dat are optional (raw little-endian, N values).
 * loaded_mask (may be NULL) receives bit k set when field k of
 * {flag, rho, vx, vy, vz} came from a file.  folder == NULL or "" behaves like
 * culbm_load_state with all NULL.  Error behaviour of initFlag/initRhoU:
 * a missing flag.dat is CULBM_ERR_IO.
 */
culbm_status culbm_load_state_folder(culbm_sim* sim, const char* folder, uint32_t* loaded_mask);

/*
 * Advances exactly nsteps time steps (stream-ordered, returns after enqueue).
 * Replaces one run lambda's inner step loop, simulator_expt_platform.cu:608-991.
 */
culbm_status culbm_step(culbm_sim* sim, uint32_t nsteps);

/* Same, then waits and reports the device time of those steps (CUDA events). */
culbm_status culbm_step_timed(culbm_sim* sim, uint32_t nsteps, float* elapsed_ms);

/* Waits for all work of sim. */
culbm_status culbm_synchronize(culbm_sim* sim);

/*
 * Dump kernel: writes rho/vx/vy/vz of the pulled populations into the
 * device macroscopic buffers where the DUMP bits are set.
 * Replaces StaticD3Q27PullDumpKernel and the per-tile dump kernels,
 * src/simulator/single_dev_expt/kernel.cu:2634-2735, 1829-1936.
 */
culbm_status culbm_moments(culbm_sim* sim);

/* Copies one device macroscopic buffer (N floats) to host_out; synchronises.
 * Replaces the cudaMemcpy of dumpRes, simulator_expt_platform.cu:572-606. */
culbm_status culbm_get_field(culbm_sim* sim, culbm_field field, float* host_out);

/*
 * One whole run from host memory to host memory: the effect of
 * culbm_load_state(flag, rho, vx, vy, vz), culbm_step(nsteps),
 * culbm_moments() and culbm_get_field() of the four fields into
 * out_rho/out_vx/out_vy/out_vz, with the same bits; synchronises.
 * The copies overlap the steps.  The domain is cut into slabs of z-planes
 * (at least two planes each).  A slab's host-to-device copy, its steps and
 * its device-to-host copy run as soon as its data and its neighbours' are
 * ready, so early slabs step while later ones still arrive and leave while
 * later ones still step.  Overlap needs page-locked host buffers
 * (cudaHostAlloc / cudaHostRegister); pageable ones give the same results
 * with the copies serialised.  The blocked policies (optPolicy > 0) and
 * kernel_variant != 0 run the four calls one after another.  Inputs may be
 * NULL as in culbm_load_state; outputs must not be.  The simulation's own
 * stream waits for earlier work first and holds the run's end when the call
 * returns.  Replaces one run of the reference's driver from its init state
 * to its dump, simulator_expt_platform.cu:944-991 with :572-606.
 */
culbm_status culbm_run_host(culbm_sim* sim, const uint32_t* flag, const float* rho, const float* vx,
                            const float* vy, const float* vz, uint32_t nsteps, float* out_rho, float* out_vx,
                            float* out_vy, float* out_vz);

/*
 * Writes <folder>/<rho|vx|vy|vz>_<step>.dat for every field whose bit is set
 * in field_mask (bit k = culbm_field k), creating the folder first even when
 * the mask is 0.  Replaces dumpRes, simulator_expt_platform.cu:572-606.
 */
culbm_status culbm_dump(culbm_sim* sim, const char* folder, uint32_t field_mask);

/* Time steps done since the last load. */
culbm_status culbm_get_step(culbm_sim* sim, uint64_t* step);

/*
 * The 27*N populations each cell would pull at the next step, out[d*N + i],
 * as float (out_type 0) or double (out_type 1).  This is the state every
 * streaming policy agrees on bit for bit.  Synchronises.
 */
culbm_status culbm_get_pulled_ddf(culbm_sim* sim, void* host_out, int32_t out_type);

/*
 * Replaces the state by post-collision populations in the standard layout
 * in[d*N + i] (what the reference's src buffer holds between steps), given as
 * float (in_type 0) or double (in_type 1).  Does not reset the step counter.
 */
culbm_status culbm_set_ddf(culbm_sim* sim, const void* host_in, int32_t in_type);

/* Total mass sum(rho) and momentum sum(rho*u) over the cells that have any of
 * LOAD|EQU, from the pulled populations, accumulated in FP64 on the device:
 * out[0] = mass, out[1..3] = momentum x,y,z.  No reference counterpart. */
culbm_status culbm_mass_momentum(culbm_sim* sim, double out[4]);

/*
 * No reference counterpart.  The reduction of culbm_mass_momentum over a
 * caller-owned FP32 population buffer in device memory: 27 planes of n
 * values, plane d at d_ddf + d*n (the layout culbm_get_pulled_ddf writes),
 * every cell counted: out[0] = sum(1 + sum_d f_d), out[1..3] = sum(c_d f_d).
 * Runs on the current device and on `stream` (a cudaStream_t; NULL is the
 * legacy default stream) and blocks until out is written.
 *
 * For callers that keep the populations in their own device memory and must
 * not allocate: a PyTorch (or other framework) process whose device memory
 * belongs to its caching allocator, or code inside a memory budget it does
 * not control.  There, cudaMalloc would take memory behind the allocator's
 * back, and cudaMalloc/cudaFree synchronise the whole device; a culbm_sim
 * would also hold a second copy of the state.
 *
 * Allocates nothing: the block partial sums live in a fixed 37,920-byte
 * static device array, so n may not exceed CULBM_NOALLOC_MAX_CELLS
 * (CULBM_ERR_INVALID_ARGUMENT beyond it).  Every GPU that loads the library
 * holds that array until the process exits, and it keeps the last call's
 * contents (each call writes every slot it reads).  The first call in each
 * CUDA context (a device's primary context, the one made again after
 * cudaDeviceReset, or one made with cuCtxCreate) looks up that array's
 * address with the device current (cudaGetSymbolAddress) and keeps it for
 * that context; make that first call before any stream capture.  Every call
 * waits for `stream` and then copies the four results into `out`.  Calls
 * that overlap on the GPU (other streams or host threads, same device) share
 * the array and race: serialise them.  The sum order depends on n alone.
 */
#define CULBM_NOALLOC_MAX_CELLS 77594624ull
culbm_status culbm_mass_momentum_noalloc(const float* d_ddf, uint64_t n, void* stream, double out[4]);

/*
 * Tile and innerLoop choice for the L2-blocked policies (--blockDim auto).
 * Restates the speed-up model of the reference's analysis/selector.py:15-69
 * (valid fraction of a tile, sector alignment of its valid rows, L2 reuse)
 * with the constants of this device, restricted to geometries the blocking
 * engine accepts for the domain (the reference's selector ignores the domain).
 */
typedef struct culbm_memory_constants {
    double dram_gbs;               /* copy bandwidth, two arrays of 3x L2 each */
    double l2_gbs;                 /* copy bandwidth, two arrays of L2/4 each */
    double lambda;                 /* dram_gbs / l2_gbs */
    double full_store_ms;          /* 1 GiB of 128-byte streaming stores, four full sectors each */
    double partial_store_ms;       /* the same with one partial sector per 128 bytes */
    double gamma;                  /* 4 partial/full - 3: cost of a partial sector in full sectors */
    uint64_t l2_bytes;
    uint32_t reserved[8];
} culbm_memory_constants;

/* Measures lambda and gamma on device `dev`: the experiments of the
 * reference's analysis/lambda/measure.cu and analysis/gamma/measure.cu,
 * written anew (allocates about 1.8 GB for a few seconds). */
culbm_status culbm_measure_memory(int32_t dev, culbm_memory_constants* out);

typedef struct culbm_tile_choice {
    uint32_t tile[3];              /* blockDim * gridDim of the chosen tile */
    int32_t inner_loop;
    double predicted_speedup;      /* model speed-up over plain streaming (S) */
    double predicted_speedup_no_alignment;  /* the same without the sector-alignment term (S0) */
    double predicted_speedup_b200; /* S of the chosen tile with B200's measured step costs
                                      (CULBM_B200_PLAIN_* and CULBM_B200_TILE_*): above 1 when
                                      blocking is expected to beat plain streaming on B200 */
    uint32_t reserved[6];
} culbm_tile_choice;

/* Constants used when lambda, gamma <= 0: culbm_measure_memory on a B200
 * (DRAM copy 6.48 TB/s, L2 copy 13.4 TB/s; a partial sector costs 8.8 full ones). */
#define CULBM_B200_LAMBDA 0.4841
#define CULBM_B200_GAMMA 8.772
/* The 16-bit formats' plain step is bound by instruction issue, not DRAM: its
 * time per update over the DRAM time of its 108 bytes at the copy bandwidth
 * (FP16-SR pull: 36.2k MLUPS against 60.6k) on a B200.  The model takes the
 * larger of memory and compute time per update, so for these formats every
 * blocked tile predicts S < 1 (the halo cells cost compute and save only
 * bandwidth) and the tile of largest S is the one with the least halo. */
#define CULBM_B200_COMPUTE_16 1.67
/* Measured step costs on B200, each as time per update over the DRAM time of
 * the format's bytes per update at the copy bandwidth.  The model takes the
 * DRAM traffic of an L2-blocked round as its time; on B200 the tile steps
 * themselves cost more than that, in L2 or not.  Plain FP32 pull: 29.2k
 * MLUPS against 30.3k.  An FP32 L2-tile step (pull tiles, per computed cell,
 * halo included): 28.7k against 30.3k.  A 16-bit tile step: 22.8k against
 * 60.6k.  The plain 16-bit step is CULBM_B200_COMPUTE_16.
 * predicted_speedup_b200 = h max(1, plain) / max(D, tile) with these. */
#define CULBM_B200_PLAIN_32 1.04
#define CULBM_B200_TILE_32 1.06
#define CULBM_B200_TILE_16 2.66

/* The tile and innerLoop of the largest model speed-up for `domain_dim` and
 * population storage `storage` (CULBM_STORAGE_*), with the compute floor of
 * the 16-bit formats (CULBM_B200_COMPUTE_16).  lambda, gamma <= 0: the B200
 * values above; l2_bytes, persist_bytes == 0: the current device's L2 size and
 * persisting-L2 limit.  A predicted speed-up below 1 means plain streaming
 * is faster. */
culbm_status culbm_select_tile(const uint32_t domain_dim[3], int32_t storage, double lambda, double gamma,
                               uint64_t l2_bytes, uint64_t persist_bytes, culbm_tile_choice* out);

/* The model's speed-up S (and S0, without the alignment term) of one tile
 * and innerLoop; same conventions as culbm_select_tile. */
culbm_status culbm_blocking_speedup(const uint32_t tile[3], int32_t inner_loop, int32_t storage, double lambda,
                                    double gamma, uint64_t l2_bytes, double* speedup, double* speedup_no_alignment);

/*
 * Tile geometry of one axis under the blocked policies, as the blocking
 * engine computes it: replaces blocking_core::validBlkAxisConfig, calcBlkNum
 * and calcValidPrev (src/blocking_core/blocking_alogrithm.hpp:7-41).  For a
 * domain extent `domain`, tile extent `tile` (blockDim*gridDim) and
 * `inner_loop`, writes the tile count to *num_tiles and, when `valid_starts`
 * is not NULL, the num_tiles + 1 valid-region bounds valid_starts[k] =
 * calcValidPrev(k) (tile k stores cells [valid_starts[k], valid_starts[k+1]))
 * into an array of `capacity` entries.  Returns CULBM_ERR_INVALID_ARGUMENT
 * (with the message culbm_create gives) for a geometry culbm_create rejects,
 * and when the bounds do not fit in `capacity`.  Host only; no device needed.
 */
culbm_status culbm_blocking_axis(uint32_t domain, uint32_t tile, int32_t inner_loop, uint32_t* num_tiles,
                                 int32_t* valid_starts, uint32_t capacity);

typedef struct culbm_info {
    uint64_t cells;                 /* N */
    uint64_t device_bytes;          /* bytes the library allocated on the device */
    uint32_t blocking_num[3];       /* tiles per axis (blocked policies), else 1 */
    uint32_t blocking_dim[3];       /* tile extent = blockDim*gridDim (blocked policies) */
    int32_t storage;
    int32_t stream_policy;
    int32_t opt_policy;
    int32_t inner_loop;
    uint64_t persisting_l2_bytes;   /* bytes of the L2 access-policy window (0 if none) */
    uint32_t kernel_launches_per_step_x1000;  /* average launches per time step, times 1000 */
    uint32_t reserved[7];
} culbm_info;

culbm_status culbm_get_info(culbm_sim* sim, culbm_info* info);

/* ------------------------------------------------------------------------
 * Discrete adjoint (no reference counterpart).
 *
 * Forward model: the same D3Q27 BGK step (pull with the per-axis clamp, EQU,
 * full-way bounce-back, BGK) in which every COLLIDE cell x carries a soft
 * obstacle value s(x) in [0,1] applied as partial bounce-back:
 *     f' = C(f) + s (B(f) - C(f)),   C = BGK, B(f)_d = f_{26-d},
 * so s = 0 is the plain step bit for bit.  Objective: the pressure drop
 *     J = mean_{t in [t0,t1]} ( mean_{inlet plane} rho/3 - mean_{outlet plane} rho/3 )
 * with rho from the pulled populations of the state after t steps, over the
 * COLLIDE cells of the planes x = plane_x[0] and x = plane_x[1].  The adjoint
 * is the exact reverse of that map (pull transposed into a push of adjoint
 * populations), run over checkpoints taken every `checkpoint_every` steps
 * with recomputation in between; parameter gradients are accumulated in FP64.
 * ---------------------------------------------------------------------- */
typedef struct culbm_adj_config {
    int32_t dev_id;
    uint32_t domain_dim[3];
    float inv_tau;                 /* default 0.5 */
    int32_t window[2];             /* [t0, t1], states after t steps; the forward runs t1 steps (default 300, 500) */
    int32_t plane_x[2];            /* inlet / outlet measurement planes (default 1 and nx-2) */
    int32_t checkpoint_every;      /* K: states kept every K steps of the forward pass.  0 = the smallest plan
                                      that fits hbm_budget_bytes: one level (K near sqrt(t1), every step
                                      recomputed once) if it fits, else two levels (recomputed twice) */
    int32_t precision;             /* 0: FP32 forward and adjoint (default), 1: FP64 */
    int32_t storage;               /* forward states and checkpoints: CULBM_STORAGE_F32 (default), _F16, _F16_SR;
                                      CULBM_STORAGE_F64 with precision 1 */
    uint64_t hbm_budget_bytes;     /* 0 = no limit given; the automatic plan then fits the device's free memory */
    int32_t checkpoint_inner;      /* K2 with K > 0: two levels.  Each K segment is recomputed once, keeping
                                      states every K2 steps, then swept K2 steps at a time; 1 <= K2 < K.
                                      0 = one level (default) */
    int32_t checkpoint_storage;    /* states kept for the reverse sweep.  0 (default): as `storage`.  With
                                      storage CULBM_STORAGE_F32: CULBM_STORAGE_F16 or _F16_SR runs the forward
                                      pass (and J) in FP32 and keeps its checkpoints in that 16-bit format; the
                                      recomputation between checkpoints and the reverse sweep then use 16-bit
                                      states, so a one-level plan needs about half the memory */
    uint32_t reserved[6];
} culbm_adj_config;

typedef struct culbm_adj culbm_adj;

typedef struct culbm_adj_info {
    int32_t checkpoint_every;
    int32_t checkpoints;
    uint64_t device_bytes;
    float forward_ms;              /* the recorded forward pass (with the objective) */
    float recompute_ms;            /* forward recomputation between checkpoints */
    float adjoint_ms;              /* adjoint sweep */
    uint64_t steps;                /* forward steps per pass (t1) */
    int32_t checkpoint_inner;      /* K2 of a two-level plan, 0 for one level */
    int32_t inner_checkpoints;     /* states held for the inner level */
    uint32_t reserved[6];
} culbm_adj_info;

culbm_status culbm_adj_config_init(culbm_adj_config* cfg);
culbm_status culbm_adj_create(const culbm_adj_config* cfg, culbm_adj** out);
culbm_status culbm_adj_destroy(culbm_adj* adj);

/* Flags, EQU macroscopic inputs (NULL: defaults as culbm_load_state) and the
 * soft field (NULL: 0) as host arrays of N values.  Cells must have STORE or
 * a zero flag word. */
culbm_status culbm_adj_set_state(culbm_adj* adj, const uint32_t* flag, const float* rho, const float* vx,
                                 const float* vy, const float* vz, const float* soft);

/* Overrides the relaxation rate invTau (double; rounded to the arithmetic type). */
culbm_status culbm_adj_set_inv_tau(culbm_adj* adj, double inv_tau);

/* Forward run from rest equilibrium; returns J. */
culbm_status culbm_adj_forward(culbm_adj* adj, double* J);

/*
 * Forward run, then the adjoint sweep.  Outputs (host, any may be NULL):
 * J; dJ/d invTau; dJ/ds per cell (N doubles, 0 where no COLLIDE); dJ/d of the
 * EQU inputs rho, vx, vy, vz per cell (4*N doubles, field-major, 0 where no EQU).
 */
culbm_status culbm_adj_gradient(culbm_adj* adj, double* J, double* dJ_dinv_tau, double* dJ_dsoft,
                                double* dJ_dmac);

culbm_status culbm_adj_get_info(culbm_adj* adj, culbm_adj_info* info);

/* Message of the last failure on this thread ("" if none). */
const char* culbm_last_error(void);

/* Constant name of a status code. */
const char* culbm_status_string(culbm_status s);

/* ABI version of the loaded library (CULBM_ABI_VERSION it was built with). */
int32_t culbm_abi_version(void);

/*
 * Fault-injection hook for the host-side error paths (tests): after `skip`
 * further CUDA runtime calls made by the library succeed, the next one is
 * reported as failed with CUDA error code `code` (the call itself is not
 * made).  code == 0 disables injection.  No device fault is involved.
 */
void culbm_debug_inject_cuda_error(int32_t skip, int32_t code);

/*
 * Test hook for the bounded waits of the row-staged step kernels: with
 * bytes > 0 every staged row announces `bytes` more than its copies deliver,
 * so its mbarrier phase never completes; the wait gives up after about a
 * second, the kernel stops and the next synchronising call returns
 * CULBM_ERR_DEVICE_TIMEOUT.  bytes <= 0 restores normal operation.  Touches
 * nothing but the announced byte count; every copy still lands.
 */
void culbm_debug_row_wait_extra_bytes(int32_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* CULBM_H */
