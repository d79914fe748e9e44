/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement of the reference's single-device D3Q27 BGK hot path
 * (cuLBM, src/simulator/single_dev_expt/kernel.cu StaticD3Q27PullKernel and
 * StaticD3Q27PullDumpKernel over the lbm_core routines of
 * src/lbm_core/device_function.hpp).  It is the checker for the CUDA kernels
 * of culbm_b200: only the tests, the smoke check and bench.py's CPU-baseline
 * leg may load it.  The product never links or calls it.
 *
 * Built with -ffp-contract=off (see oracle/Makefile) so that a*b+c stays two
 * roundings and only the reference's explicit fma calls are fused.  With that,
 * the FP32 instance rounds exactly like the reference routines compiled for
 * the host; the test suite pins this against those routines (oracle/_ref) and
 * against the committed golden fixtures.
 */
#include <math.h>
#include <stdint.h>

/* Flag bits, src/simulator/single_dev_expt/local_config.hpp:12-22. */
#define ORC_LOAD        (1u << 0)
#define ORC_EQU         (1u << 1)
#define ORC_COLLIDE     (1u << 2)
#define ORC_BOUNCE_BACK (1u << 3)
#define ORC_STORE       (1u << 4)
#define ORC_DUMP_RHO    (1u << 27)
#define ORC_DUMP_VX     (1u << 28)
#define ORC_DUMP_VY     (1u << 29)
#define ORC_DUMP_VZ     (1u << 30)
#define ORC_CORRECT     (1u << 31)

#define REAL float
#define SFX f32
#define FMA fmaf
#include "d3q27_oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

#define REAL double
#define SFX f64
#define FMA fma
#include "d3q27_oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

/* Blocking geometry of the reference's temporal blocking.
 * Restates blocking_core::validBlkAxisConfig / calcBlkNum / calcValidPrev,
 * src/blocking_core/blocking_alogrithm.hpp:7-41 (unsigned arithmetic as the
 * simulator instantiates them with std::uint32_t). */
int orc_valid_blk_axis(uint32_t dom, uint32_t blk, uint32_t iter)
{
    if (blk < dom && blk + 1 <= iter) return 0;
    if (2 * (blk + 1 - iter) < dom && blk + 2 <= iter) return 0;
    return 1;
}

uint32_t orc_blk_num(uint32_t dom, uint32_t blk, uint32_t iter)
{
    if (dom <= blk) return 1;
    if (dom <= 2 * (blk + 1 - iter)) return 2;
    const uint32_t num = dom - 2 * (blk + 1 - iter);
    const uint32_t den = blk + 2 - 2 * iter;
    return 2 + (num + den - 1) / den;
}

int32_t orc_valid_prev(int32_t idx, int32_t blk, int32_t num, int32_t iter, int32_t dom)
{
    if (idx == num) return dom;
    if (idx == 0) return 0;
    return (blk + 1 - iter) + (idx - 1) * (blk + 2 - 2 * iter);
}
