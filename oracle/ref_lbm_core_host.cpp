/*
 * ORACLE — test infrastructure only (checker and timed CPU baseline).
 *
 * Host build of the reference's own lbm_core routines.  This file includes
 * src/lbm_core/device_function.hpp from the reference tree at compile time
 * (oracle/Makefile passes the include paths; nothing of the reference is
 * copied here) and wraps bgk::calcEqu<27>, bgk::calcRhoU<27> and
 * bgk::collision2<27> in the pull loop of StaticD3Q27PullKernel
 * (src/simulator/single_dev_expt/kernel.cu:2489-2632) with OpenMP over
 * z-planes.  The output goes to oracle/_ref/ only.
 *
 * Uses:
 *   - pins the C restatement in oracle/d3q27_oracle.c (bitwise, FP32);
 *   - generates the golden fixtures under tests/golden/;
 *   - is the CPU baseline ("kind": "reference") timed by bench.py.
 */
#include <cstdint>
#include <cstring>
#include <utility>
#include <omp.h>

#include "device_function.hpp"
#include "blocking_alogrithm.hpp"

namespace {

// Flag bits, src/simulator/single_dev_expt/local_config.hpp:12-22.
constexpr std::uint32_t LOAD = 1u << 0, EQU = 1u << 1, COLLIDE = 1u << 2, BB = 1u << 3, STORE = 1u << 4;
constexpr std::uint32_t DRHO = 1u << 27, DVX = 1u << 28, DVY = 1u << 29, DVZ = 1u << 30;

inline void pull(std::int64_t nx, std::int64_t ny, std::int64_t nz, std::int64_t x, std::int64_t y,
                 std::int64_t z, const float* src, float* f)
{
    const std::int64_t n = nx * ny * nz;
    const std::int64_t i = (ny * z + y) * nx + x;
    const std::int64_t ndx = (x == 0) ? 0 : -1, pdx = (x == nx - 1) ? 0 : 1;
    const std::int64_t ndy = (y == 0) ? 0 : -nx, pdy = (y == ny - 1) ? 0 : nx;
    const std::int64_t ndz = (z == 0) ? 0 : -nx * ny, pdz = (z == nz - 1) ? 0 : nx * ny;
    for (int d = 0; d < 27; ++d) {
        const int cx = d % 3 - 1, cy = (d / 3) % 3 - 1, cz = d / 9 - 1;
        const std::int64_t ox = (cx == 1) ? ndx : (cx == -1) ? pdx : 0;
        const std::int64_t oy = (cy == 1) ? ndy : (cy == -1) ? pdy : 0;
        const std::int64_t oz = (cz == 1) ? ndz : (cz == -1) ? pdz : 0;
        f[d] = src[static_cast<std::int64_t>(d) * n + i + ox + oy + oz];
    }
}

}  // namespace

extern "C" {

void ref_equ_f32(float rho, float vx, float vy, float vz, float* f)
{
    culbm::lbm_core::bgk::calcEqu<27>(rho, vx, vy, vz, f);
}

void ref_rhou_f32(const float* f, float* rho, float* vx, float* vy, float* vz)
{
    culbm::lbm_core::bgk::calcRhoU<27>(*rho, *vx, *vy, *vz, f);
}

void ref_collide_f32(float inv_tau, float* f)
{
    culbm::lbm_core::bgk::collision2<27>(inv_tau, f);
}

int ref_valid_blk_axis(std::uint32_t dom, std::uint32_t blk, std::uint32_t iter)
{
    return culbm::blocking_core::validBlkAxisConfig<std::uint32_t>(dom, blk, iter) ? 1 : 0;
}

std::uint32_t ref_blk_num(std::uint32_t dom, std::uint32_t blk, std::uint32_t iter)
{
    return culbm::blocking_core::calcBlkNum<std::uint32_t>(dom, blk, iter);
}

std::int32_t ref_valid_prev(std::int32_t idx, std::int32_t blk, std::int32_t num, std::int32_t iter,
                            std::int32_t dom)
{
    return culbm::blocking_core::calcValidPrev<std::int32_t>(idx, blk, num, iter, dom);
}

// One pull step over the domain; z-planes [z0, z1) only (z1 <= 0 means nz),
// so that a bounded sample of a large domain can be timed.
void ref_step_f32(std::int64_t nx, std::int64_t ny, std::int64_t nz, const std::uint32_t* flag,
                  const float* rho, const float* vx, const float* vy, const float* vz, float inv_tau,
                  const float* src, float* dst, std::int64_t z0, std::int64_t z1, int nthreads)
{
    if (z1 <= 0) z1 = nz;
    const std::int64_t n = nx * ny * nz;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (std::int64_t z = z0; z < z1; ++z)
        for (std::int64_t y = 0; y < ny; ++y)
            for (std::int64_t x = 0; x < nx; ++x) {
                const std::int64_t i = (ny * z + y) * nx + x;
                const std::uint32_t fl = flag[i];
                float f[27] = {};
                if (fl & LOAD) pull(nx, ny, nz, x, y, z, src, f);
                if (fl & EQU) culbm::lbm_core::bgk::calcEqu<27>(rho[i], vx[i], vy[i], vz[i], f);
                if (fl & BB)
                    for (int d = 0; d < 13; ++d) std::swap(f[d], f[26 - d]);
                if (fl & COLLIDE) culbm::lbm_core::bgk::collision2<27>(inv_tau, f);
                if (fl & STORE)
                    for (int d = 0; d < 27; ++d) dst[static_cast<std::int64_t>(d) * n + i] = f[d];
            }
}

void ref_moments_f32(std::int64_t nx, std::int64_t ny, std::int64_t nz, const std::uint32_t* flag,
                     const float* src, float* rho, float* vx, float* vy, float* vz, int nthreads)
{
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (std::int64_t z = 0; z < nz; ++z)
        for (std::int64_t y = 0; y < ny; ++y)
            for (std::int64_t x = 0; x < nx; ++x) {
                const std::int64_t i = (ny * z + y) * nx + x;
                const std::uint32_t fl = flag[i];
                float f[27], r, ux, uy, uz;
                pull(nx, ny, nz, x, y, z, src, f);
                culbm::lbm_core::bgk::calcRhoU<27>(r, ux, uy, uz, f);
                if (fl & DRHO) rho[i] = r;
                if (fl & DVX) vx[i] = ux;
                if (fl & DVY) vy[i] = uy;
                if (fl & DVZ) vz[i] = uz;
            }
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
