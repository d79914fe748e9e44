/*
 * ORACLE — test infrastructure only (checker, never the product path).
 *
 * Type-generic body of the CPU restatement of the reference's single-device
 * D3Q27 BGK step.  Included twice by d3q27_oracle.c, once with REAL=float
 * (FP32 oracle, bit-exact target of the CUDA kernels) and once with
 * REAL=double (FP64 oracle used for error statements).
 *
 * Every arithmetic expression keeps the operand order, the parenthesisation and
 * the explicit fused multiply-adds of the reference so that, compiled with
 * -ffp-contract=off, the FP32 instance rounds exactly like the reference's
 * lbm_core routines compiled for the host with contraction disabled.
 *
 * Macros expected: REAL (float|double), SFX (f32|f64), FMA (fmaf|fma).
 */

#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* Shifted equilibrium feq_i - w_i from (rho, u).
 * Restates bgk::detail::calcEqu<27>, src/lbm_core/device_function.hpp:305-398. */
void FN(orc_equ)(REAL rho, REAL vx, REAL vy, REAL vz, REAL *f)
{
    const REAL W0 = (REAL)8 / (REAL)27;
    const REAL WS = (REAL)2 / (REAL)27;
    const REAL WE = (REAL)1 / (REAL)54;
    const REAL WC = (REAL)1 / (REAL)216;
    const REAL h = (REAL)0.5;

    const REAL rhom1 = rho - (REAL)1;
    const REAL c3 = (REAL)(-3) * (vx * vx + vy * vy + vz * vz);
    vx *= (REAL)3;
    vy *= (REAL)3;
    vz *= (REAL)3;
    const REAL v0 = vx + vy, v1 = vx + vz, v2 = vy + vz, v3 = vx - vy, v4 = vx - vz, v5 = vy - vz;
    const REAL v6 = vx + vy + vz, v7 = vx + vy - vz, v8 = vx - vy + vz, v9 = vy - vx + vz;
    const REAL rhos = WS * rho, rhoe = WE * rho, rhoc = WC * rho;
    const REAL rhom1s = WS * rhom1, rhom1e = WE * rhom1, rhom1c = WC * rhom1;

    f[0]  = FMA(rhoc, FMA(h, FMA(v6, v6, c3), -v6), rhom1c);
    f[1]  = FMA(rhoe, FMA(h, FMA(v2, v2, c3), -v2), rhom1e);
    f[2]  = FMA(rhoc, FMA(h, FMA(v9, v9, c3), -v9), rhom1c);
    f[3]  = FMA(rhoe, FMA(h, FMA(v1, v1, c3), -v1), rhom1e);
    f[4]  = FMA(rhos, FMA(h, FMA(vz, vz, c3), -vz), rhom1s);
    f[5]  = FMA(rhoe, FMA(h, FMA(v4, v4, c3), v4), rhom1e);
    f[6]  = FMA(rhoc, FMA(h, FMA(v8, v8, c3), -v8), rhom1c);
    f[7]  = FMA(rhoe, FMA(h, FMA(v5, v5, c3), v5), rhom1e);
    f[8]  = FMA(rhoc, FMA(h, FMA(v7, v7, c3), v7), rhom1c);
    f[9]  = FMA(rhoe, FMA(h, FMA(v0, v0, c3), -v0), rhom1e);
    f[10] = FMA(rhos, FMA(h, FMA(vy, vy, c3), -vy), rhom1s);
    f[11] = FMA(rhoe, FMA(h, FMA(v3, v3, c3), v3), rhom1e);
    f[12] = FMA(rhos, FMA(h, FMA(vx, vx, c3), -vx), rhom1s);
    f[13] = W0 * FMA(rho, h * c3, rhom1);
    f[14] = FMA(rhos, FMA(h, FMA(vx, vx, c3), vx), rhom1s);
    f[15] = FMA(rhoe, FMA(h, FMA(v3, v3, c3), -v3), rhom1e);
    f[16] = FMA(rhos, FMA(h, FMA(vy, vy, c3), vy), rhom1s);
    f[17] = FMA(rhoe, FMA(h, FMA(v0, v0, c3), v0), rhom1e);
    f[18] = FMA(rhoc, FMA(h, FMA(v7, v7, c3), -v7), rhom1c);
    f[19] = FMA(rhoe, FMA(h, FMA(v5, v5, c3), -v5), rhom1e);
    f[20] = FMA(rhoc, FMA(h, FMA(v8, v8, c3), v8), rhom1c);
    f[21] = FMA(rhoe, FMA(h, FMA(v4, v4, c3), -v4), rhom1e);
    f[22] = FMA(rhos, FMA(h, FMA(vz, vz, c3), vz), rhom1s);
    f[23] = FMA(rhoe, FMA(h, FMA(v1, v1, c3), v1), rhom1e);
    f[24] = FMA(rhoc, FMA(h, FMA(v9, v9, c3), v9), rhom1c);
    f[25] = FMA(rhoe, FMA(h, FMA(v2, v2, c3), v2), rhom1e);
    f[26] = FMA(rhoc, FMA(h, FMA(v6, v6, c3), v6), rhom1c);
}

/* Density rho = 1 + sum(f) in the reference's fixed pairing and velocity
 * u = (sum c f) * (1/rho).
 * Restates bgk::detail::calcRhoU<27>, src/lbm_core/device_function.hpp:439-463. */
void FN(orc_rhou)(const REAL *f, REAL *rho_out, REAL *vx_out, REAL *vy_out, REAL *vz_out)
{
    const REAL rho = ((REAL)1 + f[0]) + (f[1] + f[2]) + (f[3] + f[4]) + (f[5] + f[6]) + (f[7] + f[8])
                   + (f[9] + f[10]) + (f[11] + f[12]) + (f[13] + f[14]) + (f[15] + f[16]) + (f[17] + f[18])
                   + (f[19] + f[20]) + (f[21] + f[22]) + (f[23] + f[24]) + (f[25] + f[26]);
    const REAL inv_rho = (REAL)1 / rho;
    REAL vx = (f[2] - f[0]) + (f[5] - f[3]) + (f[8] - f[6])
            + (f[11] - f[9]) + (f[14] - f[12]) + (f[17] - f[15])
            + (f[20] - f[18]) + (f[23] - f[21]) + (f[26] - f[24]);
    REAL vy = (f[6] - f[0]) + (f[7] - f[1]) + (f[8] - f[2])
            + (f[15] - f[9]) + (f[16] - f[10]) + (f[17] - f[11])
            + (f[24] - f[18]) + (f[25] - f[19]) + (f[26] - f[20]);
    REAL vz = (f[18] - f[0]) + (f[19] - f[1]) + (f[20] - f[2])
            + (f[21] - f[3]) + (f[22] - f[4]) + (f[23] - f[5])
            + (f[24] - f[6]) + (f[25] - f[7]) + (f[26] - f[8]);
    vx *= inv_rho;
    vy *= inv_rho;
    vz *= inv_rho;
    *rho_out = rho;
    *vx_out = vx;
    *vy_out = vy;
    *vz_out = vz;
}

/* BGK relaxation f <- invTau*feq + (1-invTau)*f on shifted populations.
 * Restates bgk::detail::collision2<27>, src/lbm_core/device_function.hpp:676-754.
 * The centre term keeps the reference's association (invTau*W0)*fma(...). */
void FN(orc_collide)(REAL inv_tau, REAL *f)
{
    REAL rho, vx, vy, vz;
    FN(orc_rhou)(f, &rho, &vx, &vy, &vz);
    const REAL W0 = (REAL)8 / (REAL)27;
    const REAL WS = (REAL)2 / (REAL)27;
    const REAL WE = (REAL)1 / (REAL)54;
    const REAL WC = (REAL)1 / (REAL)216;
    const REAL h = (REAL)0.5;
    const REAL om = (REAL)1 - inv_tau;

    const REAL rhom1 = rho - (REAL)1;
    const REAL c3 = (REAL)(-3) * (vx * vx + vy * vy + vz * vz);
    vx *= (REAL)3;
    vy *= (REAL)3;
    vz *= (REAL)3;
    const REAL v0 = vx + vy, v1 = vx + vz, v2 = vy + vz, v3 = vx - vy, v4 = vx - vz, v5 = vy - vz;
    const REAL v6 = vx + vy + vz, v7 = vx + vy - vz, v8 = vx - vy + vz, v9 = vy - vx + vz;
    const REAL rhos = WS * rho, rhoe = WE * rho, rhoc = WC * rho;
    const REAL rhom1s = WS * rhom1, rhom1e = WE * rhom1, rhom1c = WC * rhom1;

#define RELAX(i, rw, rm, v, sv) f[i] = inv_tau * FMA(rw, FMA(h, FMA(v, v, c3), sv), rm) + om * f[i]
    RELAX(0, rhoc, rhom1c, v6, -v6);
    RELAX(1, rhoe, rhom1e, v2, -v2);
    RELAX(2, rhoc, rhom1c, v9, -v9);
    RELAX(3, rhoe, rhom1e, v1, -v1);
    RELAX(4, rhos, rhom1s, vz, -vz);
    RELAX(5, rhoe, rhom1e, v4, v4);
    RELAX(6, rhoc, rhom1c, v8, -v8);
    RELAX(7, rhoe, rhom1e, v5, v5);
    RELAX(8, rhoc, rhom1c, v7, v7);
    RELAX(9, rhoe, rhom1e, v0, -v0);
    RELAX(10, rhos, rhom1s, vy, -vy);
    RELAX(11, rhoe, rhom1e, v3, v3);
    RELAX(12, rhos, rhom1s, vx, -vx);
    f[13] = inv_tau * W0 * FMA(rho, h * c3, rhom1) + om * f[13];
    RELAX(14, rhos, rhom1s, vx, vx);
    RELAX(15, rhoe, rhom1e, v3, -v3);
    RELAX(16, rhos, rhom1s, vy, vy);
    RELAX(17, rhoe, rhom1e, v0, v0);
    RELAX(18, rhoc, rhom1c, v7, -v7);
    RELAX(19, rhoe, rhom1e, v5, -v5);
    RELAX(20, rhoc, rhom1c, v8, v8);
    RELAX(21, rhoe, rhom1e, v4, -v4);
    RELAX(22, rhos, rhom1s, vz, vz);
    RELAX(23, rhoe, rhom1e, v1, v1);
    RELAX(24, rhoc, rhom1c, v9, v9);
    RELAX(25, rhoe, rhom1e, v2, v2);
    RELAX(26, rhoc, rhom1c, v6, v6);
#undef RELAX
}

/* Per-cell boundary/collision sequence after the load:
 * EQU overwrite from the macroscopic buffers, full-way bounce-back swap of
 * d <-> 26-d, then BGK.  Restates src/simulator/single_dev_expt/kernel.cu:2571-2600. */
void FN(orc_cell)(uint32_t flag, REAL inv_tau, REAL rho, REAL vx, REAL vy, REAL vz, REAL *f)
{
    if (flag & ORC_EQU) {
        FN(orc_equ)(rho, vx, vy, vz, f);
    }
    if (flag & ORC_BOUNCE_BACK) {
        for (int d = 0; d < 13; ++d) {
            const REAL t = f[d];
            f[d] = f[26 - d];
            f[26 - d] = t;
        }
    }
    if (flag & ORC_COLLIDE) {
        FN(orc_collide)(inv_tau, f);
    }
}

/* Pull 27 populations of cell (x,y,z) from src: population d comes from
 * (x,y,z) - c_d, with the neighbour offset clamped to 0 at the domain edge.
 * Restates src/simulator/single_dev_expt/kernel.cu:2504-2569. */
static void FN(orc_pull)(int64_t nx, int64_t ny, int64_t nz, int64_t x, int64_t y, int64_t z,
                         const REAL *src, REAL *f)
{
    const int64_t n = nx * ny * nz;
    const int64_t i = (ny * z + y) * nx + x;
    const int64_t ndx = (x == 0) ? 0 : -1, pdx = (x == nx - 1) ? 0 : 1;
    const int64_t ndy = (y == 0) ? 0 : -nx, pdy = (y == ny - 1) ? 0 : nx;
    const int64_t ndz = (z == 0) ? 0 : -nx * ny, pdz = (z == nz - 1) ? 0 : nx * ny;
    for (int d = 0; d < 27; ++d) {
        const int cx = d % 3 - 1, cy = (d / 3) % 3 - 1, cz = d / 9 - 1;
        /* neighbour at -c: a population moving in +x comes from x-1 */
        const int64_t ox = (cx == 1) ? ndx : (cx == -1) ? pdx : 0;
        const int64_t oy = (cy == 1) ? ndy : (cy == -1) ? pdy : 0;
        const int64_t oz = (cz == 1) ? ndz : (cz == -1) ? pdz : 0;
        f[d] = src[(int64_t)d * n + i + ox + oy + oz];
    }
}

/* One fused pull-stream + EQU + bounce-back + BGK step over the whole domain,
 * double buffer src -> dst.  Cells without STORE leave dst untouched; cells
 * with neither LOAD nor EQU start from zero populations.
 * Restates StaticD3Q27PullKernel, src/simulator/single_dev_expt/kernel.cu:2489-2632. */
void FN(orc_step)(int64_t nx, int64_t ny, int64_t nz, const uint32_t *flag,
                  const float *rho, const float *vx, const float *vy, const float *vz,
                  REAL inv_tau, const REAL *src, REAL *dst)
{
    const int64_t n = nx * ny * nz;
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t i = (ny * z + y) * nx + x;
                const uint32_t fl = flag[i];
                REAL f[27];
                for (int d = 0; d < 27; ++d) f[d] = 0;
                if (fl & ORC_LOAD) FN(orc_pull)(nx, ny, nz, x, y, z, src, f);
                FN(orc_cell)(fl, inv_tau, (REAL)rho[i], (REAL)vx[i], (REAL)vy[i], (REAL)vz[i], f);
                if (fl & ORC_STORE)
                    for (int d = 0; d < 27; ++d) dst[(int64_t)d * n + i] = f[d];
            }
}

/* Moments of the pulled populations of src, written to rho/vx/vy/vz only
 * where the matching DUMP bit is set (no EQU, bounce-back or collision).
 * Restates StaticD3Q27PullDumpKernel, src/simulator/single_dev_expt/kernel.cu:2634-2735. */
void FN(orc_moments)(int64_t nx, int64_t ny, int64_t nz, const uint32_t *flag, const REAL *src,
                     float *rho, float *vx, float *vy, float *vz)
{
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t i = (ny * z + y) * nx + x;
                const uint32_t fl = flag[i];
                REAL f[27], r, ux, uy, uz;
                FN(orc_pull)(nx, ny, nz, x, y, z, src, f);
                FN(orc_rhou)(f, &r, &ux, &uy, &uz);
                if (fl & ORC_DUMP_RHO) rho[i] = (float)r;
                if (fl & ORC_DUMP_VX) vx[i] = (float)ux;
                if (fl & ORC_DUMP_VY) vy[i] = (float)uy;
                if (fl & ORC_DUMP_VZ) vz[i] = (float)uz;
            }
}

/* The 27 populations every cell would load at the next step (pull with the
 * clamped edge), laid out out[d*n + i].  This is the state all streaming
 * policies must agree on. */
void FN(orc_pulled)(int64_t nx, int64_t ny, int64_t nz, const REAL *src, REAL *out)
{
    const int64_t n = nx * ny * nz;
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t i = (ny * z + y) * nx + x;
                REAL f[27];
                FN(orc_pull)(nx, ny, nz, x, y, z, src, f);
                for (int d = 0; d < 27; ++d) out[(int64_t)d * n + i] = f[d];
            }
}

/* Rest-equilibrium fill of a 27 x n buffer (calcEqu(1,0,0,0) per direction).
 * Restates Simulator::Data::initDoubleDDFBuf,
 * src/simulator/single_dev_expt/simulator_expt_platform.cu:230-250. */
void FN(orc_fill_rest)(int64_t n, REAL *buf)
{
    REAL feq[27];
    FN(orc_equ)((REAL)1, (REAL)0, (REAL)0, (REAL)0, feq);
    for (int d = 0; d < 27; ++d)
        for (int64_t i = 0; i < n; ++i) buf[(int64_t)d * n + i] = feq[d];
}

/* nsteps pull steps starting from buffer a; returns 0 if the newest state is
 * in a, 1 if it is in b (the reference swaps src/dst after every launch,
 * simulator_expt_platform.cu:974-978). */
int FN(orc_run)(int64_t nx, int64_t ny, int64_t nz, const uint32_t *flag,
                const float *rho, const float *vx, const float *vy, const float *vz,
                REAL inv_tau, int64_t nsteps, REAL *a, REAL *b)
{
    REAL *src = a, *dst = b;
    for (int64_t s = 0; s < nsteps; ++s) {
        FN(orc_step)(nx, ny, nz, flag, rho, vx, vy, vz, inv_tau, src, dst);
        REAL *t = src; src = dst; dst = t;
    }
    return src == a ? 0 : 1;
}

#undef FN
#undef CAT
#undef CAT2
