"""Tensor-op D3Q27 step with soft obstacles in PyTorch (FP64, CPU), the
autograd reference for the adjoint tests.

Same model as the adjoint of culbm_b200: pull with the reference's per-axis
clamp (src/simulator/single_dev_expt/kernel.cu:2504-2569), EQU overwrite,
full-way bounce-back swap, BGK on shifted populations with partial
bounce-back f' = C(f) + s (B(f) - C(f)); objective = mean over the window of
(mean rho/3 on the inlet plane - mean rho/3 on the outlet plane), rho from
the pulled populations.  Straight tensor algebra, no fused arithmetic.
"""
import numpy as np
import torch

LOAD, EQU, COLLIDE, BOUNCE_BACK, STORE = 1, 2, 4, 8, 16

D = np.arange(27)
CX, CY, CZ = D % 3 - 1, (D // 3) % 3 - 1, D // 9 - 1
W = np.array([{0: 8 / 27, 1: 2 / 27, 2: 1 / 54, 3: 1 / 216}[int(k)]
              for k in (CX != 0).astype(int) + (CY != 0) + (CZ != 0)])
OPP = 26 - D


def sources(nx, ny, nz):
    """For each direction d, the flat index every cell pulls d from."""
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = []
    for d in range(27):
        sx = np.clip(x - CX[d], 0, nx - 1)
        sy = np.clip(y - CY[d], 0, ny - 1)
        sz = np.clip(z - CZ[d], 0, nz - 1)
        out.append(torch.from_numpy((sx + nx * (sy + ny * sz)).reshape(-1)))
    return out


def feq(rho, ux, uy, uz):
    c = torch.from_numpy(np.stack([CX, CY, CZ])).to(torch.float64)
    w = torch.from_numpy(W).to(torch.float64)[:, None]
    cu = c[0][:, None] * ux + c[1][:, None] * uy + c[2][:, None] * uz
    uu = ux * ux + uy * uy + uz * uz
    return w * (rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * uu) - 1)


def pressure_drop(dims, flag, rho_in, vx_in, vy_in, vz_in, soft, inv_tau, window, planes):
    """J as a differentiable function of soft (N), inv_tau (scalar), vx_in (N)."""
    nx, ny, nz = dims
    n = nx * ny * nz
    src = sources(nx, ny, nz)
    fl = torch.from_numpy(flag.astype(np.int64))
    is_equ = (fl & EQU) != 0
    is_bb = (fl & BOUNCE_BACK) != 0
    is_col = (fl & COLLIDE) != 0
    is_load = (fl & LOAD) != 0
    is_store = (fl & STORE) != 0
    c = torch.from_numpy(np.stack([CX, CY, CZ])).to(torch.float64)
    x = torch.arange(n) % nx
    in_mask = is_col & (x == planes[0])
    out_mask = is_col & (x == planes[1])
    F = torch.zeros(27, n, dtype=torch.float64)
    fe = feq(rho_in, vx_in, vy_in, vz_in)
    opp = torch.from_numpy(OPP)

    def pulled(F):
        return torch.stack([F[d][src[d]] for d in range(27)])

    def obj_term(F):
        r = 1 + pulled(F).sum(0)
        return r[in_mask].mean() / 3 - r[out_mask].mean() / 3

    J = 0.0
    t0, t1 = window
    if t0 == 0:
        J = J + obj_term(F)
    for t in range(t1):
        f = torch.where(is_load, pulled(F), torch.zeros_like(F))
        f = torch.where(is_equ, fe, f)
        f = torch.where(is_bb, f[opp], f)
        rho = 1 + f.sum(0)
        u = (c @ f) / rho
        C = inv_tau * feq(rho, u[0], u[1], u[2]) + (1 - inv_tau) * f
        f3 = C + soft * (f[opp] - C)
        f = torch.where(is_col, f3, f)
        F = torch.where(is_store, f, F)
        if t0 <= t + 1 <= t1:
            J = J + obj_term(F)
    return J / (t1 - t0 + 1)
