"""Discrete adjoint (GPU): gradients of the channel pressure drop with respect
to the soft-obstacle field, invTau and the inlet profile.

Checks: PyTorch autograd of a tensor-op D3Q27 step (FP64, CPU); FP64 central
finite differences with h = 1e-6 on the 32x16x16 case; checkpoint-stride
invariance; FP32 against FP64; the torch.autograd.Function shim; s = 0 gives
the plain step's objective.
"""
import numpy as np
import pytest
import torch

from culbm_b200 import scenes as S
from culbm_b200.adjoint import AdjointProblem, PressureDrop

from torch_d3q27 import pressure_drop

pytestmark = pytest.mark.gpu


def case(nx, ny, nz, bumps, seed=7):
    sc, soft = S.adjoint_channel(nx, ny, nz, u_peak=0.04, bumps=bumps, seed=seed)
    f, r, ux, uy, uz = sc.arrays()
    return sc, f, r, ux, uy, uz, soft.reshape(-1)


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_adjoint_matches_torch_autograd():
    dims = (14, 8, 8)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=3)
    window, planes, w = (15, 30), (1, dims[0] - 2), 0.6
    with AdjointProblem(dims, window=window, planes=planes, inv_tau=w, checkpoint_every=7, precision="fp64") as p:
        p.set_state(f, r, ux, uy, uz, soft)
        J, g_tau, g_soft, g_mac = p.gradient()
    ts = torch.tensor(soft.astype(np.float64), requires_grad=True)
    tw = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    tvx = torch.tensor(ux.astype(np.float64), requires_grad=True)
    Jt = pressure_drop(dims, f, torch.tensor(r, dtype=torch.float64), tvx, torch.tensor(uy, dtype=torch.float64),
                       torch.tensor(uz, dtype=torch.float64), ts, tw, window, planes)
    Jt.backward()
    # J is a difference of plane means near 1/3: rounding differences of the two
    # FP64 step implementations show up at the 1e-13 absolute level
    assert abs(J - Jt.item()) <= 1e-8 * abs(Jt.item())
    # FP64 both sides; the small J (a difference of means near 1/3) lifts the
    # relative rounding differences of the two implementations to ~1e-8
    assert rel(g_soft, ts.grad.numpy()) < 1e-6
    assert abs(g_tau - tw.grad.item()) <= 1e-6 * abs(tw.grad.item())
    equ = (f & S.EQU) != 0
    assert rel(g_mac[1][equ], tvx.grad.numpy()[equ]) < 1e-6
    assert np.abs(ts.grad.numpy()).max() > 0


@pytest.fixture(scope="module")
def fd_case():
    dims = (32, 16, 16)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=16)
    p = AdjointProblem(dims, window=(300, 500), inv_tau=0.5, checkpoint_every=50, precision="fp64")
    p.set_state(f, r, ux, uy, uz, soft)
    J, g_tau, g_soft, g_mac = p.gradient()
    yield dict(p=p, dims=dims, f=f, r=r, ux=ux, uy=uy, uz=uz, soft=soft, J=J, g_tau=g_tau, g_soft=g_soft,
               g_mac=g_mac)
    p.close()


def test_fd_invtau(fd_case):
    c, h = fd_case, 1e-6
    p = c["p"]
    p.set_inv_tau(0.5 + h)
    jp = p.forward()
    p.set_inv_tau(0.5 - h)
    jm = p.forward()
    p.set_inv_tau(0.5)
    fd = (jp - jm) / (2 * h)
    assert abs(fd - c["g_tau"]) <= 1e-4 * abs(fd), (fd, c["g_tau"])


def _fd_field(c, key, idx, h=1e-6):
    p = c["p"]
    base = c[key].copy()
    out = []
    for i in idx:
        plus, minus = base.copy(), base.copy()
        plus[i] = np.float32(base[i] + h)
        minus[i] = np.float32(base[i] - h)
        args = {k: c[k] for k in ("f", "r", "ux", "uy", "uz", "soft")}
        args[key] = plus
        p.set_state(args["f"], args["r"], args["ux"], args["uy"], args["uz"], args["soft"])
        jp = p.forward()
        args[key] = minus
        p.set_state(args["f"], args["r"], args["ux"], args["uy"], args["uz"], args["soft"])
        jm = p.forward()
        out.append((jp - jm) / (float(plus[i]) - float(minus[i])))
    p.set_state(c["f"], c["r"], c["ux"], c["uy"], c["uz"], c["soft"])
    return np.array(out)


def test_fd_soft_field(fd_case):
    c = fd_case
    g = c["g_soft"]
    inner = (c["soft"] > 0.02) & (c["soft"] < 0.98)
    cand = np.flatnonzero(inner)
    idx = cand[np.argsort(-np.abs(g[cand]))[:6]]
    fd = _fd_field(c, "soft", idx)
    for i, a, b in zip(idx, g[idx], fd):
        assert abs(a - b) <= 1e-4 * abs(b), (i, a, b)


def test_fd_inlet_profile(fd_case):
    c = fd_case
    g = c["g_mac"][1]
    inlet = np.flatnonzero(((c["f"] & S.EQU) != 0) & (c["ux"] > 0.01))
    idx = inlet[np.argsort(-np.abs(g[inlet]))[:4]]
    fd = _fd_field(c, "ux", idx)
    for i, a, b in zip(idx, g[idx], fd):
        assert abs(a - b) <= 1e-4 * abs(b), (i, a, b)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_checkpoint_plan_does_not_change_gradients(precision):
    """One level with K = 1, 7, 60 and two levels (K, K2) = (20, 3), (13, 12):
    recomputation is deterministic, so the gradients agree bit for bit."""
    dims = (20, 10, 10)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=4)
    outs = []
    for K, K2 in ((1, 0), (7, 0), (60, 0), (20, 3), (13, 12)):
        with AdjointProblem(dims, window=(30, 60), checkpoint_every=K, checkpoint_inner=K2,
                            precision=precision) as p:
            p.set_state(f, r, ux, uy, uz, soft)
            outs.append(p.gradient())
            assert p.info()["checkpoint_inner"] == K2
    for o in outs[1:]:
        assert o[0] == outs[0][0] and o[1] == outs[0][1]
        assert np.array_equal(o[2], outs[0][2]) and np.array_equal(o[3], outs[0][3])


def test_automatic_plan_fits_the_budget():
    """checkpoint_every = 0: one level near sqrt(t1) when it fits, two levels
    under a budget too small for that, and a clear error below any plan."""
    dims = (32, 16, 16)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=4)
    state = 27 * f.size * 4
    with AdjointProblem(dims, window=(100, 400), checkpoint_every=0) as p:
        one = p.info()
        p.set_state(f, r, ux, uy, uz, soft)
        ref = p.gradient()
    assert one["checkpoint_inner"] == 0 and 15 <= one["checkpoint_every"] <= 25
    budget = one["device_bytes"] - 12 * state
    with AdjointProblem(dims, window=(100, 400), checkpoint_every=0, hbm_budget_bytes=budget) as p:
        two = p.info()
        p.set_state(f, r, ux, uy, uz, soft)
        got = p.gradient()
    assert two["checkpoint_inner"] > 0 and two["device_bytes"] <= budget
    assert got[0] == ref[0] and got[1] == ref[1] and np.array_equal(got[2], ref[2])
    from culbm_b200._capi import CulbmError
    with pytest.raises(CulbmError, match="no checkpoint plan fits"):
        AdjointProblem(dims, window=(100, 400), checkpoint_every=0, hbm_budget_bytes=budget // 4)


def test_fp32_adjoint_close_to_fp64():
    dims = (32, 16, 16)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=16)
    res = {}
    for prec in ("fp32", "fp64"):
        with AdjointProblem(dims, window=(100, 200), checkpoint_every=20, precision=prec) as p:
            p.set_state(f, r, ux, uy, uz, soft)
            res[prec] = p.gradient()
    assert abs(res["fp32"][0] - res["fp64"][0]) <= 1e-4 * abs(res["fp64"][0])
    assert rel(res["fp32"][2], res["fp64"][2]) < 1e-3
    assert abs(res["fp32"][1] - res["fp64"][1]) <= 1e-3 * abs(res["fp64"][1])


@pytest.mark.parametrize("ck,tol", [("fp16sr", 1e-3), ("fp16", 1e-2)])
def test_fp32_forward_with_16bit_checkpoints(ck, tol):
    """checkpoint_storage: the forward pass runs in FP32 (J bit for bit that
    of the FP32 mode), checkpoints and the reverse sweep's states are 16-bit.
    The gradients stay within `tol` (relative L2) of the FP32 mode's, closer
    than those of the all-16-bit mode, whose forward trajectory itself is
    rounded every step (nearest-even checkpoints drift more than stochastic
    ones)."""
    dims = (48, 24, 24)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=8)
    res, info = {}, {}
    for name, kw in (("fp32", {}), ("mixed", {"checkpoint_storage": ck}), ("all16", {"storage": ck})):
        with AdjointProblem(dims, window=(60, 120), checkpoint_every=12, **kw) as p:
            p.set_state(f, r, ux, uy, uz, soft)
            res[name] = p.gradient()
            info[name] = p.info()
            assert p.forward() == res[name][0]
    assert res["mixed"][0] == res["fp32"][0]
    e_mixed, e_all16 = rel(res["mixed"][2], res["fp32"][2]), rel(res["all16"][2], res["fp32"][2])
    assert e_mixed < tol and e_mixed < e_all16, (e_mixed, e_all16)
    assert abs(res["mixed"][1] - res["fp32"][1]) <= tol * abs(res["fp32"][1])
    assert rel(res["mixed"][3][1], res["fp32"][3][1]) < tol
    assert info["mixed"]["checkpoint_every"] == 12


def test_torch_shim_backward():
    dims = (16, 8, 8)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=3)
    with AdjointProblem(dims, window=(10, 20), checkpoint_every=5, precision="fp64") as p:
        pd = PressureDrop(p, f, r, uy, uz)
        ts = torch.tensor(soft, dtype=torch.float64, requires_grad=True)
        tw = torch.tensor(0.5, dtype=torch.float64, requires_grad=True)
        tvx = torch.tensor(ux, dtype=torch.float64, requires_grad=True)
        J = pd.apply(ts, tw, tvx)
        (2.0 * J).backward()
        p.set_state(f, r, ux, uy, uz, soft)
        p.set_inv_tau(0.5)
        J2, g_tau, g_soft, g_mac = p.gradient()
    assert J.item() == J2
    assert np.allclose(ts.grad.numpy(), 2 * g_soft, rtol=0, atol=0)
    assert tw.grad.item() == 2 * g_tau
    assert np.array_equal(tvx.grad.numpy(), 2 * g_mac[1])


def test_zero_soft_field_is_the_plain_step(culbm):
    dims = (24, 12, 10)
    sc, f, r, ux, uy, uz, soft = case(*dims, bumps=2)
    window = (5, 15)
    with AdjointProblem(dims, window=window, checkpoint_every=5) as p:
        p.set_state(f, r, ux, uy, uz, None)
        J = p.forward()
    coll = (f & S.COLLIDE) != 0
    x = np.arange(f.size) % dims[0]
    acc = 0.0
    with culbm.Simulation(dims, stream_policy=0, inv_tau=0.5) as sim:
        sim.load_state(f, r, ux, uy, uz)
        for t in range(window[1] + 1):
            if t >= window[0]:
                sim.moments()
                rho = sim.field("rho").astype(np.float64)
                acc += rho[coll & (x == 1)].mean() / 3 - rho[coll & (x == dims[0] - 2)].mean() / 3
            if t < window[1]:
                sim.step(1)
    assert abs(J - acc / (window[1] - window[0] + 1)) <= 1e-12 * abs(J)
