"""Gradients of the channel pressure drop through the discrete adjoint
(``culbm_adj_*`` in include/culbm.h), and a ``torch.autograd.Function``
over it.

Model: the D3Q27 BGK step in which each COLLIDE cell carries a soft-obstacle
value s in [0, 1] applied as partial bounce-back, f' = C(f) + s (B(f) - C(f)).
Objective: J = mean over the states after t in [t0, t1] steps of
(mean rho/3 on the inlet plane - mean rho/3 on the outlet plane).
Gradients: dJ/ds (per cell), dJ/d invTau, dJ/d of the EQU inputs (the inlet
profile), all accumulated in FP64 on the GPU over checkpointed recomputation.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import check, lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class AdjointProblem:
    """One culbm_adj handle: geometry, objective window, checkpointing."""

    def __init__(self, domain: Sequence[int], window=(300, 500), planes=(1, None), inv_tau=0.5,
                 checkpoint_every: int = 50, precision: str = "fp32", storage: Optional[str] = None,
                 hbm_budget_bytes: int = 0, dev_id: int = 0, checkpoint_inner: int = 0,
                 checkpoint_storage: Optional[str] = None):
        """checkpoint_storage ("fp16sr" or "fp16" with storage "fp32"): the
        forward pass and J in FP32, its checkpoints and the recomputed states
        of the reverse sweep in that 16-bit format."""
        cfg = _capi.AdjConfig()
        check(lib().culbm_adj_config_init(C.byref(cfg)))
        cfg.dev_id = dev_id
        for k in range(3):
            cfg.domain_dim[k] = int(domain[k])
        cfg.inv_tau = float(inv_tau)
        cfg.window[0], cfg.window[1] = int(window[0]), int(window[1])
        cfg.plane_x[0] = int(planes[0])
        cfg.plane_x[1] = -1 if planes[1] is None else int(planes[1])
        cfg.checkpoint_every = int(checkpoint_every)
        cfg.precision = {"fp32": 0, "fp64": 1}[precision]
        if storage is None:
            storage = "fp64" if precision == "fp64" else "fp32"
        cfg.storage = _capi.STORAGE[storage]
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.checkpoint_inner = int(checkpoint_inner)
        cfg.checkpoint_storage = 0 if checkpoint_storage is None else _capi.STORAGE[checkpoint_storage]
        self.domain = tuple(int(v) for v in domain)
        self.n = self.domain[0] * self.domain[1] * self.domain[2]
        self._h = C.c_void_p()
        check(lib().culbm_adj_create(C.byref(cfg), C.byref(self._h)))

    def close(self):
        if self._h:
            lib().culbm_adj_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, flag=None, rho=None, vx=None, vy=None, vz=None, soft=None):
        arrs = []
        for a, dt in ((flag, np.uint32), (rho, np.float32), (vx, np.float32), (vy, np.float32), (vz, np.float32),
                      (soft, np.float32)):
            arrs.append(None if a is None else np.ascontiguousarray(a, dtype=dt).reshape(-1))
        for a in arrs:
            if a is not None and a.size != self.n:
                raise ValueError(f"expected {self.n} values, got {a.size}")
        self._keep = arrs
        check(lib().culbm_adj_set_state(self._h, *[_ptr(a) for a in arrs]))

    def set_inv_tau(self, inv_tau: float):
        check(lib().culbm_adj_set_inv_tau(self._h, float(inv_tau)))

    def forward(self) -> float:
        j = C.c_double()
        check(lib().culbm_adj_forward(self._h, C.byref(j)))
        return j.value

    def gradient(self):
        """(J, dJ/dinvTau, dJ/ds [N], dJ/d(rho, vx, vy, vz) of the EQU inputs [4, N])."""
        j, gt = C.c_double(), C.c_double()
        gs = np.zeros(self.n, np.float64)
        gm = np.zeros(4 * self.n, np.float64)
        check(lib().culbm_adj_gradient(self._h, C.byref(j), C.byref(gt), _ptr(gs), _ptr(gm)))
        return j.value, gt.value, gs, gm.reshape(4, self.n)

    def info(self) -> dict:
        inf = _capi.AdjInfo()
        check(lib().culbm_adj_get_info(self._h, C.byref(inf)))
        return {"checkpoint_every": inf.checkpoint_every, "checkpoints": inf.checkpoints,
                "checkpoint_inner": inf.checkpoint_inner, "inner_checkpoints": inf.inner_checkpoints,
                "device_bytes": inf.device_bytes, "forward_ms": inf.forward_ms, "recompute_ms": inf.recompute_ms,
                "adjoint_ms": inf.adjoint_ms, "steps": inf.steps}


def _torch():
    import torch
    return torch


class PressureDrop:
    """Differentiable J(soft, inv_tau, inlet_vx) for a fixed geometry.

    ``soft`` has N entries, ``inlet_vx`` N entries (used at EQU cells only);
    rho/vy/vz of the EQU cells stay fixed.  Call through :meth:`apply`.
    """

    def __init__(self, problem: AdjointProblem, flag, rho=None, vy=None, vz=None):
        self.problem = problem
        self.flag = np.ascontiguousarray(flag, np.uint32).reshape(-1)
        n = problem.n
        self.rho = np.ones(n, np.float32) if rho is None else np.ascontiguousarray(rho, np.float32).reshape(-1)
        self.vy = np.zeros(n, np.float32) if vy is None else np.ascontiguousarray(vy, np.float32).reshape(-1)
        self.vz = np.zeros(n, np.float32) if vz is None else np.ascontiguousarray(vz, np.float32).reshape(-1)

    def apply(self, soft, inv_tau, inlet_vx):
        return _PressureDropFn.apply(soft, inv_tau, inlet_vx, self)


def _make_fn():
    torch = _torch()

    class PressureDropFn(torch.autograd.Function):
        """torch.autograd.Function over culbm_adj_gradient: forward runs the
        adjoint once and keeps the gradients; backward scales them."""

        @staticmethod
        def forward(ctx, soft, inv_tau, inlet_vx, pd):
            p = pd.problem
            s_np = soft.detach().to("cpu", torch.float32).numpy()
            vx_np = inlet_vx.detach().to("cpu", torch.float32).numpy()
            p.set_state(pd.flag, pd.rho, vx_np, pd.vy, pd.vz, s_np)
            p.set_inv_tau(float(inv_tau.detach().cpu()))
            J, g_tau, g_soft, g_mac = p.gradient()
            ctx.save_for_backward(torch.from_numpy(g_soft).to(soft.device, soft.dtype),
                                  torch.tensor(g_tau, dtype=inv_tau.dtype, device=inv_tau.device),
                                  torch.from_numpy(g_mac[1]).to(inlet_vx.device, inlet_vx.dtype))
            return torch.tensor(J, dtype=torch.float64, device=soft.device)

        @staticmethod
        def backward(ctx, gJ):
            g_soft, g_tau, g_vx = ctx.saved_tensors
            return gJ.to(g_soft.dtype) * g_soft, gJ.to(g_tau.dtype) * g_tau, gJ.to(g_vx.dtype) * g_vx, None

    return PressureDropFn


class _Lazy:
    fn = None

    @classmethod
    def apply(cls, *args):
        if cls.fn is None:
            cls.fn = _make_fn()
        return cls.fn.apply(*args)


_PressureDropFn = _Lazy


def main(argv=None):
    """Run one gradient of the pressure drop on the soft-obstacle channel and
    print J, the gradient norms and the timings (JSON)."""
    import argparse
    import json

    from . import scenes
    ap = argparse.ArgumentParser(prog="python -m culbm_b200.adjoint", description=main.__doc__)
    ap.add_argument("--domain", type=int, nargs=3, default=(128, 64, 64))
    ap.add_argument("--window", type=int, nargs=2, default=(300, 500))
    ap.add_argument("--checkpoint-every", type=int, default=50, help="0: smallest plan within --hbm-budget-gb")
    ap.add_argument("--checkpoint-inner", type=int, default=0)
    ap.add_argument("--hbm-budget-gb", type=float, default=0.0)
    ap.add_argument("--bumps", type=int, default=16)
    ap.add_argument("--precision", choices=("fp32", "fp64"), default="fp32")
    ap.add_argument("--storage", default=None)
    ap.add_argument("--inv-tau", type=float, default=0.5)
    args = ap.parse_args(argv)
    sc, soft = scenes.adjoint_channel(*args.domain, u_peak=0.04, bumps=args.bumps)
    f, r, ux, uy, uz = sc.arrays()
    with AdjointProblem(args.domain, window=args.window, checkpoint_every=args.checkpoint_every,
                        checkpoint_inner=args.checkpoint_inner, hbm_budget_bytes=int(args.hbm_budget_gb * 1e9),
                        precision=args.precision, storage=args.storage, inv_tau=args.inv_tau) as p:
        p.set_state(f, r, ux, uy, uz, soft.reshape(-1))
        J, g_tau, g_soft, g_mac = p.gradient()
        info = p.info()
    print(json.dumps({"J": J, "dJ_dinv_tau": g_tau, "dJ_dsoft_norm": float(np.linalg.norm(g_soft)),
                      "dJ_dvx_in_norm": float(np.linalg.norm(g_mac[1])), **info}))


if __name__ == "__main__":
    main()
