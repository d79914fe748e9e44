"""Python front end over the C ABI: one D3Q27 BGK simulation on one GPU.

Mirrors what the reference's ``Simulator`` does between argv parsing and the
dump files (src/simulator/single_dev_expt/simulator_expt_platform.cu), with
numpy arrays instead of files.  All compute runs in libculbm.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import check, lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Simulation:
    """A culbm_sim handle.

    ``domain`` is (nx, ny, nz).  For the blocked policies (opt_policy 1..3)
    ``tile`` (or block_dim*grid_dim) is the tile extent including its halo,
    as in the reference.  For the plain pull policy (0, 0) the reference
    requires block_dim*grid_dim == domain; when neither is given the
    whole domain is used.
    """

    def __init__(self, domain: Sequence[int], stream_policy: int = 0, opt_policy: int = 0,
                 inv_tau: float = 0.5, inner_loop: int = 5, storage: str = "fp32",
                 block_dim: Optional[Sequence[int]] = None, grid_dim: Optional[Sequence[int]] = None,
                 tile: Optional[Sequence[int]] = None, use_ring: bool = False, dev_id: int = 0,
                 persist_l2: bool = False, cache_hints: bool = True, use_graphs: bool = True,
                 kernel_variant: int = 0, run_slabs: int = 0):
        cfg = _capi.default_config()
        cfg.dev_id = dev_id
        for k in range(3):
            cfg.domain_dim[k] = int(domain[k])
        if tile is not None:
            block_dim, grid_dim = tile, (1, 1, 1)
        if block_dim is None and grid_dim is None:
            block_dim, grid_dim = domain, (1, 1, 1)
        if block_dim is not None:
            for k in range(3):
                cfg.block_dim[k] = int(block_dim[k])
        if grid_dim is not None:
            for k in range(3):
                cfg.grid_dim[k] = int(grid_dim[k])
        cfg.stream_policy = int(stream_policy)
        cfg.opt_policy = int(opt_policy)
        cfg.inv_tau = float(inv_tau)
        cfg.inner_loop = int(inner_loop)
        cfg.storage = _capi.STORAGE[storage] if isinstance(storage, str) else int(storage)
        cfg.use_ring_ddf_buf = int(bool(use_ring))
        cfg.persist_l2 = int(bool(persist_l2))
        cfg.cache_hints = int(bool(cache_hints))
        cfg.use_graphs = int(bool(use_graphs))
        cfg.kernel_variant = int(kernel_variant)
        cfg.run_slabs = int(run_slabs)
        self.cfg = cfg
        self.domain = tuple(int(v) for v in domain)
        self.n = self.domain[0] * self.domain[1] * self.domain[2]
        self._h = C.c_void_p()
        check(lib().culbm_create(C.byref(cfg), C.byref(self._h)))

    # ---------------------------------------------------------------- life
    def close(self) -> None:
        if self._h:
            lib().culbm_destroy(self._h)
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

    # --------------------------------------------------------------- state
    def load_state(self, flag=None, rho=None, vx=None, vy=None, vz=None) -> None:
        arrs = []
        for a, dt in ((flag, np.uint32), (rho, np.float32), (vx, np.float32), (vy, np.float32), (vz, np.float32)):
            if a is None:
                arrs.append(None)
                continue
            a = np.ascontiguousarray(a, dtype=dt).reshape(-1)
            if a.size != self.n:
                raise ValueError(f"expected {self.n} values, got {a.size}")
            arrs.append(a)
        check(lib().culbm_load_state(self._h, *[_ptr(a) for a in arrs]))

    def load_folder(self, folder: str) -> int:
        mask = C.c_uint32(0)
        check(lib().culbm_load_state_folder(self._h, folder.encode(), C.byref(mask)))
        return mask.value

    def set_ddf(self, ddf: np.ndarray) -> None:
        ddf = np.ascontiguousarray(ddf)
        if ddf.size != 27 * self.n or ddf.dtype not in (np.float32, np.float64):
            raise ValueError("expected 27*N float32 or float64 values")
        check(lib().culbm_set_ddf(self._h, _ptr(ddf), 0 if ddf.dtype == np.float32 else 1))

    # ---------------------------------------------------------------- steps
    def step(self, nsteps: int) -> None:
        check(lib().culbm_step(self._h, int(nsteps)))

    def step_timed(self, nsteps: int) -> float:
        ms = C.c_float(0.0)
        check(lib().culbm_step_timed(self._h, int(nsteps), C.byref(ms)))
        return ms.value

    def synchronize(self) -> None:
        check(lib().culbm_synchronize(self._h))

    @property
    def step_count(self) -> int:
        v = C.c_uint64(0)
        check(lib().culbm_get_step(self._h, C.byref(v)))
        return v.value

    def run_host(self, nsteps: int, flag=None, rho=None, vx=None, vy=None, vz=None, out=None):
        """load_state, ``nsteps`` steps, moments and the four fields in one call
        (culbm_run_host): the slabs' copies overlap the steps when the arrays
        are page-locked.  ``out`` is four float32 arrays of N values (new ones
        when None); returns them as (rho, vx, vy, vz)."""
        arrs = []
        for a, dt in ((flag, np.uint32), (rho, np.float32), (vx, np.float32), (vy, np.float32), (vz, np.float32)):
            if a is None:
                arrs.append(None)
                continue
            if not (isinstance(a, np.ndarray) and a.dtype == dt and a.flags.c_contiguous):
                a = np.ascontiguousarray(a, dtype=dt)
            a = a.reshape(-1)
            if a.size != self.n:
                raise ValueError(f"expected {self.n} values, got {a.size}")
            arrs.append(a)
        if out is None:
            out = tuple(np.empty(self.n, dtype=np.float32) for _ in range(4))
        for o in out:
            if not (isinstance(o, np.ndarray) and o.dtype == np.float32 and o.flags.c_contiguous and o.size == self.n):
                raise ValueError(f"each output must be a contiguous float32 array of {self.n} values")
        check(lib().culbm_run_host(self._h, *[_ptr(a) for a in arrs], int(nsteps), *[_ptr(o) for o in out]))
        return tuple(out)

    # -------------------------------------------------------------- outputs
    def moments(self) -> None:
        check(lib().culbm_moments(self._h))

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float32)
        check(lib().culbm_get_field(self._h, _capi.FIELD[name], _ptr(out)))
        return out

    def fields(self):
        return tuple(self.field(k) for k in ("rho", "vx", "vy", "vz"))

    def dump(self, folder: str, rho=False, vx=False, vy=False, vz=False) -> None:
        mask = (1 if rho else 0) | (2 if vx else 0) | (4 if vy else 0) | (8 if vz else 0)
        check(lib().culbm_dump(self._h, folder.encode(), mask))

    def pulled_ddf(self, dtype=np.float32) -> np.ndarray:
        out = np.empty(27 * self.n, dtype=dtype)
        check(lib().culbm_get_pulled_ddf(self._h, _ptr(out), 0 if out.dtype == np.float32 else 1))
        return out

    def mass_momentum(self) -> np.ndarray:
        out = (C.c_double * 4)()
        check(lib().culbm_mass_momentum(self._h, out))
        return np.array(out[:], dtype=np.float64)

    def info(self) -> dict:
        inf = _capi.Info()
        check(lib().culbm_get_info(self._h, C.byref(inf)))
        return {
            "cells": inf.cells, "device_bytes": inf.device_bytes,
            "blocking_num": tuple(inf.blocking_num), "blocking_dim": tuple(inf.blocking_dim),
            "storage": inf.storage, "stream_policy": inf.stream_policy, "opt_policy": inf.opt_policy,
            "inner_loop": inf.inner_loop, "persisting_l2_bytes": inf.persisting_l2_bytes,
            "launches_per_step": inf.kernel_launches_per_step_x1000 / 1000.0,
        }
