"""ORACLE — test infrastructure only.

ctypes bindings of the CPU checker libraries:

* ``liboracle.so`` — the C restatement of the reference's D3Q27 BGK pull step
  (``oracle/d3q27_oracle.c``), FP32 and FP64;
* ``_ref/libref_lbm_core.so`` — the reference's own lbm_core routines compiled
  for the host (``oracle/ref_lbm_core_host.cpp``), when it was built.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The product package ``culbm_b200`` never
does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_lbm_core.so")
REF_BIN_DIR = os.path.join(HERE, "_ref")

# Flag bits, reference src/simulator/single_dev_expt/local_config.hpp:12-22.
LOAD, EQU, COLLIDE, BOUNCE_BACK, STORE = 1 << 0, 1 << 1, 1 << 2, 1 << 3, 1 << 4
DUMP_RHO, DUMP_VX, DUMP_VY, DUMP_VZ, CORRECT = 1 << 27, 1 << 28, 1 << 29, 1 << 30, 1 << 31
DUMP_ALL = DUMP_RHO | DUMP_VX | DUMP_VY | DUMP_VZ

_i64 = C.c_int64
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so (and, when the reference tree is present, _ref/)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    """Load liboracle.so, building it on first use if needed."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for sfx, rp in (("f32", _f32p), ("f64", _f64p)):
            real = C.c_float if sfx == "f32" else C.c_double
            getattr(L, f"orc_equ_{sfx}").argtypes = [real, real, real, real, rp]
            getattr(L, f"orc_rhou_{sfx}").argtypes = [rp, C.POINTER(real), C.POINTER(real),
                                                      C.POINTER(real), C.POINTER(real)]
            getattr(L, f"orc_collide_{sfx}").argtypes = [real, rp]
            getattr(L, f"orc_cell_{sfx}").argtypes = [C.c_uint32, real, real, real, real, real, rp]
            getattr(L, f"orc_step_{sfx}").argtypes = [_i64, _i64, _i64, _u32p, _f32p, _f32p, _f32p, _f32p,
                                                      real, rp, rp]
            getattr(L, f"orc_moments_{sfx}").argtypes = [_i64, _i64, _i64, _u32p, rp, _f32p, _f32p, _f32p, _f32p]
            getattr(L, f"orc_pulled_{sfx}").argtypes = [_i64, _i64, _i64, rp, rp]
            getattr(L, f"orc_fill_rest_{sfx}").argtypes = [_i64, rp]
            getattr(L, f"orc_run_{sfx}").argtypes = [_i64, _i64, _i64, _u32p, _f32p, _f32p, _f32p, _f32p,
                                                     real, _i64, rp, rp]
            getattr(L, f"orc_run_{sfx}").restype = C.c_int
        u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
        L.orc_step_s16.argtypes = [C.c_int, _i64, _i64, _i64, _u32p, _f32p, _f32p, _f32p, _f32p, C.c_float,
                                   u16p, u16p, C.c_uint32]
        L.orc_decode_s16.argtypes = [C.c_int, _i64, u16p, _f32p]
        L.orc_cell_fast_f32.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
        L.orc_encode_s16.argtypes = [C.c_int, _i64, _f32p, u16p, C.c_uint32]
        L.orc_step_seed.argtypes = [C.c_uint32]
        L.orc_round16_sr_n.argtypes = [C.c_int, _i64, _f32p, _u32p, u16p]
        L.orc_sr_bits.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_sr_bits.restype = C.c_uint32
        L.orc_step_seed.restype = C.c_uint32
        L.orc_valid_blk_axis.argtypes = [C.c_uint32] * 3
        L.orc_valid_blk_axis.restype = C.c_int
        L.orc_blk_num.argtypes = [C.c_uint32] * 3
        L.orc_blk_num.restype = C.c_uint32
        L.orc_valid_prev.argtypes = [C.c_int32] * 5
        L.orc_valid_prev.restype = C.c_int32
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref():
    """The reference's lbm_core built for the host (oracle/_ref), or None."""
    global _ref
    if _ref is None and ref_available():
        L = C.CDLL(REF_LIB_PATH)
        L.ref_equ_f32.argtypes = [C.c_float] * 4 + [_f32p]
        L.ref_rhou_f32.argtypes = [_f32p] + [C.POINTER(C.c_float)] * 4
        L.ref_collide_f32.argtypes = [C.c_float, _f32p]
        L.ref_valid_blk_axis.argtypes = [C.c_uint32] * 3
        L.ref_valid_blk_axis.restype = C.c_int
        L.ref_blk_num.argtypes = [C.c_uint32] * 3
        L.ref_blk_num.restype = C.c_uint32
        L.ref_valid_prev.argtypes = [C.c_int32] * 5
        L.ref_valid_prev.restype = C.c_int32
        L.ref_step_f32.argtypes = [_i64, _i64, _i64, _u32p, _f32p, _f32p, _f32p, _f32p, C.c_float,
                                   _f32p, _f32p, _i64, _i64, C.c_int]
        L.ref_moments_f32.argtypes = [_i64, _i64, _i64, _u32p, _f32p, _f32p, _f32p, _f32p, _f32p, C.c_int]
        L.ref_max_threads.restype = C.c_int
        _ref = L
    return _ref


def _real(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def rest_state(n: int, dtype=np.float32) -> np.ndarray:
    buf = np.empty(27 * n, dtype=dtype)
    getattr(lib(), f"orc_fill_rest_{_real(dtype)}")(n, buf)
    return buf


def equ(rho, vx, vy, vz, dtype=np.float32) -> np.ndarray:
    f = np.zeros(27, dtype=dtype)
    getattr(lib(), f"orc_equ_{_real(dtype)}")(rho, vx, vy, vz, f)
    return f


def collide(inv_tau, f) -> np.ndarray:
    f = np.ascontiguousarray(f).copy()
    getattr(lib(), f"orc_collide_{_real(f.dtype)}")(inv_tau, f)
    return f


def rhou(f):
    real = C.c_float if f.dtype == np.float32 else C.c_double
    out = [real() for _ in range(4)]
    getattr(lib(), f"orc_rhou_{_real(f.dtype)}")(np.ascontiguousarray(f), *[C.byref(o) for o in out])
    return tuple(o.value for o in out)


class Scene:
    """Flags and macroscopic buffers of one init state (numpy, x-fastest)."""

    def __init__(self, nx, ny, nz, flag=None, rho=None, vx=None, vy=None, vz=None):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        n = self.n
        fluid = LOAD | COLLIDE | STORE | DUMP_ALL
        self.flag = np.ascontiguousarray(flag if flag is not None else np.full(n, fluid, np.uint32),
                                         dtype=np.uint32).reshape(-1)
        self.rho = np.ascontiguousarray(rho if rho is not None else np.ones(n, np.float32), np.float32).reshape(-1)
        self.vx = np.ascontiguousarray(vx if vx is not None else np.zeros(n, np.float32), np.float32).reshape(-1)
        self.vy = np.ascontiguousarray(vy if vy is not None else np.zeros(n, np.float32), np.float32).reshape(-1)
        self.vz = np.ascontiguousarray(vz if vz is not None else np.zeros(n, np.float32), np.float32).reshape(-1)

    @property
    def n(self):
        return self.nx * self.ny * self.nz


def step(scene: Scene, inv_tau, src, dst) -> None:
    getattr(lib(), f"orc_step_{_real(src.dtype)}")(scene.nx, scene.ny, scene.nz, scene.flag, scene.rho,
                                                   scene.vx, scene.vy, scene.vz, inv_tau, src, dst)


def run(scene: Scene, inv_tau, nsteps, dtype=np.float32, state=None):
    """nsteps pull steps from rest equilibrium (or from `state`); returns the newest DDF buffer."""
    a = rest_state(scene.n, dtype) if state is None else np.ascontiguousarray(state, dtype=dtype).copy()
    b = a.copy()
    which = getattr(lib(), f"orc_run_{_real(dtype)}")(scene.nx, scene.ny, scene.nz, scene.flag, scene.rho,
                                                      scene.vx, scene.vy, scene.vz, inv_tau, nsteps, a, b)
    return a if which == 0 else b


def moments(scene: Scene, ddf, rho=None, vx=None, vy=None, vz=None):
    """Dump kernel semantics: returns (rho, vx, vy, vz) after writing the DUMP-bit cells over the inputs."""
    out = [np.array(a if a is not None else b, dtype=np.float32, copy=True)
           for a, b in ((rho, scene.rho), (vx, scene.vx), (vy, scene.vy), (vz, scene.vz))]
    getattr(lib(), f"orc_moments_{_real(ddf.dtype)}")(scene.nx, scene.ny, scene.nz, scene.flag,
                                                      np.ascontiguousarray(ddf), *out)
    return tuple(out)


def pulled(scene: Scene, ddf):
    out = np.empty_like(ddf)
    getattr(lib(), f"orc_pulled_{_real(ddf.dtype)}")(scene.nx, scene.ny, scene.nz, np.ascontiguousarray(ddf), out)
    return out


def ref_step(scene: Scene, inv_tau, src, dst, z0=0, z1=0, nthreads=0) -> None:
    ref().ref_step_f32(scene.nx, scene.ny, scene.nz, scene.flag, scene.rho, scene.vx, scene.vy, scene.vz,
                       inv_tau, src, dst, z0, z1, nthreads)


def ref_run(scene: Scene, inv_tau, nsteps, nthreads=0):
    a = rest_state(scene.n, np.float32)
    b = a.copy()
    for _ in range(nsteps):
        ref_step(scene, inv_tau, a, b, nthreads=nthreads)
        a, b = b, a
    return a


def ref_moments(scene: Scene, ddf, nthreads=0):
    out = [scene.rho.copy(), scene.vx.copy(), scene.vy.copy(), scene.vz.copy()]
    ref().ref_moments_f32(scene.nx, scene.ny, scene.nz, scene.flag, np.ascontiguousarray(ddf), *out, nthreads)
    return tuple(out)


# 16-bit storage kinds of orc_step_s16 (match culbm_b200's storage names)
S16_KIND = {"fp16": 0, "bf16": 1, "fp16sr": 2, "bf16sr": 3}


def run_s16(scene: Scene, storage: str, inv_tau, nsteps, state=None):
    """nsteps pull steps with 16-bit storage from rest (or from an FP32 state
    narrowed with nearest-even / stochastic rounding keyed on step 0); returns
    the newest state widened to FP32."""
    kind = S16_KIND[storage]
    L = lib()
    f32 = rest_state(scene.n) if state is None else np.ascontiguousarray(state, np.float32)
    a = np.empty(27 * scene.n, np.uint16)
    L.orc_encode_s16(kind, scene.n, f32, a, 0)
    b = a.copy()
    for t in range(nsteps):
        L.orc_step_s16(kind, scene.nx, scene.ny, scene.nz, scene.flag, scene.rho, scene.vx, scene.vy, scene.vz,
                       inv_tau, a, b, t)
        a, b = b, a
    out = np.empty(27 * scene.n, np.float32)
    L.orc_decode_s16(kind, 27 * scene.n, a, out)
    return out


def round16_sr(kind: str, values, rbits):
    """Stochastic rounding of FP32 values to IEEE half ("f16") or bfloat16
    ("bf16") with one random integer each (the restatement of sm_100a's
    cvt.rs rule); returns the uint16 patterns."""
    v = np.ascontiguousarray(values, dtype=np.float32)
    r = np.ascontiguousarray(rbits, dtype=np.uint32)
    out = np.empty(v.size, np.uint16)
    lib().orc_round16_sr_n({"f16": 0, "bf16": 1}[kind], v.size, v, r, out)
    return out
