"""ctypes bindings of the C ABI in ``include/culbm.h`` (``culbm_b200/libculbm.so``).

The library is loaded from this package directory only.  If it is missing
the import of the binding fails loudly: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libculbm.so")

OK = 0
STATUS_NAMES = {
    0: "CULBM_OK",
    1: "CULBM_ERR_INVALID_ARGUMENT",
    2: "CULBM_ERR_CUDA",
    3: "CULBM_ERR_OUT_OF_MEMORY",
    4: "CULBM_ERR_IO",
    5: "CULBM_ERR_STATE",
    6: "CULBM_ERR_UNSUPPORTED",
    7: "CULBM_ERR_DEVICE_TIMEOUT",
}

STREAM_PULL, STREAM_INPLACE = 0, 1
OPT_NONE, OPT_STATIC_L2, OPT_L1L2, OPT_DYNAMIC_L2 = 0, 1, 2, 3
STORAGE = {"fp32": 0, "fp16": 1, "bf16": 2, "fp64": 3, "fp16sr": 4, "bf16sr": 5}
FIELD = {"rho": 0, "vx": 1, "vy": 2, "vz": 3}

# Every symbol include/culbm.h declares.
EXPORTED = (
    "culbm_config_init", "culbm_create", "culbm_destroy", "culbm_load_state", "culbm_load_state_folder",
    "culbm_step", "culbm_step_timed", "culbm_synchronize", "culbm_moments", "culbm_get_field", "culbm_run_host", "culbm_dump",
    "culbm_get_step", "culbm_get_pulled_ddf", "culbm_set_ddf", "culbm_mass_momentum", "culbm_mass_momentum_noalloc", "culbm_measure_memory",
    "culbm_select_tile", "culbm_blocking_speedup", "culbm_blocking_axis", "culbm_get_info",
    "culbm_last_error", "culbm_status_string", "culbm_abi_version", "culbm_debug_inject_cuda_error",
    "culbm_debug_row_wait_extra_bytes",
    "culbm_adj_config_init", "culbm_adj_create", "culbm_adj_destroy", "culbm_adj_set_state",
    "culbm_adj_set_inv_tau", "culbm_adj_forward", "culbm_adj_gradient", "culbm_adj_get_info",
)


class Config(C.Structure):
    _fields_ = [
        ("dev_id", C.c_int32),
        ("block_dim", C.c_uint32 * 3),
        ("grid_dim", C.c_uint32 * 3),
        ("domain_dim", C.c_uint32 * 3),
        ("inner_loop", C.c_int32),
        ("stream_policy", C.c_int32),
        ("opt_policy", C.c_int32),
        ("vel_set", C.c_int32),
        ("inv_tau", C.c_float),
        ("use_ring_ddf_buf", C.c_int32),
        ("storage", C.c_int32),
        ("persist_l2", C.c_int32),
        ("cache_hints", C.c_int32),
        ("use_graphs", C.c_int32),
        ("kernel_variant", C.c_int32),
        ("run_slabs", C.c_int32),
        ("reserved", C.c_uint32 * 6),
    ]


class Info(C.Structure):
    _fields_ = [
        ("cells", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("blocking_num", C.c_uint32 * 3),
        ("blocking_dim", C.c_uint32 * 3),
        ("storage", C.c_int32),
        ("stream_policy", C.c_int32),
        ("opt_policy", C.c_int32),
        ("inner_loop", C.c_int32),
        ("persisting_l2_bytes", C.c_uint64),
        ("kernel_launches_per_step_x1000", C.c_uint32),
        ("reserved", C.c_uint32 * 7),
    ]


class AdjConfig(C.Structure):
    _fields_ = [
        ("dev_id", C.c_int32),
        ("domain_dim", C.c_uint32 * 3),
        ("inv_tau", C.c_float),
        ("window", C.c_int32 * 2),
        ("plane_x", C.c_int32 * 2),
        ("checkpoint_every", C.c_int32),
        ("precision", C.c_int32),
        ("storage", C.c_int32),
        ("hbm_budget_bytes", C.c_uint64),
        ("checkpoint_inner", C.c_int32),
        ("checkpoint_storage", C.c_int32),
        ("reserved", C.c_uint32 * 6),
    ]


class AdjInfo(C.Structure):
    _fields_ = [
        ("checkpoint_every", C.c_int32),
        ("checkpoints", C.c_int32),
        ("device_bytes", C.c_uint64),
        ("forward_ms", C.c_float),
        ("recompute_ms", C.c_float),
        ("adjoint_ms", C.c_float),
        ("steps", C.c_uint64),
        ("checkpoint_inner", C.c_int32),
        ("inner_checkpoints", C.c_int32),
        ("reserved", C.c_uint32 * 6),
    ]


class MemoryConstants(C.Structure):
    _fields_ = [
        ("dram_gbs", C.c_double),
        ("l2_gbs", C.c_double),
        ("lambda_", C.c_double),
        ("full_store_ms", C.c_double),
        ("partial_store_ms", C.c_double),
        ("gamma", C.c_double),
        ("l2_bytes", C.c_uint64),
        ("reserved", C.c_uint32 * 8),
    ]


class TileChoice(C.Structure):
    _fields_ = [
        ("tile", C.c_uint32 * 3),
        ("inner_loop", C.c_int32),
        ("predicted_speedup", C.c_double),
        ("predicted_speedup_no_alignment", C.c_double),
        ("predicted_speedup_b200", C.c_double),
        ("reserved", C.c_uint32 * 6),
    ]


class CulbmError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


_lib = None


def lib():
    """Load libculbm.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m culbm_b200.build` "
                           "(the CUDA library is required; there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.culbm_config_init.argtypes = [C.POINTER(Config)]
    L.culbm_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.culbm_destroy.argtypes = [vp]
    L.culbm_load_state.argtypes = [vp, vp, vp, vp, vp, vp]
    L.culbm_load_state_folder.argtypes = [vp, C.c_char_p, C.POINTER(C.c_uint32)]
    L.culbm_step.argtypes = [vp, C.c_uint32]
    L.culbm_step_timed.argtypes = [vp, C.c_uint32, C.POINTER(C.c_float)]
    L.culbm_synchronize.argtypes = [vp]
    L.culbm_moments.argtypes = [vp]
    L.culbm_get_field.argtypes = [vp, C.c_int, vp]
    L.culbm_run_host.argtypes = [vp, vp, vp, vp, vp, vp, C.c_uint32, vp, vp, vp, vp]
    L.culbm_dump.argtypes = [vp, C.c_char_p, C.c_uint32]
    L.culbm_get_step.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.culbm_get_pulled_ddf.argtypes = [vp, vp, C.c_int32]
    L.culbm_set_ddf.argtypes = [vp, vp, C.c_int32]
    L.culbm_mass_momentum.argtypes = [vp, C.POINTER(C.c_double)]
    L.culbm_mass_momentum_noalloc.argtypes = [vp, C.c_uint64, vp, C.POINTER(C.c_double)]
    L.culbm_measure_memory.argtypes = [C.c_int32, C.POINTER(MemoryConstants)]
    L.culbm_select_tile.argtypes = [C.POINTER(C.c_uint32), C.c_int32, C.c_double, C.c_double, C.c_uint64,
                                    C.c_uint64, C.POINTER(TileChoice)]
    L.culbm_blocking_speedup.argtypes = [C.POINTER(C.c_uint32), C.c_int32, C.c_int32, C.c_double, C.c_double,
                                         C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.culbm_blocking_axis.argtypes = [C.c_uint32, C.c_uint32, C.c_int32, C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_int32), C.c_uint32]
    L.culbm_get_info.argtypes = [vp, C.POINTER(Info)]
    L.culbm_last_error.restype = C.c_char_p
    L.culbm_status_string.restype = C.c_char_p
    L.culbm_status_string.argtypes = [C.c_int]
    L.culbm_abi_version.restype = C.c_int32
    L.culbm_debug_inject_cuda_error.argtypes = [C.c_int32, C.c_int32]
    L.culbm_debug_inject_cuda_error.restype = None
    L.culbm_debug_row_wait_extra_bytes.argtypes = [C.c_int32]
    L.culbm_debug_row_wait_extra_bytes.restype = None
    L.culbm_adj_config_init.argtypes = [C.POINTER(AdjConfig)]
    L.culbm_adj_create.argtypes = [C.POINTER(AdjConfig), C.POINTER(vp)]
    L.culbm_adj_destroy.argtypes = [vp]
    L.culbm_adj_set_state.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.culbm_adj_set_inv_tau.argtypes = [vp, C.c_double]
    L.culbm_adj_forward.argtypes = [vp, C.POINTER(C.c_double)]
    L.culbm_adj_gradient.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), vp, vp]
    L.culbm_adj_get_info.argtypes = [vp, C.POINTER(AdjInfo)]
    _lib = L
    return L


def check(status: int) -> None:
    if status != OK:
        raise CulbmError(status, lib().culbm_last_error().decode(errors="replace"))


def default_config() -> Config:
    cfg = Config()
    check(lib().culbm_config_init(C.byref(cfg)))
    return cfg
