"""C ABI checks that need no GPU: the library loads, exports every declared
symbol, fills the reference's defaults and rejects bad configurations with
the reference's messages before touching the device.  CUDA failures are
injected on the host (culbm_debug_inject_cuda_error); no device fault."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            names.update(re.findall(r"\b(culbm_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(culbm):
    from culbm_b200 import _capi
    lib = _capi.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for name in syms:
        assert hasattr(lib, name), name
    assert lib.culbm_abi_version() == 1


def test_config_defaults_are_the_reference_cli_defaults(culbm):
    from culbm_b200 import _capi
    cfg = _capi.default_config()
    assert list(cfg.block_dim) == [32, 16, 2]
    assert list(cfg.grid_dim) == [2, 3, 19]
    assert list(cfg.domain_dim) == [256, 256, 256]
    assert cfg.inner_loop == 5 and cfg.inv_tau == 0.5
    assert cfg.stream_policy == 0 and cfg.opt_policy == 0 and cfg.vel_set == 0 and cfg.dev_id == 0
    assert cfg.use_ring_ddf_buf == 0 and cfg.storage == 0


def _create(cfg):
    from culbm_b200 import _capi
    h = C.c_void_p()
    st = _capi.lib().culbm_create(C.byref(cfg), C.byref(h))
    msg = _capi.lib().culbm_last_error().decode()
    if st == 0:
        _capi.lib().culbm_destroy(h)
    return st, msg


@pytest.mark.parametrize("mutate,needle", [
    (lambda c: setattr(c, "use_ring_ddf_buf", 1), "--useRingDDFBuf is unimplemented"),
    (lambda c: c.domain_dim.__setitem__(0, 100), "Dimension of domain doesn't match computation grid!"),
    (lambda c: setattr(c, "vel_set", 3), "Unsupport Velocity Set"),
    (lambda c: setattr(c, "stream_policy", 2), "streamPolicy"),
    (lambda c: setattr(c, "inv_tau", 2.5), "invTau"),
    (lambda c: c.domain_dim.__setitem__(2, 0), "domainDim"),
    # in-place launches use one row of cells per block, so ny is the grid's y extent
    (lambda c: (setattr(c, "stream_policy", 1), c.domain_dim.__setitem__(0, 32),
                c.domain_dim.__setitem__(1, 70000), c.domain_dim.__setitem__(2, 4)), "grid y above 65535"),
])
def test_invalid_configs_rejected_before_device(culbm, mutate, needle):
    from culbm_b200 import _capi
    cfg = _capi.default_config()
    cfg.grid_dim[0], cfg.grid_dim[1], cfg.grid_dim[2] = 8, 16, 128   # 32*8=256, 16*16=256, 2*128=256
    mutate(cfg)
    st, msg = _create(cfg)
    assert st == 1, (st, msg)
    assert needle in msg


def test_injected_cuda_error_is_reported(culbm):
    from culbm_b200 import _capi
    cfg = _capi.default_config()
    cfg.domain_dim[0] = cfg.domain_dim[1] = cfg.domain_dim[2] = 8
    cfg.block_dim[0] = cfg.block_dim[1] = cfg.block_dim[2] = 8
    cfg.grid_dim[0] = cfg.grid_dim[1] = cfg.grid_dim[2] = 1
    _capi.lib().culbm_debug_inject_cuda_error(0, 2)   # cudaErrorMemoryAllocation on the first call
    try:
        st, msg = _create(cfg)
    finally:
        _capi.lib().culbm_debug_inject_cuda_error(0, 0)
    assert st == 3, (st, msg)          # CULBM_ERR_OUT_OF_MEMORY
    assert "cudaErrorMemoryAllocation" in msg


def test_status_strings(culbm):
    from culbm_b200 import _capi
    lib = _capi.lib()
    for code, name in _capi.STATUS_NAMES.items():
        assert lib.culbm_status_string(code).decode() == name


def test_null_arguments(culbm):
    from culbm_b200 import _capi
    lib = _capi.lib()
    assert lib.culbm_create(None, None) == 1
    assert lib.culbm_step(None, 1) == 1
    assert lib.culbm_destroy(None) == 0


@pytest.mark.parametrize("dims,tile,inner,needle", [
    ((64, 64, 64), (4, 64, 64), 3, "don't match"),      # B + 2 - 2I <= 0 with more than two tiles
    ((64, 64, 64), (8, 8, 8), 9, "don't match"),        # B + 1 <= I with B < dom (reference check)
    ((64, 64, 64), (16, 16, 16), 0, "innerLoop"),
])
def test_invalid_blocking_rejected_before_device(culbm, dims, tile, inner, needle):
    from culbm_b200 import _capi
    cfg = _capi.default_config()
    for k in range(3):
        cfg.domain_dim[k] = dims[k]
        cfg.block_dim[k] = tile[k]
        cfg.grid_dim[k] = 1
    cfg.stream_policy, cfg.opt_policy, cfg.inner_loop = 1, 3, inner
    st, msg = _create(cfg)
    assert st == 1, (st, msg)
    assert needle in msg


@pytest.mark.parametrize("mutate,needle", [
    (lambda c: setattr(c, "checkpoint_inner", 50), "checkpoint_inner"),
    (lambda c: setattr(c, "checkpoint_inner", -1), "checkpoint_inner"),
    (lambda c: (setattr(c, "checkpoint_every", 0), setattr(c, "checkpoint_inner", 4)), "checkpoint_inner"),
    (lambda c: c.window.__setitem__(1, 10), "objective window"),
    (lambda c: setattr(c, "inv_tau", 2.0), "invTau"),
    (lambda c: setattr(c, "precision", 1), "FP64 precision"),
    (lambda c: setattr(c, "precision", 2), "precision"),
    (lambda c: c.domain_dim.__setitem__(2, 0), "domain_dim"),
])
def test_adjoint_config_rejected_before_the_device(culbm, mutate, needle):
    from culbm_b200 import _capi
    cfg = _capi.AdjConfig()
    assert _capi.lib().culbm_adj_config_init(C.byref(cfg)) == 0
    assert cfg.checkpoint_every == 50 and cfg.checkpoint_inner == 0 and list(cfg.window) == [300, 500]
    mutate(cfg)
    h = C.c_void_p()
    st = _capi.lib().culbm_adj_create(C.byref(cfg), C.byref(h))
    assert st != 0 and not h.value
    assert needle in _capi.lib().culbm_last_error().decode()


def test_blocking_axis_matches_the_reference_geometry(culbm, orc):
    """culbm_blocking_axis (the blocking engine's own geometry) against the
    reference's blocking_core compiled for the host (when oracle/_ref is
    built) and the oracle's restatement: same accept/reject decision as
    culbm_create, same tile count, same valid-region bounds."""
    from culbm_b200 import _capi
    lib = _capi.lib()
    L = orc.lib()
    R = orc.ref() if orc.ref_available() else None
    cap = 4096
    starts = (C.c_int32 * cap)()
    num = C.c_uint32()
    checked = 0
    for dom in (1, 2, 7, 13, 64, 96, 280, 288, 384, 768, 1000):
        for blk in (1, 2, 3, 4, 7, 16, 36, 64, 76, 96, 128, 160, 288):
            for it in (1, 2, 3, 4, 5, 9):
                st = lib.culbm_blocking_axis(dom, blk, it, C.byref(num), starts, cap)
                ok = bool(L.orc_valid_blk_axis(dom, blk, it))
                if R is not None:
                    assert ok == bool(R.ref_valid_blk_axis(dom, blk, it)), (dom, blk, it)
                # Admitted by validBlkAxisConfig but rejected here: calcBlkNum
                # would divide by blk + 2 - 2*it <= 0.
                degenerate = dom > blk and dom > 2 * (blk + 1 - it) and blk + 2 - 2 * it <= 0
                if not ok or degenerate:
                    assert st == 1, (dom, blk, it)
                    assert "don't match" in lib.culbm_last_error().decode()
                    continue
                assert st == 0, (dom, blk, it, lib.culbm_last_error().decode())
                n = num.value
                assert n == L.orc_blk_num(dom, blk, it)
                got = list(starts[:n + 1])
                assert got == [L.orc_valid_prev(k, blk, n, it, dom) for k in range(n + 1)]
                if R is not None:
                    assert n == R.ref_blk_num(dom, blk, it)
                    assert got == [R.ref_valid_prev(k, blk, n, it, dom) for k in range(n + 1)]
                assert got[0] == 0 and got[-1] == dom and all(b > a for a, b in zip(got, got[1:]))
                checked += 1
    assert checked > 300


def test_blocking_axis_argument_errors(culbm):
    from culbm_b200 import _capi
    lib = _capi.lib()
    num = C.c_uint32()
    small = (C.c_int32 * 2)()
    assert lib.culbm_blocking_axis(288, 64, 5, None, None, 0) == 1
    assert lib.culbm_blocking_axis(288, 64, 0, C.byref(num), None, 0) == 1
    assert "innerLoop" in lib.culbm_last_error().decode()
    assert lib.culbm_blocking_axis(0, 64, 5, C.byref(num), None, 0) == 1
    assert lib.culbm_blocking_axis(288, 70000, 5, C.byref(num), None, 0) == 1
    assert "65535" in lib.culbm_last_error().decode()
    assert lib.culbm_blocking_axis(288, 64, 5, C.byref(num), None, 0) == 0 and num.value == 5
    assert lib.culbm_blocking_axis(288, 64, 5, C.byref(num), small, 2) == 1
    assert "6 entries" in lib.culbm_last_error().decode()
