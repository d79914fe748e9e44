"""Tile and innerLoop choice for the L2-blocked policies, and the memory
constants its speed-up model needs (``culbm_select_tile``,
``culbm_blocking_speedup`` and ``culbm_measure_memory`` in include/culbm.h).

The model is the reference's (analysis/selector.py): the speed-up over plain
streaming of a tile advanced innerLoop steps per round in L2, from the tile's
valid fraction, the sector alignment of its valid rows and the ratio lambda of
DRAM to L2 bandwidth (gamma: cost of a partial store sector).  A predicted
speed-up below 1 means plain streaming (optPolicy 0) is faster.

    python -m culbm_b200.selector --domain 288 272 280 [--storage fp32] [--measure]
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

from . import _capi
from ._capi import check, lib


def measure(dev: int = 0) -> dict:
    """lambda, gamma and the bandwidths behind them, measured on device `dev`."""
    m = _capi.MemoryConstants()
    check(lib().culbm_measure_memory(dev, C.byref(m)))
    return {"dram_gbs": m.dram_gbs, "l2_gbs": m.l2_gbs, "lambda": m.lambda_, "full_store_ms": m.full_store_ms,
            "partial_store_ms": m.partial_store_ms, "gamma": m.gamma, "l2_bytes": m.l2_bytes}


def select(domain: Sequence[int], storage: str = "fp32", lam: float = 0.0, gamma: float = 0.0, l2_bytes: int = 0,
           persist_bytes: int = 0) -> dict:
    """Tile (blockDim*gridDim) and innerLoop of the largest model speed-up."""
    d = (C.c_uint32 * 3)(*[int(v) for v in domain])
    t = _capi.TileChoice()
    check(lib().culbm_select_tile(d, _capi.STORAGE[storage], float(lam), float(gamma), int(l2_bytes),
                                  int(persist_bytes), C.byref(t)))
    return {"tile": list(t.tile), "inner_loop": t.inner_loop, "speedup": t.predicted_speedup,
            "speedup_no_alignment": t.predicted_speedup_no_alignment, "speedup_b200": t.predicted_speedup_b200}


def speedup(tile: Sequence[int], inner_loop: int, storage: str = "fp32", lam: float = 0.0, gamma: float = 0.0,
            l2_bytes: int = 0):
    """(S, S0) of one tile and innerLoop."""
    tb = (C.c_uint32 * 3)(*[int(v) for v in tile])
    s, s0 = C.c_double(), C.c_double()
    check(lib().culbm_blocking_speedup(tb, int(inner_loop), _capi.STORAGE[storage], float(lam), float(gamma),
                                       int(l2_bytes), C.byref(s), C.byref(s0)))
    return s.value, s0.value


def blocking_axis(domain: int, tile: int, inner_loop: int) -> list:
    """Valid-region bounds of the tiles along one axis, [0, ..., domain]
    (tile k stores cells [b[k], b[k+1])), as the blocking engine computes
    them (``culbm_blocking_axis``: blocking_core's calcBlkNum and
    calcValidPrev).  Raises CulbmError for a geometry culbm_create rejects."""
    num = C.c_uint32()
    check(lib().culbm_blocking_axis(int(domain), int(tile), int(inner_loop), C.byref(num), None, 0))
    starts = (C.c_int32 * (num.value + 1))()
    check(lib().culbm_blocking_axis(int(domain), int(tile), int(inner_loop), C.byref(num), starts, num.value + 1))
    return list(starts)


def main(argv: Optional[Sequence[str]] = None) -> int:
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m culbm_b200.selector", description=__doc__.split("\n\n")[0])
    ap.add_argument("--domain", type=int, nargs=3, required=True)
    ap.add_argument("--storage", default="fp32", choices=sorted(_capi.STORAGE))
    ap.add_argument("--measure", action="store_true", help="measure lambda and gamma on this GPU first")
    ap.add_argument("--lambda", dest="lam", type=float, default=0.0)
    ap.add_argument("--gamma", type=float, default=0.0)
    ap.add_argument("--dev", type=int, default=0)
    args = ap.parse_args(argv)
    out = {}
    lam, gam = args.lam, args.gamma
    if args.measure:
        out["measured"] = measure(args.dev)
        lam, gam = out["measured"]["lambda"], out["measured"]["gamma"]
    out["choice"] = select(args.domain, args.storage, lam, gam)
    t = out["choice"]["tile"]
    out["tiles_per_axis"] = [len(blocking_axis(d, b, out["choice"]["inner_loop"])) - 1
                             for d, b in zip(args.domain, t)]
    out["cli"] = (f"--blockDim [{t[0]},{t[1]},{t[2]}] --gridDim [1,1,1] --innerLoop {out['choice']['inner_loop']} "
                  f"--streamPolicy 1 --optPolicy 3")
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
