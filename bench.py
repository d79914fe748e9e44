"""D3Q27 BGK throughput on one B200 (MLUPS), with its roofline, an end-to-end
number through the C ABI and the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 288x272x280 channel with 40 seeded spheres (radii 4-12),
invTau 0.5, inlet ux 0.05 (synthetic, seeded; the reference ships no dataset).
A step is one lattice update of every cell.  The headline `value` is FP32
in-place streaming (streamPolicy 1, optPolicy 0) timed on the device over K
steps with inputs resident in HBM; the population buffers (2.37 GB) are far
larger than L2, so no flush is needed between steps.  The line also carries
FP32 pull, blocked and FP16/BF16-storage speeds, and the FP16/BF16/FP32 error
against an FP64 run of the scaled 128x128x64 copy of the 512x512x256 workload.

--impl reference times the reference's own lbm_core routines compiled for
the host (oracle/_ref, OpenMP over all host cores) on the same workload.
With torchrun (N > 1) every rank runs an independent replica (the hot path
has no data-path exchange); value = all ranks' updates / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "D3Q27 MLUPS, FP32 vs FP16-store at stated FP64 err; adjoint/forward cost"
BYTES_PER_LUP = {"fp32": 216, "fp16": 108, "bf16": 108, "fp16sr": 108, "bf16sr": 108, "fp64": 432}
WORKLOAD = "288x272x280 channel, 40 seeded spheres r in [4,12], invTau 0.5, ux_in 0.05"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle-reason sampling (NVML, every 10 ms) for the whole
    run, with per-window summaries; falls back to nvidia-smi when NVML is
    unavailable."""

    # NVML clocks-event-reason bits (nvml.h)
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index=0):
        self.index = index
        self.samples = []          # (perf_counter time, SM MHz, reason bits)
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def _run_nvml(self, nv):
        h = nv.nvmlDeviceGetHandleByIndex(self.index)
        self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            try:
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except AttributeError:
                r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.samples.append((time.perf_counter(), float(sm), int(r)))
            self._stop.wait(0.01)

    def _run_smi(self):
        q = "clocks.sm,clocks.max.sm,clocks_event_reasons.active"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=10).stdout.strip().split(",")
                self.max_mhz = float(out[1])
                self.samples.append((time.perf_counter(), float(out[0]), int(out[2].strip(), 16)))
            except Exception:
                pass
            self._stop.wait(0.05)

    def _run(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            try:
                self._run_nvml(nv)
            finally:
                nv.nvmlShutdown()
        except Exception:
            self._run_smi()

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        time.sleep(0.05)
        return self

    def stop(self):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=15)

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def summary(self, t0=None, t1=None):
        """Median SM clock, max clock and the throttle reasons seen between
        perf_counter times t0 and t1 (the whole run when both are None); a
        window shorter than the sampling period takes the nearest sample."""
        sel = [s for s in self.samples if (t0 is None or s[0] >= t0) and (t1 is None or s[0] <= t1)]
        if not sel and self.samples and t0 is not None:
            mid = 0.5 * (t0 + (t1 if t1 is not None else t0))
            sel = [min(self.samples, key=lambda s: abs(s[0] - mid))]
        if not sel:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"], "samples": 0}
        sm = [s[1] for s in sel]
        reasons = sorted({name for _, _, r in sel for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sel)}


def dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return ws, rank


def dist_init(ws):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as tdist
    tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return tdist


def max_over_ranks(tdist, v):
    if tdist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def barrier(tdist):
    if tdist is not None:
        tdist.barrier()


def aggregate_mlups(ws, cells, steps, ms_max):
    """Whole-job MLUPS of ws independent replicas of `cells` cells run for
    `steps` steps, timed by the slowest rank (ms_max, device time)."""
    return ws * cells * steps / (ms_max * 1e-3) / 1e6


def pinned(arr):
    """A page-locked host copy of arr (torch pinned memory, viewed by numpy)."""
    import torch
    t = torch.empty(arr.size, dtype={np.uint32: torch.int32, np.float32: torch.float32}[arr.dtype.type],
                    pin_memory=True)
    out = t.numpy().view(arr.dtype)
    out[:] = arr.reshape(-1)
    return out, t


def traffic_from_profiles(kernel_key):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    entry = d.get(kernel_key)
    return None if entry is None else entry["bytes"]


# ------------------------------------------------------------------- ours ---

def measure(culbm, scene, sp, op, storage, steps, warmup, tile=None, inner=5, ring=False, clocks=None, split=None):
    """MLUPS of one policy.  `tile` is the tile extent (blockDim = tile,
    gridDim = 1); `split` = (blockDim, gridDim) gives the tile as the
    reference's launch split instead (for optPolicy 2 the CTA and cluster shape)."""
    arrs = scene.arrays()
    kw = {"dev_id": int(os.environ.get("LOCAL_RANK", "0"))}
    if op and split is not None:
        kw.update(block_dim=split[0], grid_dim=split[1], inner_loop=inner, use_ring=ring)
    elif op:
        kw.update(tile=tile, inner_loop=inner, use_ring=ring)
    with culbm.Simulation(scene.shape, stream_policy=sp, opt_policy=op, storage=storage, inv_tau=0.5, **kw) as sim:
        sim.load_state(*arrs)
        sim.step(warmup)
        sim.synchronize()
        t0 = time.perf_counter()
        ms = sim.step_timed(steps)
        t1 = time.perf_counter()
        info = sim.info()
    if clocks is not None:
        info["clocks"] = clocks.summary(t0, t1)
    return scene.n * steps / (ms * 1e-3) / 1e6, ms / steps, info


def fp64_errors(culbm, steps=1000):
    """Relative rho/u error after `steps` steps against FP64 storage+arithmetic, on the
    scaled 128x128x64 copy of the 512x512x256 workload."""
    from culbm_b200 import scenes
    sc = scenes.spheres_512(scale=0.25)
    arrs = sc.arrays()
    fluid = (arrs[0] & scenes.COLLIDE) != 0

    def fields(storage):
        with culbm.Simulation(sc.shape, stream_policy=1, storage=storage, inv_tau=0.5) as sim:
            sim.load_state(*arrs)
            sim.step(steps)
            sim.moments()
            return [f.astype(np.float64) for f in sim.fields()]

    ref = fields("fp64")
    umag = np.sqrt(ref[1] ** 2 + ref[2] ** 2 + ref[3] ** 2)
    out = {}
    for st in ("fp32", "fp16", "fp16sr", "bf16", "bf16sr"):
        got = fields(st)
        du = np.sqrt(sum((got[k] - ref[k]) ** 2 for k in (1, 2, 3)))
        out[st] = {
            "rel_u_l2": float(np.linalg.norm(du[fluid]) / np.linalg.norm(umag[fluid])),
            "rel_u_max": float(np.max(du[fluid]) / np.max(umag[fluid])),
            "rel_rho_max": float(np.max(np.abs(got[0] - ref[0])[fluid] / ref[0][fluid])),
        }
    return {"workload": f"{sc.shape[0]}x{sc.shape[1]}x{sc.shape[2]} spheres (512x512x256 generator at 1/4), "
                        f"{steps} steps, vs FP64 storage+arithmetic", "errors": out}


def selector_summary(sel):
    """culbm_select_tile's pick: the model's speed-up over plain streaming
    (the reference's model, with the 16-bit compute floor), the same tile's
    speed-up with B200's measured step costs, and whether blocking is
    expected to pay (the latter above 1).  --blockDim auto with a blocked
    optPolicy prints both."""
    return {"tile": list(sel["tile"]), "inner_loop": sel["inner_loop"],
            "predicted_speedup": round(sel["speedup"], 4),
            "predicted_speedup_b200": round(sel["speedup_b200"], 4),
            "blocking_pays": bool(sel["speedup_b200"] > 1.0)}


def mixed_precision_512(culbm, steps):
    """The 512x512x256 channel with 120 spheres (radii 6-18): in-place
    streaming with FP32, FP16 and BF16 storage, plain and L2-blocked."""
    from culbm_b200 import scenes
    sc = scenes.spheres_512()
    peak, _ = peaks()
    out = {"workload": "512x512x256 channel, 120 seeded spheres r in [6,18], invTau 0.5, ux_in 0.05",
           "cells": sc.n, "steps": steps, "runs": {}}
    from culbm_b200 import selector
    s32, s16 = selector.select(sc.shape, "fp32"), selector.select(sc.shape, "fp16sr")
    out["selector"] = {k: selector_summary(v) for k, v in (("fp32", s32), ("fp16sr", s16))}
    for name, (op, st, tile, inner) in {
        "inplace_fp32": (0, "fp32", None, 5),
        "inplace_fp16": (0, "fp16", None, 5),
        "inplace_fp16sr": (0, "fp16sr", None, 5),
        "inplace_bf16": (0, "bf16", None, 5),
        "inplace_bf16sr": (0, "bf16sr", None, 5),
        "blocked_inplace_fp32": (3, "fp32", tuple(s32["tile"]), s32["inner_loop"]),
        "blocked_inplace_fp16sr": (3, "fp16sr", tuple(s16["tile"]), s16["inner_loop"]),
    }.items():
        try:
            mlups, mps, _ = measure(culbm, sc, 1, op, st, steps, 3, tile=tile, inner=inner)
            out["runs"][name] = {"mlups": round(mlups, 1), "ms_per_step": round(mps, 4),
                                 "hbm_frac_of_measured": round(mlups * 1e6 * BYTES_PER_LUP[st] / 1e9 / peak, 4),
                                 "policy": "streamPolicy 1, optPolicy %d" % op +
                                           (f", tile {tile} (culbm_select_tile), innerLoop {inner}" if op else "")}
        except Exception as e:   # report, do not hide
            out["runs"][name] = {"error": str(e)}
    return out


def adjoint_runs():
    """Gradient of the pressure drop on the soft-obstacle channels: the
    128x64x64 case (FP32, window 300-500, checkpoints every 50) and the
    288x272x280 case (48 bumps, 2000 steps, plan chosen for a 120 GB budget)
    with FP32 states, FP16-SR states, and an FP32 forward pass with FP16-SR
    checkpoints, the last two with their gradient error against FP32 states."""
    from culbm_b200 import scenes
    from culbm_b200.adjoint import AdjointProblem

    def run(dims, bumps, window, storage, **kw):
        sc, soft = scenes.adjoint_channel(*dims, u_peak=0.04, bumps=bumps, seed=7)
        with AdjointProblem(dims, window=window, storage=storage, **kw) as p:
            p.set_state(*sc.arrays(), soft.reshape(-1))
            J, gt, gs, gm = p.gradient()
            inf = p.info()
        n, T = sc.n, window[1]
        total = inf["forward_ms"] + inf["recompute_ms"] + inf["adjoint_ms"]
        summary = {"storage": storage, "checkpoint_storage": kw.get("checkpoint_storage") or storage, "J": J,
                   "dJ_dinv_tau": gt,
                   "checkpoint_every": inf["checkpoint_every"], "checkpoint_inner": inf["checkpoint_inner"],
                   "device_gb": round(inf["device_bytes"] / 1e9, 2),
                   "forward_ms": round(inf["forward_ms"], 2), "recompute_ms": round(inf["recompute_ms"], 2),
                   "adjoint_ms": round(inf["adjoint_ms"], 2),
                   "cost_ratio": round((inf["recompute_ms"] + inf["adjoint_ms"]) / inf["forward_ms"], 3),
                   "forward_mlups": round(n * T / (inf["forward_ms"] * 1e-3) / 1e6, 1),
                   "adjoint_step_mlups": round(n * T / (inf["adjoint_ms"] * 1e-3) / 1e6, 1),
                   "gradient_mlups": round(n * T / (total * 1e-3) / 1e6, 1)}
        return summary, (J, gt, gs, gm)

    out = {"cost_ratio_definition": "(recompute + adjoint sweep) / forward pass, device time"}
    out["channel_128x64x64"], _ = run((128, 64, 64), 16, (300, 500), "fp32", checkpoint_every=50)
    budget = 120e9
    big = {}
    for name, st, ck in (("fp16sr", "fp16sr", None), ("fp32", "fp32", None), ("fp32_ck_fp16sr", "fp32", "fp16sr")):
        big[name] = run((288, 272, 280), 48, (1500, 2000), st, checkpoint_every=0, hbm_budget_bytes=int(budget),
                        checkpoint_storage=ck)
    g32 = big["fp32"][1]

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))

    def versus(g):
        return {"J_rel": rel(g[0], g32[0]), "dJ_dinv_tau_rel": rel(g[1], g32[1]),
                "dJ_dsoft_rel_l2": rel(g[2], g32[2]), "dJ_dvx_in_rel_l2": rel(g[3][1], g32[3][1])}

    out["channel_288x272x280"] = {
        "hbm_budget_gb": budget / 1e9, "fp16sr": big["fp16sr"][0], "fp32": big["fp32"][0],
        "fp32_ck_fp16sr": big["fp32_ck_fp16sr"][0],
        "fp16sr_vs_fp32": versus(big["fp16sr"][1]), "fp32_ck_fp16sr_vs_fp32": versus(big["fp32_ck_fp16sr"][1])}
    return out


def e2e_run(culbm, scene, steps, sp=1, reps=3, tdist=None, ws=1, dev_id=0):
    """Through the public API with page-locked host buffers, host wall clock,
    best of `reps`; with several ranks each rank runs its own replica between
    barriers, the time is the slowest rank's and the MLUPS the whole job's.
    `overlapped`: one culbm_run_host call (the init state in, `steps` steps,
    the dump kernel and rho/vx/vy/vz out, with the slabs' copies overlapping
    the steps).  `sequential`: the same run as culbm_load_state + culbm_step +
    culbm_moments + 4x culbm_get_field, which copy before and after the
    steps."""
    import ctypes as C

    from culbm_b200 import _capi
    arrs = scene.arrays()
    host = [pinned(a) for a in arrs]
    outs = [pinned(np.zeros(scene.n, np.float32)) for _ in range(4)]
    out_arrays = tuple(o[0] for o in outs)
    best = {"overlapped": float("inf"), "sequential": float("inf")}
    same = True

    def timed(fn):
        barrier(tdist)
        t0 = time.perf_counter()
        fn()
        return max_over_ranks(tdist, time.perf_counter() - t0)

    with culbm.Simulation(scene.shape, stream_policy=sp, inv_tau=0.5, dev_id=dev_id) as sim:
        lib = _capi.lib()
        sim.run_host(5, *[h[0] for h in host], out=out_arrays)   # creates the run's streams

        def sequential():
            _capi.check(lib.culbm_load_state(sim._h, *[h[0].ctypes.data_as(C.c_void_p) for h in host]))
            sim.step(steps)
            sim.moments()
            for k in range(4):
                _capi.check(lib.culbm_get_field(sim._h, k, out_arrays[k].ctypes.data_as(C.c_void_p)))

        for _ in range(reps):
            best["overlapped"] = min(best["overlapped"],
                                     timed(lambda: sim.run_host(steps, *[h[0] for h in host], out=out_arrays)))
            first = [o.copy() for o in out_arrays]
            best["sequential"] = min(best["sequential"], timed(sequential))
            same = same and all(np.array_equal(a.view(np.uint32), b.view(np.uint32)) for a, b in zip(first, out_arrays))
    h2d = sum(h[0].nbytes for h in host)
    d2h = sum(o[0].nbytes for o in outs)
    mlups = {k: ws * scene.n * steps / v / 1e6 for k, v in best.items()}
    return mlups, h2d, d2h, same


# The reference's own parser of its speed lines (analysis/blocking_experiments.py:40).
SPEED_RE = __import__("re").compile(r"speed = ([0-9]+(?:\.[0-9]+)?) \(MLUPS\)")
REF_BIN_DIR = os.path.join(ROOT, "oracle", "_ref")

# Launch shapes of the reference's CUDA binary on the 288x272x280 workload:
# README.md:41-61 ((0,0) [32,16,2]x[9,17,140]; (1,3) [32,16,2]x[2,6,38],
# innerLoop 5), the best (0,0) block shape of a B200 retune, and the two build
# variants of src/simulator/single_dev_expt/CMakeLists.txt:28-41 on the (1,3)
# README shape.
REF_BINARY_LEGS = {
    "readme_00": ("single_dev_expt_main", (32, 16, 2), (9, 17, 140), 0, 0),
    "retuned_00": ("single_dev_expt_main", (32, 8, 1), (9, 34, 280), 0, 0),
    "readme_13": ("single_dev_expt_main", (32, 16, 2), (2, 6, 38), 1, 3),
    "variant_no_persist_no_hint_13": ("single_dev_expt_no_persist_no_hint_main", (32, 16, 2), (2, 6, 38), 1, 3),
    "variant_no_persist_hint_only_13": ("single_dev_expt_no_persist_hint_only_main", (32, 16, 2), (2, 6, 38), 1, 3),
}


def parse_speeds(stdout):
    """MLUPS of a reference-style run: the median of its `speed = X (MLUPS)`
    lines with the first skipped, as analysis/blocking_experiments.py:115 does."""
    speeds = [float(v) for v in SPEED_RE.findall(stdout)][1:]
    return statistics.median(speeds) if speeds else None


def reference_binary_legs(scene, peak, nstep=600, dstep=100, clocks=None):
    """The reference's single_dev_expt_main, compiled from its own sources for
    sm_100a (oracle/_ref, make -C oracle ref-gpu), on the same init-state
    folder, timed by its own CUDA events (simulator_expt_platform.cu:971-984)."""
    import shutil
    import tempfile

    from culbm_b200 import scenes
    if not os.path.exists(os.path.join(REF_BIN_DIR, "single_dev_expt_main")):
        return {"unavailable": "oracle/_ref/single_dev_expt_main not built (make -C oracle ref-gpu needs the "
                               "reference tree)"}
    tmp = tempfile.mkdtemp(prefix="culbm_refbin_")
    out = {"workload": WORKLOAD, "steps": nstep, "dstep": dstep,
           "how": "median of the binary's speed lines, first skipped (analysis/blocking_experiments.py:115)",
           "legs": {}}
    try:
        folder = os.path.join(tmp, "init")
        scenes.write_folder(scene, folder)
        nx, ny, nz = scene.shape
        vec = lambda v: "[" + ",".join(str(int(a)) for a in v) + "]"
        for name, (binary, block, grid, sp, op) in REF_BINARY_LEGS.items():
            path = os.path.join(REF_BIN_DIR, binary)
            if not os.path.exists(path):
                out["legs"][name] = {"error": f"{binary} not built"}
                continue
            cmd = [path, "--domainDim", vec((nx, ny, nz)), "--blockDim", vec(block), "--gridDim", vec(grid),
                   "--streamPolicy", str(sp), "--optPolicy", str(op), "--innerLoop", "5", "--invTau", "0.5",
                   "--nstep", str(nstep), "--dstep", str(dstep), "--initStateFolder", folder,
                   "--dumpFolder", os.path.join(tmp, "dump")]
            t0 = time.perf_counter()
            try:
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
            except subprocess.TimeoutExpired:
                out["legs"][name] = {"error": "timed out"}
                continue
            t1 = time.perf_counter()
            mlups = parse_speeds(r.stdout)
            leg = {"binary": binary, "blockDim": list(block), "gridDim": list(grid),
                   "policy": f"streamPolicy {sp}, optPolicy {op}" + (", innerLoop 5" if op else ""),
                   "exit_code": r.returncode}
            if mlups is None:
                leg["error"] = (r.stderr or r.stdout)[-300:]
            else:
                leg["mlups"] = round(mlups, 1)
                leg["hbm_frac_of_measured"] = round(mlups * 1e6 * BYTES_PER_LUP["fp32"] / 1e9 / peak, 4)
            if clocks is not None:
                leg["clocks"] = clocks.summary(t0, t1)
            out["legs"][name] = leg
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def workload_config(sc, ws):
    """The `config` of both arms' JSON lines (same keys and values)."""
    return {"workload": WORKLOAD, "cells": sc.n, "solid_fraction": round(sc.solid_fraction(), 4),
            "storage": "fp32", "l2": "no flush: 2.37 GB of populations per step, 19x the 126 MB L2",
            "parallelism": f"{ws} independent replica(s), one per GPU"}


def cpu_baseline(scene, budget_s=12.0):
    import oracle
    if not oracle.ref_available():
        return None
    f, r, ux, uy, uz = scene.arrays()
    nx, ny, nz = scene.shape
    o = oracle.Scene(nx, ny, nz, f, r, ux, uy, uz)
    a = oracle.rest_state(o.n)
    b = a.copy()
    threads = oracle.ref().ref_max_threads()
    oracle.ref_step(o, 0.5, a, b)     # warm-up (page faults, thread pool)
    steps, t0 = 0, time.perf_counter()
    while True:
        oracle.ref_step(o, 0.5, a, b)
        a, b = b, a
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= 200:
            break
    dt = time.perf_counter() - t0
    return {"value": round(o.n * steps / dt / 1e6, 2), "unit": "MLUPS", "cores": threads, "kind": "reference",
            "sample": f"{steps} full steps of the same 288x272x280 workload ({dt:.1f} s); the reference's "
                      f"lbm_core (device_function.hpp) compiled for the host, pull loop of StaticD3Q27PullKernel, "
                      f"OpenMP over z with {threads} threads"}


def run_ours(args):
    ws, rank = dist()
    tdist = dist_init(ws)
    import culbm_b200
    from culbm_b200 import _capi, scenes
    _capi.lib()
    sc = scenes.spheres_288()
    arrs = sc.arrays()
    peak, peak_kind = peaks()

    local = int(os.environ.get("LOCAL_RANK", "0"))
    clocks = ClockSampler(local).start()
    # headline: FP32 in-place, whole domain
    with culbm_b200.Simulation(sc.shape, stream_policy=1, opt_policy=0, storage="fp32", inv_tau=0.5,
                               dev_id=local) as sim:
        sim.load_state(*arrs)
        sim.step(args.warmup)
        sim.synchronize()
        barrier(tdist)
        t0 = time.perf_counter()
        ms = sim.step_timed(args.steps)
        t1 = time.perf_counter()
        info = sim.info()
    headline_clocks = clocks.summary(t0, t1)
    barrier(tdist)
    ms_max = max_over_ranks(tdist, ms)
    value = aggregate_mlups(ws, sc.n, args.steps, ms_max)
    ms_per_step = ms_max / args.steps
    launches = int(round(info["launches_per_step"] * args.steps))

    # End to end on every rank (its own replica), before the single-rank legs.
    e2e = None
    if not args.headline_only:
        e2e = e2e_run(culbm_b200, sc, args.steps, tdist=tdist, ws=ws, dev_id=local)
    if rank != 0:
        clocks.stop()
        if tdist is not None:
            tdist.destroy_process_group()
        return

    achieved = BYTES_PER_LUP["fp32"] * sc.n / (ms / args.steps * 1e-3) / 1e9
    if args.headline_only:
        clocks.stop()
        print(json.dumps({"metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": ws,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
                          "headline_only": True, "gpu_launches": launches, "clocks": headline_clocks}), flush=True)
        if tdist is not None:
            tdist.destroy_process_group()
        return
    extra = {}
    k2 = max(20, args.steps // 4)
    from culbm_b200 import selector
    sel = selector.select(sc.shape, "fp32")
    for name, (sp, op, st, tile, inner) in {
        "pull_fp32": (0, 0, "fp32", None, 5),
        "inplace_fp16": (1, 0, "fp16", None, 5),
        "inplace_fp16sr": (1, 0, "fp16sr", None, 5),
        "inplace_bf16": (1, 0, "bf16", None, 5),
        "pull_fp16": (0, 0, "fp16", None, 5),
        "pull_fp16sr": (0, 0, "fp16sr", None, 5),
        # the reference README's (1,3) launch shape: tile [32,16,2] x [2,6,38]
        "blocked_inplace_fp32_readme_tile": (1, 3, "fp32", (64, 96, 76), 5),
        "blocked_inplace_fp32_selected_tile": (1, 3, "fp32", tuple(sel["tile"]), sel["inner_loop"]),
        # (0,3): pull L2 tiles, the same two tiles
        "blocked_pull_fp32_readme_tile": (0, 3, "fp32", (64, 96, 76), 5),
        "blocked_pull_fp32_selected_tile": (0, 3, "fp32", tuple(sel["tile"]), sel["inner_loop"]),
        # (0,2): the cluster engine, tile 32x8x16 as 16 CTAs of 32x4x2 cells
        "blocked_pull_fp32_l1l2_cluster": (0, 2, "fp32", ((32, 4, 2), (1, 2, 8)), 2),
    }.items():
        try:
            split = tile if op == 2 else None
            mlups, mps, inf = measure(culbm_b200, sc, sp, op, st, k2, 3, tile=None if split else tile, inner=inner,
                                      clocks=clocks, split=split)
            if split:
                tile = tuple(b * g for b, g in zip(*split))
            extra[name] = {"mlups": round(mlups, 1), "ms_per_step": round(mps, 4),
                           "hbm_frac_of_measured": round(mlups * 1e6 * BYTES_PER_LUP[st] / 1e9 / peak, 4),
                           "policy": f"streamPolicy {sp}, optPolicy {op}" +
                                     (f", tile {tile}, innerLoop {inner}" if op else "") +
                                     (f", CTA {split[0]} x cluster {split[1]}" if split else ""),
                           "launches_per_step": inf.get("launches_per_step"),
                           "clocks": inf.get("clocks")}
        except Exception as e:   # report, do not hide
            extra[name] = {"error": str(e)}
    try:
        ref_bin = reference_binary_legs(sc, peak, clocks=clocks)
    except Exception as e:
        ref_bin = {"error": str(e)}
    try:
        errs = fp64_errors(culbm_b200, steps=args.err_steps)
    except Exception as e:
        errs = {"error": str(e)}
    try:
        mixed = mixed_precision_512(culbm_b200, max(20, args.steps // 10))
    except Exception as e:
        mixed = {"error": str(e)}
    try:
        adjoint = adjoint_runs() if not args.no_adjoint else None
    except Exception as e:
        adjoint = {"error": str(e)}
    e2e_mlups, h2d, d2h, e2e_same = e2e
    cpu = cpu_baseline(sc) if ws == 1 else None
    clocks.stop()

    line = {
        "metric": METRIC,
        "value": round(value, 1),
        "unit": "MLUPS",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded sphere channel in the reference's flag.dat format)",
        "config": workload_config(sc, ws),
        "policy": "streamPolicy 1 (in-place AA), optPolicy 0",
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} copy bandwidth",
                     "algorithmic_bytes_per_lup": BYTES_PER_LUP["fp32"],
                     "traffic": traffic_from_profiles("inplace_fp32_per_step"),
                     "traffic_unit": "DRAM bytes per launch (ncu, profiles/traffic.json)",
                     "algorithmic_bytes_per_launch": BYTES_PER_LUP["fp32"] * sc.n},
        "e2e": {"value": round(e2e_mlups["overlapped"], 1), "unit": "MLUPS",
                "h2d_bytes_per_step": round(h2d / args.steps), "d2h_bytes_per_step": round(d2h / args.steps),
                "what": f"one culbm_run_host call: init state (flag, rho, u) from page-locked host memory, "
                        f"{args.steps} steps, dump kernel, rho/vx/vy/vz to page-locked host memory; the slabs' "
                        f"copies overlap the steps; host wall clock, best of 3",
                "sequential": round(e2e_mlups["sequential"], 1),
                "sequential_what": "culbm_load_state + culbm_step + culbm_moments + 4x culbm_get_field "
                                   "(copies before and after the steps), same buffers",
                "same_bits": bool(e2e_same)},
        "gpu_launches": launches,
        "clocks": headline_clocks,
        "clocks_whole_run": clocks.summary(),
        "cpu_baseline": cpu,
        "variants": extra,
        "selector": {"fp32": selector_summary(sel)},
        "reference_binary": ref_bin,
        "fp64_error": errs,
        "mixed_precision_512x512x256": mixed,
        "adjoint": adjoint,
    }
    print(json.dumps(line), flush=True)
    if tdist is not None:
        tdist.destroy_process_group()


# -------------------------------------------------------------- reference ---

def run_reference(args):
    ws, rank = dist()
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_lbm_core.so not built "
                                                             "(make -C oracle ref-cpu needs the reference tree)"}))
        return
    from culbm_b200 import scenes
    sc = scenes.spheres_288()
    f, r, ux, uy, uz = sc.arrays()
    nx, ny, nz = sc.shape
    o = oracle.Scene(nx, ny, nz, f, r, ux, uy, uz)
    a = oracle.rest_state(o.n)
    b = a.copy()
    threads = oracle.ref().ref_max_threads()
    # Each step is one lattice update of a z-slab sample sized so that the
    # whole run stays within about two minutes of CPU time.
    t0 = time.perf_counter()
    oracle.ref_step(o, 0.5, a, b)
    full_s = time.perf_counter() - t0
    total = args.steps + args.warmup
    frac = min(1.0, 100.0 / max(full_s * total, 1e-9))
    z1 = max(1, int(round(nz * frac)))
    for _ in range(args.warmup):
        oracle.ref_step(o, 0.5, a, b, 0, z1)
        a, b = b, a
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.ref_step(o, 0.5, a, b, 0, z1)
        a, b = b, a
    dt = time.perf_counter() - t0
    cells = nx * ny * z1
    mlups = cells * args.steps / dt / 1e6
    sample = (f"z-planes [0,{z1}) of {nz} ({cells} cells) per step, {args.steps} steps; reference lbm_core "
              f"(device_function.hpp) compiled for the host, OpenMP over z, {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(mlups, 2), "unit": "MLUPS", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded sphere channel in the reference's flag.dat format)",
        "config": workload_config(sc, ws),
        "policy": "the reference's lbm_core pull step (StaticD3Q27PullKernel order) on the host cores",
        "cpu_baseline": {"value": round(mlups, 2), "unit": "MLUPS", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(mlups, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--err-steps", type=int, default=1000)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint runs (about 30 s)")
    ap.add_argument("--headline-only", action="store_true",
                    help="time the headline and print its line without the other legs (for profiler launch lists)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
