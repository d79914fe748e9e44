"""Host logic of the benchmark on the CPU.  The reference arm (``bench.py
--impl reference``): the reference's own lbm_core step compiled for the host,
timed on the same 288x272x280 workload and metric as the CUDA arm, one JSON
line from rank 0, nothing from the other ranks.  The clock summary and the
roofline's traffic figure of the CUDA arm."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(args, **env):
    e = dict(os.environ)
    e.update({k: str(v) for k, v in env.items()})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line(orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (make -C oracle ref-cpu)")
    sys.path.insert(0, ROOT)
    import bench
    r = _bench(["--impl", "reference", "--steps", "3", "--warmup", "3"], WORLD_SIZE=1, RANK=0)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "MLUPS" and line["higher_is_better"] is True
    assert line["n_gpus"] == 1 and line["steps"] == 3 and line["warmup"] == 3
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["config"]["workload"] == bench.WORKLOAD and line["config"]["cells"] == 288 * 272 * 280
    from culbm_b200 import scenes
    assert line["config"] == bench.workload_config(scenes.spheres_288(), 1)
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench(["--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "3"], WORLD_SIZE=2, RANK=1)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_fewer_than_three_warmup_steps_rejected():
    r = _bench(["--impl", "reference", "--steps", "3", "--warmup", "2"], WORLD_SIZE=1, RANK=0)
    assert r.returncode == 2 and "warmup" in r.stderr


def test_clock_summary_names_throttle_reasons():
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler()
    assert c.summary()["reasons"] == ["no samples"]
    c.max_mhz = 1965
    c.samples = [(0.0, 1965.0, 0), (1.0, 1800.0, 0x4), (2.0, 1700.0, 0x4 | 0x8), (3.0, 1965.0, 0x40)]
    s = c.summary()
    assert s["sm_mhz"] == 1882.5 and s["sm_max_mhz"] == 1965 and s["samples"] == 4
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap"]
    # a window: only its samples; a window between samples takes the nearest one
    w = c.summary(0.5, 2.5)
    assert w["samples"] == 2 and w["sm_mhz"] == 1750.0 and w["reasons"] == ["hw_slowdown", "sw_power_cap"]
    n = c.summary(2.9, 2.95)
    assert n["samples"] == 1 and n["sm_mhz"] == 1965.0 and n["reasons"] == ["hw_thermal_slowdown"]


def test_speed_lines_parse_like_the_reference_sweep():
    """Median of the `speed = X (MLUPS)` lines with the first skipped
    (analysis/blocking_experiments.py:40,115), from both drivers' output."""
    sys.path.insert(0, ROOT)
    import bench
    out = ("Init flag successfully\nspeed = 100.0000 (MLUPS)\nspeed = 25000.5000 (MLUPS)\n"
           "speed = 26000.0000 (MLUPS)\nspeed = 27000.2500 (MLUPS)\n")
    assert bench.parse_speeds(out) == 26000.0
    assert bench.parse_speeds("no speed here") is None
    assert set(bench.REF_BINARY_LEGS) >= {"readme_00", "retuned_00", "readme_13"}


def test_both_arms_share_the_config():
    sys.path.insert(0, ROOT)
    import bench
    from culbm_b200 import scenes
    sc = scenes.sphere_64()
    a, b = bench.workload_config(sc, 1), bench.workload_config(sc, 1)
    assert a == b and set(a) == {"workload", "cells", "solid_fraction", "storage", "l2", "parallelism"}


def test_roofline_traffic_is_the_committed_profile():
    sys.path.insert(0, ROOT)
    import bench
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
        d = json.load(f)["inplace_fp32_per_step"]
    assert bench.traffic_from_profiles("inplace_fp32_per_step") == d["bytes"]
    assert d["algorithmic_bytes"] == 216 * 288 * 272 * 280
    assert bench.traffic_from_profiles("no such kernel") is None
