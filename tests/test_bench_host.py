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
    c.samples = [(1965.0, 0), (1800.0, 0x4), (1700.0, 0x4 | 0x8), (1965.0, 0x40)]
    s = c.summary()
    assert s["sm_mhz"] == 1882.5 and s["sm_max_mhz"] == 1965 and s["samples"] == 4
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap"]


def test_roofline_traffic_is_the_committed_profile():
    sys.path.insert(0, ROOT)
    import bench
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
        d = json.load(f)["inplace_fp32_per_step"]
    assert bench.traffic_from_profiles("inplace_fp32_per_step") == d["bytes"]
    assert d["algorithmic_bytes"] == 216 * 288 * 272 * 280
    assert bench.traffic_from_profiles("no such kernel") is None
