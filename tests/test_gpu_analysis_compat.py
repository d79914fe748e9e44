"""The reference's analysis tooling against our CLI (GPU).

* analysis/blocking_experiments.py:40,115 parses a run's `speed = X (MLUPS)`
  lines with one regular expression and takes them after the first;
* analysis/correctness/run.sh:13-37 runs the solver twice on the
  generate.py scene (plain pull; in-place dynamic L2 blocking with innerLoop 9
  and the ring buffer), and compare.sh:6-9 requires the four dump files of the
  last step to be byte-identical (`cmp`).

Both are exercised here against culbm_b200/bin/single_dev_expt_main with the
same flags, the correctness pair on a scaled-down domain (run.sh's is
768x384x384 for 1539 steps: 27 GB of populations).
"""
import filecmp
import os
import re
import subprocess

import numpy as np
import pytest

from culbm_b200 import scenes as S

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUR_BIN = os.path.join(ROOT, "culbm_b200", "bin", "single_dev_expt_main")
# analysis/blocking_experiments.py:40
SPEED_RE = re.compile(r"speed = ([0-9]+(?:\.[0-9]+)?) \(MLUPS\)")


def vec(v):
    return "[" + ",".join(str(int(a)) for a in v) + "]"


def run(args):
    r = subprocess.run([OUR_BIN, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (args, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def test_speed_lines_parse_with_the_sweep_regex(tmp_path):
    """The sweep script's regex finds one speed per dstep, and the values are
    positive MLUPS (the sweep keeps all but the first)."""
    out = run(["--domainDim", "[64,32,32]", "--blockDim", "[64,32,32]", "--gridDim", "[1,1,1]", "--nstep", "40",
               "--dstep", "10", "--dumpFolder", str(tmp_path / "d")])
    speeds = [float(v) for v in SPEED_RE.findall(out)]
    assert len(speeds) == 4 and all(s > 0 for s in speeds)
    assert len(speeds[1:]) == 3


def test_correctness_pair_dumps_are_byte_identical(tmp_path):
    """run.sh's two launches, scaled to 192x96x96 (tile [96,1,1] x [1,46,42],
    innerLoop 9, 153 = 17 x 9 steps, as 1539 = 171 x 9: the blocked driver
    advances whole rounds of innerLoop steps per dump period), then
    compare.sh's four `cmp`s on the last step's dumps."""
    dims = (192, 96, 96)
    case = tmp_path / "case"
    S.write_folder(S.correctness_case(*dims, cube=(32, 32, 32, 64, 64, 64)), str(case), fields=("flag", "vx"))
    nstep = 153
    common = ["--devId", "0", "--domainDim", vec(dims), "--invTau", "0.2857142857142857", "--dstep", str(nstep),
              "--nstep", str(nstep), "--initStateFolder", str(case), "--dumpRho", "--dumpVx", "--dumpVy", "--dumpVz"]
    run([*common, "--dumpFolder", str(tmp_path / "plain"), "--blockDim", "[32,4,2]", "--gridDim", "[6,24,48]",
         "--streamPolicy", "0", "--optPolicy", "0"])
    run([*common, "--dumpFolder", str(tmp_path / "temporal"), "--blockDim", "[96,1,1]", "--gridDim", "[1,46,42]",
         "--innerLoop", "9", "--streamPolicy", "1", "--optPolicy", "3", "--useRingDDFBuf"])
    for field in ("rho", "vx", "vy", "vz"):
        a, b = tmp_path / "plain" / f"{field}_{nstep}.dat", tmp_path / "temporal" / f"{field}_{nstep}.dat"
        assert filecmp.cmp(a, b, shallow=False), field
    vx = np.fromfile(tmp_path / "plain" / f"vx_{nstep}.dat", dtype="<f4")
    assert np.max(np.abs(vx)) > 0.01   # the flow developed
