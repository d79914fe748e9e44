"""Known answers of sm_100a's packed stochastic-rounding conversions
(cvt.rs.f16x2.f32 and cvt.rs.bf16x2.f32), for tests/test_oracle.py.

Needs a B200 (sm_100a) and nvcc: compiles tests/golden/cvt_rs_probe.cu, runs
it, and keeps the structured cases plus a seeded sample of the random ones in
cvt_rs_sm100a.npz (inputs a, b, rbits and the packed f16x2 / bf16x2 results
without saturation).

    python tests/golden/make_cvt_rs_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def run_probe(workdir: str):
    """Builds and runs the probe; returns (a, b, rbits, f16x2, f16x2_sat, bf16x2, bf16x2_sat)."""
    exe = os.path.join(workdir, "cvt_rs_probe")
    out = os.path.join(workdir, "cvt_rs_probe.bin")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++20", "-o", exe,
                    os.path.join(HERE, "cvt_rs_probe.cu")], check=True)
    subprocess.run([exe, out], check=True)
    raw = np.fromfile(out, dtype=np.uint32)
    n = int(raw[0])
    cols = [raw[1 + k * n:1 + (k + 1) * n] for k in range(7)]
    return (cols[0].view(np.float32), cols[1].view(np.float32), cols[2], *cols[3:])


def main() -> int:
    with tempfile.TemporaryDirectory() as tmp:
        a, b, r, h, hs, bf, bfs = run_probe(tmp)
    rng = np.random.default_rng(2026)
    keep = np.concatenate([np.arange(160), 160 + rng.choice(a.size - 160, 4000, replace=False)])
    np.savez_compressed(os.path.join(HERE, "cvt_rs_sm100a.npz"), a=a[keep], b=b[keep], rbits=r[keep],
                        f16x2=h[keep], bf16x2=bf[keep])
    print(f"wrote {keep.size} cases")
    return 0


if __name__ == "__main__":
    sys.exit(main())
