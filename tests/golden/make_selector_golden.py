"""Golden values of the reference's blocking speed-up model
(analysis/selector.py of the reference tree), for tests/test_selector.py.

Runs the reference's own script (it searches at import time), then
re-evaluates its S and S0 functions and its argmax under other constants by
rebinding the module globals those functions read.  Writes selector_reference.json.

    python tests/golden/make_selector_golden.py /path/to/reference
"""
import json
import os
import runpy
import sys

import numpy as np

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CULBM_REFERENCE", "/root/reference")
g = runpy.run_path(os.path.join(ref, "analysis", "selector.py"))

out = {"source": "analysis/selector.py", "cell_bytes": int(g["CELL_BYTES"]), "cases": []}
for lam, gam, l2, persist in [(0.19103, 10.1228, 128 * 2**20, 80 * 2**20),
                              (0.4, 3.0, 126 * 2**20, 82 * 2**20),
                              (0.6, 1.5, 126 * 2**20, 50 * 2**20)]:
    # run_path returns a copy of the module namespace: rebind in the one the
    # model's functions read
    ns = g["S"].__globals__
    ns["LAMBDA"], ns["GAMMA"], ns["L2"], ns["PERSISTING_L2"] = lam, gam, l2, persist
    I, Bx, By, Bz = np.ogrid[g["I_MIN"]:g["I_MAX"] + 1, 32:g["B_MAX"] + 1:32, 1:g["B_MAX"] + 1, 1:g["B_MAX"] + 1]
    cb = g["CELL_BYTES"]
    valid = (Bx * By * Bz <= persist / cb) & (Bx > 2 * (I - 1)) & (By >= Bz) & (Bz > 2 * (I - 1))
    score = np.where(valid, g["S"](Bx, By, Bz, I), -np.inf)
    i, bx, by, bz = np.unravel_index(np.argmax(score), score.shape)
    best = [int(32 * (bx + 1)), int(by + 1), int(bz + 1), int(i + g["I_MIN"])]
    points = []
    for (x, y, z, it) in [(96, 94, 86, 9), (64, 96, 76, 5), (32, 32, 32, 2), (160, 160, 40, 12), (128, 60, 30, 7),
                          (96, 50, 44, 3)]:
        a = lambda v: np.array([v])
        points.append([x, y, z, it, float(g["S"](a(x), a(y), a(z), a(it))[0]),
                       float(g["S0"](a(x), a(y), a(z), a(it))[0])])
    out["cases"].append({"lambda": lam, "gamma": gam, "l2_bytes": l2, "persist_bytes": persist,
                         "argmax": best, "S_argmax": float(score.max()), "points": points})
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_reference.json"), "w") as f:
    json.dump(out, f, indent=1)
print(json.dumps(out)[:400])
