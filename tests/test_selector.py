"""Tile/innerLoop selector of the L2-blocked policies (culbm_select_tile,
culbm_blocking_speedup): the model restated in selector.cu against golden
values of the reference's own analysis/selector.py (tests/golden/
make_selector_golden.py), on CPU: with the constants given, no device is
touched."""
import json
import os

import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "selector_reference.json")


def cases():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", cases(), ids=lambda c: f"lambda{c['lambda']}")
def test_model_values_match_the_reference(culbm, case):
    from culbm_b200 import selector
    for bx, by, bz, it, s_ref, s0_ref in case["points"]:
        s, s0 = selector.speedup((bx, by, bz), it, "fp32", case["lambda"], case["gamma"], case["l2_bytes"])
        assert s == pytest.approx(s_ref, rel=1e-12), (bx, by, bz, it)
        assert s0 == pytest.approx(s0_ref, rel=1e-12), (bx, by, bz, it)


@pytest.mark.parametrize("case", cases(), ids=lambda c: f"lambda{c['lambda']}")
def test_choice_matches_the_reference_on_a_large_domain(culbm, case):
    """On a domain large enough for every tile the choice is the model's argmax."""
    from culbm_b200 import selector
    got = selector.select((4096, 4096, 4096), "fp32", case["lambda"], case["gamma"], case["l2_bytes"],
                          case["persist_bytes"])
    assert got["tile"] + [got["inner_loop"]] == case["argmax"]
    assert got["speedup"] == pytest.approx(case["S_argmax"], rel=1e-12)


def test_choice_respects_the_domain_and_storage(culbm):
    from culbm_b200 import selector
    from culbm_b200._capi import CulbmError
    c = cases()[0]
    big = selector.select((4096, 4096, 4096), "fp32", c["lambda"], c["gamma"], c["l2_bytes"], c["persist_bytes"])
    half = selector.select((4096, 4096, 4096), "fp16", c["lambda"], c["gamma"], c["l2_bytes"], c["persist_bytes"])
    # half the bytes per cell: at least as large a tile fits the persisting window
    assert half["tile"][0] * half["tile"][1] * half["tile"][2] >= big["tile"][0] * big["tile"][1] * big["tile"][2]
    small = selector.select((64, 40, 40), "fp32", c["lambda"], c["gamma"], c["l2_bytes"], c["persist_bytes"])
    from culbm_b200 import _capi
    import oracle
    L = oracle.lib()
    for k, dom in enumerate((64, 40, 40)):
        assert L.orc_valid_blk_axis(dom, small["tile"][k], small["inner_loop"])
    with pytest.raises(CulbmError):
        selector.select((4096, 4096, 4096), "fp32", c["lambda"], c["gamma"], c["l2_bytes"], 1000)


def test_blocking_axis_bounds(culbm):
    from culbm_b200 import _capi, selector
    # 288 cells, tile 64, innerLoop 5: first valid region 64 + 1 - 5 = 60
    # cells, then 64 + 2 - 10 = 56 per tile, the last tile takes the rest.
    assert selector.blocking_axis(288, 64, 5) == [0, 60, 116, 172, 228, 288]
    assert selector.blocking_axis(280, 288, 3) == [0, 280]
    with pytest.raises(_capi.CulbmError, match="don't match"):
        selector.blocking_axis(64, 4, 3)


def _header_constant(name):
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "culbm.h")
    m = re.search(r"#define\s+" + name + r"\s+([0-9.]+)", open(path).read())
    return float(m.group(1))


@pytest.mark.parametrize("domain", [(288, 272, 280), (512, 512, 256), (1024, 512, 512)])
def test_b200_speedup_uses_the_measured_step_costs(culbm, domain):
    """predicted_speedup_b200 = h max(1, plain) / max(D, tile) for the chosen
    tile, with the header's measured B200 costs; below 1 (plain streaming is
    faster on B200) for FP32 and the 16-bit formats; FP64 has no measured costs
    and keeps the model's value."""
    from culbm_b200 import selector
    l2, persist = 126 << 20, 80 << 20
    plain32, tile32 = _header_constant("CULBM_B200_PLAIN_32"), _header_constant("CULBM_B200_TILE_32")
    plain16, tile16 = _header_constant("CULBM_B200_COMPUTE_16"), _header_constant("CULBM_B200_TILE_16")
    for storage in ("fp32", "fp16sr", "bf16", "fp64"):
        s = selector.select(domain, storage, l2_bytes=l2, persist_bytes=persist)
        r = s["inner_loop"] - 1
        h = 1.0
        for b in s["tile"]:
            h *= 1 - 2 * r / b
        if storage == "fp64":
            assert s["speedup_b200"] == pytest.approx(s["speedup"], rel=1e-12)
            continue
        if storage == "fp32":
            d = h / s["speedup"]          # the model's own round time (S = h / D for FP32)
            want = h * max(1.0, plain32) / max(d, tile32)
        else:
            want = h * max(1.0, plain16) / tile16   # D is far below the tile cost here
        assert s["speedup_b200"] == pytest.approx(want, rel=1e-9)
        assert s["speedup_b200"] < 1.0
