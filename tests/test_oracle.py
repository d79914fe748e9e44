"""The CPU oracle pinned against the reference (CPU only).

Two pins: the golden fixtures of tests/golden/ (made from the reference's own
lbm_core routines, see make_golden.py) and, when oracle/_ref was built, the
reference routines called live on fresh random inputs.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32 if a.dtype == np.float32 else np.uint64)


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_unit_vectors_bitwise(orc):
    g = load("unit_vectors.npz")
    for k in range(g["rho"].size):
        e = orc.equ(g["rho"][k], *g["u"][k])
        assert np.array_equal(bits(e), bits(g["equ"][k])), k
        c = orc.collide(g["inv_tau"][k], g["f"][k])
        assert np.array_equal(bits(c), bits(g["collide"][k])), k
        m = np.array(orc.rhou(np.ascontiguousarray(g["f"][k])), np.float32)
        assert np.array_equal(bits(m), bits(g["moments"][k])), k


@pytest.mark.parametrize("name", ["random_13x11x9.npz", "channel_16x12x10.npz", "stream_9x7x5.npz"])
def test_stepped_fixtures_bitwise(orc, name):
    g = load(name)
    sc = orc.Scene(int(g["nx"]), int(g["ny"]), int(g["nz"]), g["flag"], g["rho"], g["vx"], g["vy"], g["vz"])
    out = orc.run(sc, float(g["inv_tau"]), int(g["nsteps"]), state=g["state0"])
    assert np.array_equal(bits(out), bits(g["state"]))
    assert np.array_equal(bits(orc.pulled(sc, out)), bits(g["pulled"]))
    mom = orc.moments(sc, out)
    for got, key in zip(mom, ("d_rho", "d_vx", "d_vy", "d_vz")):
        assert np.array_equal(bits(got), bits(g[key])), key


def test_streaming_fixture_is_permutation(orc):
    """LOAD|STORE only: every pulled value is some population of the start state."""
    g = load("stream_9x7x5.npz")
    start = set(bits(g["state0"]).tolist())
    assert set(bits(g["state"]).tolist()) <= start


def test_oracle_matches_reference_live(orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (make -C oracle ref-cpu)")
    rng = np.random.default_rng(7)
    nx, ny, nz = 11, 9, 7
    n = nx * ny * nz
    combos = np.array([orc.LOAD | orc.COLLIDE | orc.STORE | orc.DUMP_ALL, orc.LOAD | orc.BOUNCE_BACK | orc.STORE,
                       orc.EQU | orc.STORE, orc.LOAD | orc.COLLIDE, 0], np.uint32)
    sc = orc.Scene(nx, ny, nz, rng.choice(combos, n), rho=(1 + 0.01 * rng.standard_normal(n)).astype(np.float32),
                   vx=(0.02 * rng.standard_normal(n)).astype(np.float32))
    a = orc.run(sc, 1.3, 9)
    b = orc.ref_run(sc, 1.3, 9)
    assert np.array_equal(bits(a), bits(b))
    for x, y in zip(orc.moments(sc, a), orc.ref_moments(sc, b)):
        assert np.array_equal(bits(x), bits(y))


@pytest.mark.parametrize("dims", [(1, 1, 1), (1, 5, 4), (5, 1, 4), (5, 4, 1), (2, 2, 2), (3, 2, 5), (33, 3, 2)])
def test_oracle_matches_reference_live_on_degenerate_domains(orc, dims):
    """Single-cell, one- and two-cell-thick domains: every pull is clamped on
    at least one axis (kernel.cu:2506-2511), so each population of a cell is
    read from itself or from a neighbour along a face."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (make -C oracle ref-cpu)")
    nx, ny, nz = dims
    n = nx * ny * nz
    rng = np.random.default_rng(nx * 10007 + ny * 101 + nz)
    combos = np.array([orc.LOAD | orc.COLLIDE | orc.STORE | orc.DUMP_ALL, orc.LOAD | orc.BOUNCE_BACK | orc.STORE,
                       orc.EQU | orc.STORE | orc.DUMP_ALL, orc.LOAD | orc.STORE, orc.LOAD | orc.COLLIDE, 0], np.uint32)
    sc = orc.Scene(nx, ny, nz, rng.choice(combos, n), rho=(1 + 0.01 * rng.standard_normal(n)).astype(np.float32),
                   vx=(0.02 * rng.standard_normal(n)).astype(np.float32),
                   vy=(0.01 * rng.standard_normal(n)).astype(np.float32),
                   vz=(0.01 * rng.standard_normal(n)).astype(np.float32))
    a = orc.run(sc, 0.7, 5)
    b = orc.ref_run(sc, 0.7, 5)
    assert np.array_equal(bits(a), bits(b))
    for x, y in zip(orc.moments(sc, a), orc.ref_moments(sc, b)):
        assert np.array_equal(bits(x), bits(y))


def test_fp64_oracle_close_to_fp32(orc):
    g = load("channel_16x12x10.npz")
    sc = orc.Scene(int(g["nx"]), int(g["ny"]), int(g["nz"]), g["flag"], g["rho"], g["vx"], g["vy"], g["vz"])
    f32 = orc.run(sc, 0.5, 30)
    f64 = orc.run(sc, 0.5, 30, dtype=np.float64)
    assert np.max(np.abs(f64 - f32)) < 1e-6
    assert np.max(np.abs(f64)) > 1e-3   # the flow is not trivial


def test_blocking_geometry_matches_reference(orc):
    L = orc.lib()
    R = orc.ref() if orc.ref_available() else None
    for dom in (7, 64, 96, 280, 288, 384, 768):
        for blk in (4, 16, 64, 76, 96, 128):
            for it in (1, 2, 3, 5, 9):
                v = L.orc_valid_blk_axis(dom, blk, it)
                if R is not None:
                    assert v == R.ref_valid_blk_axis(dom, blk, it)
                if not v:
                    continue
                if dom > blk and dom > 2 * (blk + 1 - it) and blk + 2 - 2 * it <= 0:
                    # validBlkAxisConfig lets this through but calcBlkNum then
                    # divides by blk+2-2*it <= 0 (the reference crashes or wraps);
                    # culbm_b200 rejects it at create time instead.
                    continue
                num = L.orc_blk_num(dom, blk, it)
                if R is not None:
                    assert num == R.ref_blk_num(dom, blk, it)
                prev = [L.orc_valid_prev(k, blk, num, it, dom) for k in range(num + 1)]
                if R is not None:
                    assert prev == [R.ref_valid_prev(k, blk, num, it, dom) for k in range(num + 1)]
                assert prev[0] == 0 and prev[-1] == dom
                assert all(b >= a for a, b in zip(prev, prev[1:]))


def test_compact_update_of_16bit_formats_is_the_same_bgk(orc):
    """The compact cell update used with 16-bit storage (oracle restatement of
    cell_update_fast) and the reference-order update are the same BGK step up
    to FP32 rounding.  Judged against the FP64 update, the compact form stays
    within a few ulp of the largest population (the reference's order loses
    more to cancellation on these random states)."""
    L = orc.lib()
    rng = np.random.default_rng(5)
    worst = 0.0
    for flag in (orc.LOAD | orc.COLLIDE | orc.STORE, orc.EQU | orc.COLLIDE | orc.STORE,
                 orc.LOAD | orc.BOUNCE_BACK | orc.COLLIDE | orc.STORE, orc.EQU | orc.STORE):
        for _ in range(200):
            f0 = (0.02 * rng.standard_normal(27)).astype(np.float32)
            w = np.float32(rng.uniform(0.3, 1.9))
            r_in, ux, uy, uz = np.float32(1 + 0.02 * rng.standard_normal()), *(0.05 * rng.standard_normal(3)).astype(
                np.float32)
            fast, exact = f0.copy(), f0.copy()
            exact64 = f0.astype(np.float64)
            L.orc_cell_fast_f32(flag, w, r_in, ux, uy, uz, fast)
            L.orc_cell_f32(flag, w, r_in, ux, uy, uz, exact)
            L.orc_cell_f64(flag, float(w), float(r_in), float(ux), float(uy), float(uz), exact64)
            scale = np.max(np.abs(exact64)) + 1e-30
            e_fast = np.max(np.abs(fast - exact64)) / scale
            e_exact = np.max(np.abs(exact - exact64)) / scale
            assert e_fast < 1e-6 and e_exact < 1e-4, (flag, e_fast, e_exact)
            worst = max(worst, e_fast)
    assert worst > 0   # the two forms do differ in rounding


def test_stochastic_rounding_rule_matches_sm100a_known_answers(orc):
    """The oracle's restatement of cvt.rs (f16 and bf16, no saturation) against
    outputs of sm_100a's cvt.rs.f16x2.f32 / cvt.rs.bf16x2.f32 recorded on a
    B200 (tests/golden/make_cvt_rs_golden.py): rbits bits 0-12 / 0-15 round the
    low half, bits 16-28 / 16-31 the high half.  Structured cases (carry from
    an all-ones fraction per random bit, zeros, infinities, NaN, overflow,
    half subnormals) and seeded random values over the whole FP32 range."""
    g = np.load(os.path.join(GOLDEN, "cvt_rs_sm100a.npz"))
    a, b, r = g["a"], g["b"], g["rbits"]
    for kind, mask, packed in (("f16", 0x1FFF, g["f16x2"]), ("bf16", 0xFFFF, g["bf16x2"])):
        lo = orc.round16_sr(kind, b, r & mask)
        hi = orc.round16_sr(kind, a, (r >> 16) & mask)
        assert np.array_equal(lo, (packed & 0xFFFF).astype(np.uint16)), kind
        assert np.array_equal(hi, (packed >> 16).astype(np.uint16)), kind
