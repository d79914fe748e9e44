"""L2 temporal blocking (optPolicy 1, 2, 3): every blocked configuration must
give the plain pull step's state bit for bit (GPU).

The reference pins its (1,3)+ring path the same way: analysis/correctness/
compare.sh requires bitwise-equal dumps against the plain pull.  Here the
comparison is against the oracle's pull step, on full populations.
"""
import numpy as np
import pytest

from culbm_b200 import scenes as S

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def oracle_pulled(orc, scene, inv_tau, nsteps, state0=None, dtype=np.float32):
    f, r, ux, uy, uz = scene.arrays()
    nx, ny, nz = scene.shape
    o = orc.Scene(nx, ny, nz, f, r, ux, uy, uz)
    return orc.pulled(o, orc.run(o, inv_tau, nsteps, dtype=dtype, state=state0))


def run_blocked(culbm, scene, sp, op, tile, inner, nsteps, inv_tau=0.6, ring=False, state0=None, storage="fp32",
                graphs=True, splits=None, persist=False):
    with culbm.Simulation(scene.shape, stream_policy=sp, opt_policy=op, inv_tau=inv_tau, inner_loop=inner,
                          tile=tile, use_ring=ring, storage=storage, use_graphs=graphs, persist_l2=persist) as sim:
        sim.load_state(*scene.arrays())
        if state0 is not None:
            sim.set_ddf(state0)
        for k in (splits or [nsteps]):
            sim.step(k)
        info = sim.info()
        return sim.pulled_ddf(np.float64 if storage == "fp64" else np.float32), info


CASES = [
    # (stream, opt, ring, tile, innerLoop)
    (1, 3, False, (16, 12, 10), 3),
    (1, 3, True, (16, 12, 10), 3),
    (1, 3, True, (37, 29, 9), 4),
    (0, 3, False, (16, 12, 10), 3),
    (0, 1, False, (16, 12, 10), 2),
    (1, 1, False, (20, 16, 12), 5),
    (0, 2, False, (37, 8, 23), 2),
    (1, 3, False, (16, 12, 10), 1),
    (0, 3, False, (16, 12, 10), 1),
]


@pytest.mark.parametrize("sp,op,ring,tile,inner", CASES)
def test_blocked_equals_pull_default_flags(culbm, orc, sp, op, ring, tile, inner):
    """Fluid everywhere: domain faces inside tiles exercise the per-axis clamp."""
    sc = S.default_scene(37, 29, 23)
    rng = np.random.default_rng(inner)
    state0 = (0.01 * rng.standard_normal(27 * sc.n)).astype(np.float32)
    nsteps = 2 * inner + 1 if inner > 1 else 3     # a remainder round when inner > 1
    got, info = run_blocked(culbm, sc, sp, op, tile, inner, nsteps, state0=state0, ring=ring)
    assert np.array_equal(bits(got), bits(oracle_pulled(orc, sc, 0.6, nsteps, state0)))
    L = orc.lib()
    assert info["blocking_num"] == tuple(int(L.orc_blk_num(d, b, inner)) for d, b in zip((37, 29, 23), tile))


@pytest.mark.parametrize("sp,ring", [(1, False), (1, True), (0, False)])
def test_blocked_channel_with_obstacle(culbm, orc, sp, ring):
    """The reference's channel + cube scene, 3 rounds of innerLoop 5."""
    sc = S.reference_channel_cube(48, 40, 36, 0.05)
    got, _ = run_blocked(culbm, sc, sp, 3, (24, 20, 18), 5, 15, inv_tau=0.5, ring=ring)
    assert np.array_equal(bits(got), bits(oracle_pulled(orc, sc, 0.5, 15)))


def test_blocked_graphs_off_and_split_steps(culbm, orc):
    sc = S.reference_channel(30, 20, 16, 0.05)
    want = oracle_pulled(orc, sc, 0.5, 13)
    for graphs, splits in ((False, [13]), (True, [4, 9]), (True, [1, 1, 11])):
        got, _ = run_blocked(culbm, sc, 1, 3, (16, 12, 10), 3, 13, inv_tau=0.5, graphs=graphs, splits=splits)
        assert np.array_equal(bits(got), bits(want)), (graphs, splits)


@pytest.mark.parametrize("sp", [1, 0])
def test_blocked_tile_lanes_and_persisting_window(culbm, orc, sp):
    """Tiles of a round run on two streams (each with its own tile and edge
    buffers) unless the ring buffer is on; with the persisting-L2 window they
    do so only when both lanes' buffers fit in L2.  An odd tile count leaves
    the lanes uneven.  Every combination gives the plain pull's bits."""
    sc = S.reference_channel_cube(45, 30, 26, 0.05)
    want = oracle_pulled(orc, sc, 0.5, 8)
    for persist in (False, True):
        for graphs in (True, False):
            got, info = run_blocked(culbm, sc, sp, 3, (18, 14, 12), 3, 8, inv_tau=0.5, graphs=graphs,
                                    persist=persist)
            assert np.array_equal(bits(got), bits(want)), (persist, graphs)
            if not persist:
                assert info["persisting_l2_bytes"] == 0
        assert info["blocking_num"][0] * info["blocking_num"][1] * info["blocking_num"][2] % 2 == 1


def test_blocked_fp64_and_moments(culbm, orc):
    sc = S.reference_channel(26, 18, 14, 0.05)
    got, _ = run_blocked(culbm, sc, 1, 3, (14, 10, 8), 3, 9, inv_tau=0.5, storage="fp64")
    assert np.array_equal(bits(got), bits(oracle_pulled(orc, sc, 0.5, 9, dtype=np.float64)))
    f, r, ux, uy, uz = sc.arrays()
    o = orc.Scene(26, 18, 14, f, r, ux, uy, uz)
    want = orc.moments(o, orc.run(o, 0.5, 9))
    for ring in (False, True):
        with culbm.Simulation(sc.shape, stream_policy=1, opt_policy=3, inner_loop=3, tile=(14, 10, 8),
                              use_ring=ring, inv_tau=0.5) as sim:
            sim.load_state(f, r, ux, uy, uz)
            sim.step(9)
            sim.moments()
            for k, w in zip(("rho", "vx", "vy", "vz"), want):
                assert np.array_equal(bits(sim.field(k)), bits(w)), (ring, k)


def _valid_axis(dom, blk, it):
    """blocking_core::validBlkAxisConfig and the engine's extra check (the
    tile must be large enough for innerLoop when more than two are needed)."""
    if blk < dom and blk + 1 <= it:
        return False
    if 2 * (blk + 1 - it) < dom and blk + 2 <= it:
        return False
    if dom > blk and dom > 2 * (blk + 1 - it) and blk + 2 - 2 * it <= 0:
        return False
    return True


@pytest.mark.parametrize("seed", range(6))
def test_blocked_random_geometries(culbm, orc, seed):
    """Seeded random domains, tile extents and innerLoops with several tiles
    per axis (two concurrent tile lanes), in-place and pull tiles, graphs on
    and off, against the oracle's pull bit for bit."""
    rng = np.random.default_rng(1000 + seed)
    while True:
        dims = tuple(int(v) for v in rng.integers(14, 41, size=3))
        inner = int(rng.integers(2, 6))
        tile = tuple(int(rng.integers(max(2 * inner, 6), max(2 * inner + 1, d // 2 + 3))) for d in dims)
        if all(_valid_axis(d, b, inner) for d, b in zip(dims, tile)):
            break
    sc = S.reference_channel_cube(*dims, 0.05)
    nsteps = 2 * inner + int(rng.integers(0, inner))
    want = oracle_pulled(orc, sc, 0.6, nsteps)
    for sp in (1, 0):
        got, info = run_blocked(culbm, sc, sp, 3, tile, inner, nsteps, graphs=bool(seed % 2))
        assert np.array_equal(bits(got), bits(want)), (dims, tile, inner, sp)


@pytest.mark.parametrize("sp,op,ring", [(1, 3, False), (1, 3, True), (0, 3, False), (1, 1, False)])
def test_blocked_without_cache_hints_equals_pull(culbm, orc, sp, op, ring):
    """cache_hints = 0 (no evict-first / evict-last hints, the reference build
    switch CULBM_EXPT_CACHE_HINT_POLICY=0 of src/simulator/single_dev_expt/
    CMakeLists.txt:28-41): the same bits as the plain pull."""
    sc = S.reference_channel_cube(37, 29, 23, 0.05)
    nsteps = 13
    want = oracle_pulled(orc, sc, 0.6, nsteps)
    with culbm.Simulation(sc.shape, stream_policy=sp, opt_policy=op, inv_tau=0.6, inner_loop=3, tile=(16, 12, 10),
                          use_ring=ring, cache_hints=False) as sim:
        sim.load_state(*sc.arrays())
        sim.step(nsteps)
        got = sim.pulled_ddf()
    assert np.array_equal(bits(got), bits(want))

