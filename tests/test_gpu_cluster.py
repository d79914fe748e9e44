"""optPolicy 2 with pull streaming on the cluster engine (one thread-block
cluster per tile, populations in registers, streaming through shared memory
and DSMEM, one launch per round): the plain pull step's state bit for bit
(GPU).

The reference's own check of its blocked policies is the same comparison
against the plain pull (analysis/correctness/compare.sh).  The engine in use
shows in the launch count: two launches per round (the tiles and the
round-state advance), where the L2 tile engine needs one per tile and step.
"""
import numpy as np
import pytest

from culbm_b200 import scenes as S

from test_gpu_blocked import _valid_axis, bits, oracle_pulled, run_blocked

pytestmark = pytest.mark.gpu

# The cluster engine's limits: 16 CTAs of at most 512 threads, one per cell.
MAX_CTAS, MAX_THREADS = 16, 512


def fits_cluster(tile):
    """Whether the engine finds a CTA shape for `tile`: CTA widths that are
    multiples of 32 or the tile's own width, at most MAX_THREADS threads per
    CTA and MAX_CTAS CTAs."""
    bx, by, bz = tile
    widths = [t for t in range(32, MAX_THREADS + 1, 32) if t - 32 < bx]
    if bx % 32 and bx <= MAX_THREADS:
        widths.append(bx)
    for tx in widths:
        for ty in range(1, min(by, MAX_THREADS // tx) + 1):
            for tz in range(1, min(bz, MAX_THREADS // (tx * ty)) + 1):
                if -(-bx // tx) * -(-by // ty) * -(-bz // tz) <= MAX_CTAS:
                    return True
    return False


def rounds(nsteps, inner):
    return nsteps // inner + (1 if nsteps % inner else 0)


def assert_cluster_engine(info, nsteps, inner):
    assert info["launches_per_step"] == pytest.approx(2.0 * rounds(nsteps, inner) / nsteps, abs=1e-3)


@pytest.mark.parametrize("seed", range(6))
def test_cluster_random_geometries(culbm, orc, seed):
    """Seeded random domains, tiles (several per axis) and innerLoops, with a
    remainder round, on the channel + cube scene; graphs on and off."""
    rng = np.random.default_rng(2000 + seed)
    while True:
        dims = tuple(int(v) for v in rng.integers(14, 45, size=3))
        inner = int(rng.integers(2, 6))
        tile = tuple(int(rng.integers(max(2 * inner, 6), max(2 * inner + 1, d // 2 + 3))) for d in dims)
        if all(_valid_axis(d, b, inner) for d, b in zip(dims, tile)) and fits_cluster(tile):
            break
    sc = S.reference_channel_cube(*dims, 0.05)
    nsteps = 2 * inner + int(rng.integers(1, inner + 1))
    got, info = run_blocked(culbm, sc, 0, 2, tile, inner, nsteps, graphs=bool(seed % 2))
    assert np.array_equal(bits(got), bits(oracle_pulled(orc, sc, 0.6, nsteps))), (dims, tile, inner)
    assert_cluster_engine(info, nsteps, inner)


@pytest.mark.parametrize("inner", [1, 2, 3])
def test_cluster_random_state_and_split_steps(culbm, orc, inner):
    """Fluid everywhere from a random state: domain faces inside tiles take
    the per-axis clamp; the steps are cut into calls that leave remainder
    rounds."""
    sc = S.default_scene(37, 29, 23)
    rng = np.random.default_rng(inner)
    state0 = (0.01 * rng.standard_normal(27 * sc.n)).astype(np.float32)
    splits = [inner + 1, 2 * inner, 1]
    nsteps = sum(splits)
    got, info = run_blocked(culbm, sc, 0, 2, (20, 16, 12), inner, nsteps, state0=state0, splits=splits)
    assert np.array_equal(bits(got), bits(oracle_pulled(orc, sc, 0.6, nsteps, state0)))
    assert info["blocking_num"] == tuple(int(orc.lib().orc_blk_num(d, b, inner)) for d, b in zip((37, 29, 23),
                                                                                                   (20, 16, 12)))
    launches = sum(2 * rounds(k, inner) for k in splits)
    assert info["launches_per_step"] == pytest.approx(launches / nsteps, abs=1e-3)


@pytest.mark.parametrize("storage", ["fp64", "fp16", "fp16sr", "bf16", "bf16sr"])
def test_cluster_storages_equal_plain_pull(culbm, storage):
    """Every storage format: the exchanged populations take the format's
    rounding (stochastic bits included), so the state equals the plain pull's."""
    sc = S.reference_channel_cube(40, 30, 26, 0.05)
    dtype = np.float64 if storage == "fp64" else np.float32
    with culbm.Simulation(sc.shape, stream_policy=0, opt_policy=0, inv_tau=0.55, storage=storage) as sim:
        sim.load_state(*sc.arrays())
        sim.step(11)
        want = sim.pulled_ddf(dtype)
    got, info = run_blocked(culbm, sc, 0, 2, (22, 18, 16), 4, 11, inv_tau=0.55, storage=storage)
    assert np.array_equal(bits(got), bits(want))
    assert_cluster_engine(info, 11, 4)


def test_cluster_without_cache_hints(culbm, orc):
    sc = S.reference_channel_cube(37, 29, 23, 0.05)
    want = oracle_pulled(orc, sc, 0.6, 10)
    with culbm.Simulation(sc.shape, stream_policy=0, opt_policy=2, inv_tau=0.6, inner_loop=3, tile=(16, 12, 10),
                          cache_hints=False) as sim:
        sim.load_state(*sc.arrays())
        sim.step(10)
        got = sim.pulled_ddf()
        info = sim.info()
    assert np.array_equal(bits(got), bits(want))
    assert_cluster_engine(info, 10, 3)


def test_cluster_user_grid_and_large_tile(culbm, orc):
    """The tile is blockDim * gridDim whatever the split.  The reference's
    split is kept when it fits a cluster (blockDim at most 512 threads,
    gridDim at most 16 CTAs), else the engine picks its own; a tile no
    cluster holds runs on the L2 tile engine, with the same bits."""
    sc = S.reference_channel_cube(70, 44, 30, 0.05)
    want = oracle_pulled(orc, sc, 0.6, 7)
    for block, grid, cluster in (((32, 4, 4), (1, 4, 4), True), ((16, 4, 2), (2, 4, 4), True),
                                 ((32, 8, 2), (2, 5, 15), False)):
        with culbm.Simulation(sc.shape, stream_policy=0, opt_policy=2, inv_tau=0.6, inner_loop=3, block_dim=block,
                              grid_dim=grid) as sim:
            sim.load_state(*sc.arrays())
            sim.step(7)
            got = sim.pulled_ddf()
            info = sim.info()
        assert np.array_equal(bits(got), bits(want)), (block, grid)
        tile = tuple(b * g for b, g in zip(block, grid))
        assert fits_cluster(tile) == cluster
        if cluster:
            assert_cluster_engine(info, 7, 3)
        else:
            assert info["launches_per_step"] > 2.0
