"""16-bit population storage (FP16 scaled by 2^15, BF16; nearest-even and
stochastic rounding) against the oracle's 16-bit emulation, bit for bit, in
every streaming policy (GPU).  The reference has no 16-bit path; the oracle
widens, runs its FP32 pull step and narrows with the same rules."""
import numpy as np
import pytest

from culbm_b200 import scenes as S

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def oracle_pulled16(orc, scene, storage, inv_tau, nsteps):
    f, r, ux, uy, uz = scene.arrays()
    nx, ny, nz = scene.shape
    o = orc.Scene(nx, ny, nz, f, r, ux, uy, uz)
    return orc.pulled(o, orc.run_s16(o, storage, inv_tau, nsteps))


@pytest.mark.parametrize("storage", ["fp16", "bf16", "fp16sr", "bf16sr"])
@pytest.mark.parametrize("policy", [(0, 0), (1, 0), (1, 3), (0, 3)])
def test_storage16_matches_oracle(culbm, orc, storage, policy):
    sc = S.reference_channel_cube(34, 22, 18, 0.05)
    sc.flag[0, :, :] = S.FLUID          # one fluid face: exercises the clamped edge too
    nsteps = 11
    want = oracle_pulled16(orc, sc, storage, 0.55, nsteps)
    sp, op = policy
    kw = dict(tile=(18, 14, 12), inner_loop=3) if op else {}
    with culbm.Simulation(sc.shape, stream_policy=sp, opt_policy=op, inv_tau=0.55, storage=storage, **kw) as sim:
        sim.load_state(*sc.arrays())
        sim.step(nsteps)
        got = sim.pulled_ddf()
    assert np.array_equal(bits(got), bits(want)), (storage, policy)


@pytest.mark.parametrize("storage", ["fp16", "bf16", "fp16sr", "bf16sr"])
@pytest.mark.parametrize("dims", [(150, 5, 4), (151, 4, 5), (7, 3, 3), (1, 4, 3), (2, 3, 3)])
def test_storage16_pull_pairs_and_x_faces(culbm, orc, storage, dims):
    """The two-cells-per-thread pull of the 16-bit formats: even nx (packed
    stores) and odd nx (single stores), warps away from and at the x-faces
    (nx > 128), pairs with a non-storing (solid) cell, single-cell rows."""
    sc = S.reference_channel(*dims, 0.05)
    sc.flag[0, :, :] = S.FLUID
    rng = np.random.default_rng(sum(dims))
    solid = rng.random(sc.flag.shape) < 0.08
    sc.flag[solid] = 0
    nsteps = 5
    want = oracle_pulled16(orc, sc, storage, 0.7, nsteps)
    with culbm.Simulation(sc.shape, stream_policy=0, inv_tau=0.7, storage=storage) as sim:
        sim.load_state(*sc.arrays())
        sim.step(nsteps)
        got = sim.pulled_ddf()
    assert np.array_equal(bits(got), bits(want)), (storage, dims)


def test_stochastic_rounding_is_unbiased(culbm):
    """Mean of many stochastically rounded copies of one value tends to the
    value (nearest-even would sit on one side); checked through a state
    import, where every (cell, direction) gets independent random bits."""
    dims = (64, 32, 16)
    n = dims[0] * dims[1] * dims[2]
    v = np.float32(1.2345678e-3)
    state = np.full(27 * n, v, np.float32)
    with culbm.Simulation(dims, stream_policy=0, storage="fp16sr") as sim:
        sim.set_ddf(state)
        got = sim.pulled_ddf().astype(np.float64)
    interior = got.reshape(27, dims[2], dims[1], dims[0])[:, 1:-1, 1:-1, 1:-1]
    ulp = 2.0 ** 5 * 2.0 ** -10 / 32768.0    # ulp of v*2^15 = 40.45 (exponent 2^5), back in f units
    assert abs(interior.mean() - float(v)) < 0.02 * ulp
    assert len(np.unique(interior)) == 2
