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


def test_hardware_stochastic_rounding_matches_oracle_rule(orc, tmp_path):
    """sm_100a's cvt.rs.f16x2.f32 / cvt.rs.bf16x2.f32, run now on this GPU
    over 2^20 seeded (a, b, rbits) triples (tests/golden/cvt_rs_probe.cu),
    against the oracle's restatement of the rule the storage kernels use."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "make_cvt_rs_golden", os.path.join(os.path.dirname(__file__), "golden", "make_cvt_rs_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    a, b, r, f16, _, bf16, _ = gen.run_probe(str(tmp_path))
    for kind, mask, packed in (("f16", 0x1FFF, f16), ("bf16", 0xFFFF, bf16)):
        lo = orc.round16_sr(kind, b, r & mask)
        hi = orc.round16_sr(kind, a, (r >> 16) & mask)
        assert np.array_equal(lo, (packed & 0xFFFF).astype(np.uint16)), kind
        assert np.array_equal(hi, (packed >> 16).astype(np.uint16)), kind


ROW_DOMAINS = [(32, 3, 3), (48, 7, 5), (64, 12, 10), (96, 5, 9)]


@pytest.mark.parametrize("storage", ["fp16", "bf16", "fp16sr", "bf16sr"])
@pytest.mark.parametrize("sp", [0, 1])
@pytest.mark.parametrize("dims", ROW_DOMAINS)
def test_row_staged_kernels_match_oracle(culbm, orc, storage, sp, dims):
    """The row-staged 16-bit kernels (nx a multiple of 16): pull over every
    row, in place over the inner rows with the face rows on the per-cell
    kernels.  Fluid x faces (clamped pulls of inner rows from the edge
    buffer), solid cells without STORE, EQU inlet/outlet rows; odd and even
    step counts."""
    sc = S.reference_channel(*dims, 0.05)
    sc.flag[:, :, 0] = S.FLUID
    sc.flag[:, :, -1] = S.FLUID
    rng = np.random.default_rng(sum(dims) + sp)
    solid = rng.random(sc.flag.shape) < 0.06
    sc.flag[solid] = 0
    for nsteps in (6, 7):
        want = oracle_pulled16(orc, sc, storage, 0.6, nsteps)
        with culbm.Simulation(sc.shape, stream_policy=sp, inv_tau=0.6, storage=storage, kernel_variant=1) as sim:
            sim.load_state(*sc.arrays())
            sim.step(nsteps)
            got = sim.pulled_ddf()
            launches = sim.info()["launches_per_step"]
        assert launches == (2.0 if sp == 1 else 1.0)   # the row path ran (in place: face rows + inner rows)
        assert np.array_equal(bits(got), bits(want)), (storage, sp, dims, nsteps)


@pytest.mark.parametrize("storage", ["fp16sr", "bf16"])
@pytest.mark.parametrize("sp", [0, 1])
def test_row_staged_kernels_equal_per_cell_kernels(culbm, storage, sp):
    """kernel_variant 0 (per-cell) and 1, 2 (row-staged, one or two output
    buffers) give the same bits on a larger domain with random flags, over
    many rows per block."""
    dims = (160, 40, 36)
    sc = S.default_scene(*dims)
    rng = np.random.default_rng(17)
    pick = rng.random(sc.flag.shape)
    sc.flag[pick < 0.05] = S.WALL
    sc.flag[(pick >= 0.05) & (pick < 0.07)] = S.EQUILIBRIUM
    sc.flag[(pick >= 0.07) & (pick < 0.08)] = 0
    sc.rho[:] = (1 + 0.01 * rng.standard_normal(sc.flag.shape)).astype(np.float32)
    sc.vx[:] = (0.02 * rng.standard_normal(sc.flag.shape)).astype(np.float32)
    out = []
    for variant in (0, 1, 2):
        with culbm.Simulation(dims, stream_policy=sp, inv_tau=0.55, storage=storage, kernel_variant=variant) as sim:
            sim.load_state(*sc.arrays())
            sim.step(9)
            out.append(sim.pulled_ddf())
    assert np.array_equal(bits(out[0]), bits(out[1]))
    assert np.array_equal(bits(out[0]), bits(out[2]))


def test_row_staged_wait_gives_up_and_reports(culbm):
    """A staged row whose mbarrier phase cannot complete (announced bytes that
    never arrive): the bounded wait gives up after about a second, the next
    synchronising call reports CULBM_ERR_DEVICE_TIMEOUT, and the device stays
    usable for the next run."""
    from culbm_b200 import _capi
    lib = _capi.lib()
    dims = (64, 8, 6)
    lib.culbm_debug_row_wait_extra_bytes(16)
    try:
        with culbm.Simulation(dims, stream_policy=0, storage="fp16", kernel_variant=1) as sim:
            sim.step(1)
            rc = lib.culbm_synchronize(sim._h)
            assert rc == 7, lib.culbm_last_error().decode()    # CULBM_ERR_DEVICE_TIMEOUT
            assert "bounded wait" in lib.culbm_last_error().decode()
    finally:
        lib.culbm_debug_row_wait_extra_bytes(0)
    with culbm.Simulation(dims, stream_policy=0, storage="fp16", kernel_variant=1) as sim:
        sim.step(2)
        sim.synchronize()
        assert np.isfinite(sim.pulled_ddf()).all()


WARP_DOMAINS = [(40, 5, 4), (56, 6, 5), (96, 7, 6), (8, 4, 3)]


@pytest.mark.parametrize("variant", [3, 4])
@pytest.mark.parametrize("storage", ["fp16", "bf16", "fp16sr", "bf16sr"])
@pytest.mark.parametrize("dims", WARP_DOMAINS)
def test_warp_staged_pull_matches_oracle(culbm, orc, storage, dims, variant):
    """The warp-staged 16-bit pull (kernel_variant 3 and 4, nx a multiple of 8):
    one and several 32-cell segments per row, a partial last segment, rows
    narrower than the 48-value window, fluid x faces (clamped pulls), solid
    cells without STORE, EQU rows."""
    sc = S.reference_channel(*dims, 0.05)
    sc.flag[:, :, 0] = S.FLUID
    sc.flag[:, :, -1] = S.FLUID
    rng = np.random.default_rng(sum(dims) + 3)
    solid = rng.random(sc.flag.shape) < 0.06
    sc.flag[solid] = 0
    for nsteps in (5, 6):
        want = oracle_pulled16(orc, sc, storage, 0.6, nsteps)
        with culbm.Simulation(sc.shape, stream_policy=0, inv_tau=0.6, storage=storage,
                              kernel_variant=variant) as sim:
            sim.load_state(*sc.arrays())
            sim.step(nsteps)
            got = sim.pulled_ddf()
        assert np.array_equal(bits(got), bits(want)), (storage, dims, nsteps)


@pytest.mark.parametrize("storage", ["fp16sr", "bf16"])
def test_warp_staged_pull_equals_per_cell_pull(culbm, storage):
    """kernel_variant 3, 4 and 0 give the same bits with random flags over
    many segments per warp."""
    dims = (168, 40, 36)
    sc = S.default_scene(*dims)
    rng = np.random.default_rng(23)
    pick = rng.random(sc.flag.shape)
    sc.flag[pick < 0.05] = S.WALL
    sc.flag[(pick >= 0.05) & (pick < 0.07)] = S.EQUILIBRIUM
    sc.flag[(pick >= 0.07) & (pick < 0.08)] = 0
    sc.rho[:] = (1 + 0.01 * rng.standard_normal(sc.flag.shape)).astype(np.float32)
    sc.vx[:] = (0.02 * rng.standard_normal(sc.flag.shape)).astype(np.float32)
    out = []
    for variant in (0, 3, 4):
        with culbm.Simulation(dims, stream_policy=0, inv_tau=0.55, storage=storage, kernel_variant=variant) as sim:
            sim.load_state(*sc.arrays())
            sim.step(9)
            out.append(sim.pulled_ddf())
    assert np.array_equal(bits(out[0]), bits(out[1]))
    assert np.array_equal(bits(out[0]), bits(out[2]))


def test_warp_staged_wait_gives_up_and_reports(culbm):
    """The warp-staged pull's bounded wait: a phase that cannot complete is
    reported as CULBM_ERR_DEVICE_TIMEOUT and the device stays usable."""
    from culbm_b200 import _capi
    lib = _capi.lib()
    dims = (64, 8, 6)
    lib.culbm_debug_row_wait_extra_bytes(16)
    try:
        with culbm.Simulation(dims, stream_policy=0, storage="fp16", kernel_variant=3) as sim:
            sim.step(1)
            rc = lib.culbm_synchronize(sim._h)
            assert rc == 7, lib.culbm_last_error().decode()
    finally:
        lib.culbm_debug_row_wait_extra_bytes(0)
    with culbm.Simulation(dims, stream_policy=0, storage="fp16", kernel_variant=3) as sim:
        sim.step(2)
        sim.synchronize()
        assert np.isfinite(sim.pulled_ddf()).all()

