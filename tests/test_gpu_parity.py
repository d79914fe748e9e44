"""Parity of the CUDA path against the oracle (GPU).

Every comparison goes through the C ABI (libculbm.so).  FP32 and FP64 are
bit-exact against the oracle, which is itself pinned bitwise to the
reference's lbm_core routines (tests/test_oracle.py).
"""
import os

import numpy as np
import pytest

from culbm_b200 import scenes as S

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def assert_bitwise(got, want, what=""):
    gb, wb = bits(got), bits(want)
    if not np.array_equal(gb, wb):
        bad = np.flatnonzero(gb != wb)
        raise AssertionError(f"{what}: {bad.size} of {gb.size} values differ; first at {bad[:5]}: "
                             f"{np.asarray(got).reshape(-1)[bad[:5]]} vs {np.asarray(want).reshape(-1)[bad[:5]]}")


def oracle_scene(orc, scene):
    f, r, ux, uy, uz = scene.arrays()
    nx, ny, nz = scene.shape
    return orc.Scene(nx, ny, nz, f, r, ux, uy, uz)


PLAIN = [(0, 0), (1, 0)]


def make_sim(culbm, dims, policy, storage="fp32", inv_tau=0.5, **kw):
    sp, op = policy
    return culbm.Simulation(dims, stream_policy=sp, opt_policy=op, inv_tau=inv_tau, storage=storage, **kw)


@pytest.mark.parametrize("policy", PLAIN)
@pytest.mark.parametrize("name", ["random_13x11x9.npz", "channel_16x12x10.npz", "stream_9x7x5.npz"])
def test_golden_fixtures_bitwise(culbm, name, policy):
    g = np.load(os.path.join(GOLDEN, name))
    dims = (int(g["nx"]), int(g["ny"]), int(g["nz"]))
    with make_sim(culbm, dims, policy, inv_tau=float(g["inv_tau"])) as sim:
        sim.load_state(g["flag"], g["rho"], g["vx"], g["vy"], g["vz"])
        sim.set_ddf(g["state0"])
        sim.step(int(g["nsteps"]))
        assert_bitwise(sim.pulled_ddf(), g["pulled"], "pulled populations")
        sim.moments()
        for k, key in zip(("rho", "vx", "vy", "vz"), ("d_rho", "d_vx", "d_vy", "d_vz")):
            assert_bitwise(sim.field(k), g[key], key)


@pytest.mark.parametrize("policy", PLAIN)
@pytest.mark.parametrize("nsteps", [1, 2, 7, 8])
def test_default_flags_clamped_edges_bitwise(culbm, orc, policy, nsteps):
    """No init folder: fluid everywhere, so every boundary cell pulls through
    the clamped edge (the case the in-place edge buffer exists for)."""
    dims = (19, 14, 11)
    sc = S.default_scene(*dims)
    rng = np.random.default_rng(nsteps)
    state0 = (0.01 * rng.standard_normal(27 * sc.n)).astype(np.float32)
    o = oracle_scene(orc, sc)
    want = orc.run(o, 0.7, nsteps, state=state0)
    with make_sim(culbm, dims, policy, inv_tau=0.7) as sim:
        sim.load_state(*sc.arrays())
        sim.set_ddf(state0)
        sim.step(nsteps)
        assert_bitwise(sim.pulled_ddf(), orc.pulled(o, want), "pulled")


@pytest.mark.parametrize("policy", PLAIN)
def test_sphere_64_200_steps_bitwise(culbm, orc, policy):
    """64^3 channel with one sphere, 200 steps from rest (the 64^3 workload)."""
    sc = S.sphere_64()
    o = oracle_scene(orc, sc)
    want = orc.run(o, 0.5, 200)
    with make_sim(culbm, sc.shape, policy) as sim:
        sim.load_state(*sc.arrays())
        sim.step(200)
        assert_bitwise(sim.pulled_ddf(), orc.pulled(o, want), "pulled")
        sim.moments()
        wm = orc.moments(o, want)
        for k, w in zip(("rho", "vx", "vy", "vz"), wm):
            assert_bitwise(sim.field(k), w, k)


@pytest.mark.parametrize("policy", PLAIN)
def test_fp64_storage_matches_fp64_oracle(culbm, orc, policy):
    g = np.load(os.path.join(GOLDEN, "random_13x11x9.npz"))
    dims = (int(g["nx"]), int(g["ny"]), int(g["nz"]))
    o = orc.Scene(*dims, g["flag"], g["rho"], g["vx"], g["vy"], g["vz"])
    state0 = g["state0"].astype(np.float64)
    want = orc.run(o, float(g["inv_tau"]), 11, dtype=np.float64, state=state0)
    with make_sim(culbm, dims, policy, storage="fp64", inv_tau=float(g["inv_tau"])) as sim:
        sim.load_state(g["flag"], g["rho"], g["vx"], g["vy"], g["vz"])
        sim.set_ddf(state0)
        sim.step(11)
        assert_bitwise(sim.pulled_ddf(np.float64), orc.pulled(o, want), "pulled fp64")


def test_streaming_is_a_permutation(culbm, orc):
    """LOAD|STORE only: the step is pure data movement; index payload comes
    back at the pulled positions bit for bit, in both streaming policies."""
    dims = (33, 9, 6)
    n = dims[0] * dims[1] * dims[2]
    flag = np.full(n, S.LOAD | S.STORE | S.DUMP_ALL, np.uint32)
    payload = (np.arange(27 * n) % 8191).astype(np.float32)
    o = orc.Scene(*dims, flag)
    for nsteps in (1, 4, 5):
        want = orc.pulled(o, orc.run(o, 0.5, nsteps, state=payload))
        for policy in PLAIN:
            with make_sim(culbm, dims, policy) as sim:
                sim.load_state(flag)
                sim.set_ddf(payload)
                sim.step(nsteps)
                assert_bitwise(sim.pulled_ddf(), want, f"policy {policy} steps {nsteps}")


def test_step_counter_and_split_steps(culbm, orc):
    """step(3)+step(4) == step(7), and the counter follows."""
    sc = S.reference_channel(20, 12, 10, 0.05)
    outs = []
    for split in ((7,), (3, 4), (1, 1, 5)):
        with make_sim(culbm, sc.shape, (1, 0)) as sim:
            sim.load_state(*sc.arrays())
            for k in split:
                sim.step(k)
            assert sim.step_count == 7
            outs.append(sim.pulled_ddf())
    assert_bitwise(outs[1], outs[0], "3+4")
    assert_bitwise(outs[2], outs[0], "1+1+5")


def test_mass_momentum_fp64(culbm, orc):
    sc = S.reference_channel(24, 14, 12, 0.05)
    o = oracle_scene(orc, sc)
    want = orc.pulled(o, orc.run(o, 0.5, 40)).astype(np.float64).reshape(27, -1)
    active = (sc.flag.reshape(-1) & (S.LOAD | S.EQU)) != 0
    d = np.arange(27)
    cx, cy, cz = d % 3 - 1, (d // 3) % 3 - 1, d // 9 - 1
    ref = np.array([np.sum(1.0 + want[:, active].sum(0)), (cx[:, None] * want[:, active]).sum(),
                    (cy[:, None] * want[:, active]).sum(), (cz[:, None] * want[:, active]).sum()])
    for policy in PLAIN:
        with make_sim(culbm, sc.shape, policy) as sim:
            sim.load_state(*sc.arrays())
            sim.step(40)
            got = sim.mass_momentum()
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-9), (got, ref)


def test_dump_files_layout(culbm, orc, tmp_path):
    sc = S.reference_channel(16, 10, 8, 0.05)
    o = oracle_scene(orc, sc)
    want = orc.moments(o, orc.run(o, 0.5, 12))
    with make_sim(culbm, sc.shape, (0, 0)) as sim:
        sim.load_state(*sc.arrays())
        sim.step(12)
        sim.moments()
        sim.dump(str(tmp_path), rho=True, vx=True, vz=True)
    for k, w in zip(("rho", "vx", "vy", "vz"), want):
        p = tmp_path / f"{k}_12.dat"
        if k == "vy":
            assert not p.exists()
            continue
        assert_bitwise(np.fromfile(p, dtype="<f4"), w, k)


@pytest.mark.parametrize("dims", [(1, 5, 4), (5, 1, 4), (5, 4, 1), (2, 2, 2), (3, 2, 5), (7, 3, 2), (33, 3, 3),
                                  (40, 6, 5)])
def test_degenerate_domains_bitwise(culbm, orc, dims):
    """Thin domains: every row set, x-face and clamp combination of the
    in-place kernels, against the oracle's pull with the per-axis clamp."""
    sc = S.default_scene(*dims)
    rng = np.random.default_rng(sum(dims))
    state0 = (0.01 * rng.standard_normal(27 * sc.n)).astype(np.float32)
    o = oracle_scene(orc, sc)
    for nsteps in (1, 2, 5):
        want = orc.pulled(o, orc.run(o, 0.8, nsteps, state=state0))
        for policy in PLAIN:
            with make_sim(culbm, dims, policy, inv_tau=0.8) as sim:
                sim.load_state(*sc.arrays())
                sim.set_ddf(state0)
                sim.step(nsteps)
                assert_bitwise(sim.pulled_ddf(), want, f"{dims} {policy} {nsteps}")
