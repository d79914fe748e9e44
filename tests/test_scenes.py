"""Scene generators and the init-state / dump file format (CPU only)."""
import numpy as np

from culbm_b200 import scenes as S


def test_reference_channel_matches_notebook_layout():
    s = S.reference_channel(12, 10, 8, 0.05)
    f = s.flag
    assert (f[1:-1, 1:-1, 1:-1] == S.FLUID).all()
    assert (f[:, 0, :] == S.WALL).all() and (f[:, -1, :] == S.WALL).all()
    assert (f[0, 1:-1, :] == S.WALL).all() and (f[-1, 1:-1, :] == S.WALL).all()
    assert (f[1:-1, 1:-1, 0] == S.EQUILIBRIUM).all() and (f[1:-1, 1:-1, -1] == S.EQUILIBRIUM).all()
    assert (s.vx[1:-1, 1:-1, 0] == np.float32(0.05)).all()
    assert s.vx[1:-1, 1:-1, 1:].sum() == 0


def test_correctness_case_layout():
    s = S.correctness_case(40, 24, 20, cube=(8, 8, 8, 16, 16, 16))
    f = s.flag
    assert (f[8:16, 8:16, 8:16] == S.WALL).all()
    assert (f[:, (0, -1), :] == S.WALL).all() and (f[(0, -1), :, :] == S.WALL).all()
    assert (f[1:-1, 1:-1, 0] == S.EQUILIBRIUM).all()
    assert (s.vx[1:-1, 1:-1, 0] == np.float32(0.05)).all()
    assert (s.vx[:, 0, :] == 0).all()


def test_sphere_64_config():
    s = S.sphere_64()
    assert s.shape == (64, 64, 64)
    assert s.flag[32, 32, 16] == S.WALL          # sphere centre (z, y, x)
    assert s.flag[32, 32, 30] == S.FLUID
    assert np.isclose(s.vx[32, 32, 0], 0.02)
    assert (s.rho == 1).all()
    assert s.flag[32, 32, 63] == S.EQUILIBRIUM and s.vx[32, 32, 63] == 0


def test_seeded_spheres_are_reproducible():
    a = S.spheres_512(scale=0.125)
    b = S.spheres_512(scale=0.125)
    assert np.array_equal(a.flag, b.flag)
    assert a.shape == (64, 64, 32)
    assert 0.0 < a.solid_fraction() < 0.6


def test_folder_round_trip(tmp_path):
    s = S.reference_channel_cube(24, 20, 16, 0.04)
    S.write_folder(s, str(tmp_path))
    t = S.read_folder(str(tmp_path), 24, 20, 16)
    for k in ("flag", "rho", "vx", "vy", "vz"):
        assert np.array_equal(getattr(s, k), getattr(t, k)), k
    raw = np.fromfile(tmp_path / "flag.dat", dtype="<u4")
    assert raw.size == 24 * 20 * 16 and raw[0] == S.WALL


def test_soft_field_range():
    s, soft = S.adjoint_channel(32, 16, 16, bumps=4)
    assert soft.shape == (16, 16, 32)
    assert soft.min() >= 0 and soft.max() <= 1 and soft.max() > 0.1
    assert (soft[s.flag != S.FLUID] == 0).all()


def test_scene_cli_writes_a_folder_the_solver_reads(tmp_path):
    from culbm_b200 import scenes as S
    out = tmp_path / "case"
    assert S.main(["spheres", str(out), "--domain", "48", "40", "36", "--spheres", "4", "--radii", "3", "5",
                   "--seed", "9"]) == 0
    got = S.read_folder(str(out), 48, 40, 36)
    c, r = S.random_spheres(48, 40, 36, 4, 3.0, 5.0, 9)
    ref = S.sphere_channel(48, 40, 36, 0.05, c, r)
    for name in ("flag", "rho", "vx", "vy", "vz"):
        assert np.array_equal(getattr(got, name), getattr(ref, name)), name
    adj = tmp_path / "adj"
    assert S.main(["adjoint-channel", str(adj), "--domain", "32", "16", "16", "--u-in", "0.04", "--seed", "7"]) == 0
    soft = np.fromfile(adj / "soft.dat", dtype="<f4")
    _, ref_soft = S.adjoint_channel(32, 16, 16, u_peak=0.04, bumps=16, seed=7)
    assert np.array_equal(soft, ref_soft.reshape(-1).astype(np.float32))
