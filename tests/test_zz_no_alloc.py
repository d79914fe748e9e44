"""culbm_mass_momentum_noalloc: the FP64 mass/momentum reduction over a
caller-owned device population buffer, with its scratch in a fixed static
device array (no device allocation).  It serves callers that must not
allocate device memory themselves, such as a PyTorch process whose memory
belongs to the caching allocator (cudaMalloc would bypass it, and
cudaMalloc/cudaFree synchronise the device).  Collected last so that it also
runs after every other test has used the library on the same device."""
import ctypes as C

import numpy as np
import pytest

LIMIT = 77594624
INVALID = 1   # CULBM_ERR_INVALID_ARGUMENT


def _call(lib, ptr, n, out):
    return lib.culbm_mass_momentum_noalloc(C.c_void_p(ptr), C.c_uint64(n), None, out)


def test_rejects_sizes_beyond_the_limit(culbm):
    """Checked before the device is touched (no GPU needed)."""
    from culbm_b200 import _capi
    lib = _capi.lib()
    out = (C.c_double * 4)()
    assert _call(lib, 16, LIMIT + 1, out) == INVALID
    msg = lib.culbm_last_error().decode()
    assert "77594624" in msg and "exceed" in msg
    assert _call(lib, 0, 100, out) == INVALID
    assert _call(lib, 16, 0, out) == INVALID


@pytest.mark.gpu
def test_matches_the_sim_reduction_on_two_calls_in_a_row(culbm):
    """All-fluid flags, so the sim's LOAD|EQU mask keeps every cell and both
    entry points sum the same pulled populations (in a different order)."""
    import torch
    from culbm_b200 import _capi
    lib = _capi.lib()
    dims = (72, 40, 36)
    n = dims[0] * dims[1] * dims[2]
    rng = np.random.default_rng(11)
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    vx, vy, vz = (0.03 * rng.standard_normal((3, n))).astype(np.float32)
    with culbm.Simulation(dims, stream_policy=0, storage="fp32", inv_tau=0.6) as sim:
        sim.load_state(None, rho, vx, vy, vz)
        for _ in range(2):
            sim.step(3)
            ref = sim.mass_momentum()
            buf = torch.from_numpy(sim.pulled_ddf(np.float32)).to("cuda")
            torch.cuda.synchronize()
            got = (C.c_double * 4)()
            assert _call(lib, buf.data_ptr(), n, got) == 0, lib.culbm_last_error().decode()
            got = np.array(got[:])
            assert abs(got[0] - ref[0]) <= 1e-12 * abs(ref[0])
            assert np.allclose(got[1:], ref[1:], rtol=1e-10, atol=1e-9 * abs(ref[0]))
            again = (C.c_double * 4)()
            assert _call(lib, buf.data_ptr(), n, again) == 0
            assert np.array_equal(np.array(again[:]), got)


def _numpy_sums(pops):
    """FP64 mass and momentum of a (27, n) FP32 population array."""
    d = np.arange(27)
    c = np.stack([d % 3 - 1, (d // 3) % 3 - 1, d // 9 - 1]).astype(np.float64)
    p = pops.astype(np.float64)
    return np.array([p.shape[1] + p.sum(), *(c @ p.sum(axis=1))])


@pytest.mark.gpu
def test_caller_stream_and_a_smaller_call_after_a_larger_one(culbm):
    """The caller's own stream is honoured, and a call over fewer blocks
    after one over many reads none of the earlier call's partial sums."""
    import torch
    from culbm_b200 import _capi
    lib = _capi.lib()
    rng = np.random.default_rng(5)
    stream = torch.cuda.Stream()
    for n in (300_000, 1_000, 131_073):
        pops = (0.01 * rng.standard_normal((27, n))).astype(np.float32)
        with torch.cuda.stream(stream):
            buf = torch.from_numpy(pops.reshape(-1)).to("cuda", non_blocking=False)
        got = (C.c_double * 4)()
        rc = lib.culbm_mass_momentum_noalloc(C.c_void_p(buf.data_ptr()), C.c_uint64(n),
                                             C.c_void_p(stream.cuda_stream), got)
        assert rc == 0, lib.culbm_last_error().decode()
        want = _numpy_sums(pops)
        got = np.array(got[:])
        assert abs(got[0] - want[0]) <= 1e-12 * abs(want[0])
        assert np.allclose(got[1:], want[1:], rtol=1e-9, atol=1e-9 * abs(want[0]))
