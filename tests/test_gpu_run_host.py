"""culbm_run_host: one run from host arrays to host fields with the copies
overlapping the steps (GPU).

The call must give the bits of culbm_load_state + culbm_step + culbm_moments +
culbm_get_field, whose results the parity tests pin to the oracle.  The tests
ask for 16 slabs (run_slabs), which the library caps at nz/2 so that every
slab keeps two planes: the domains below cover one, two, four and sixteen
slabs, thin and uneven slabs, runs shorter and longer than two skewed phases
(2 x slabs steps; longer runs take whole-domain steps in between), both stream
policies, odd and even step counts (the in-place layout at the end differs),
16-bit and FP64 storage, default inputs, page-locked buffers, repeated calls,
the automatic slab count, and the configurations that run the calls in
sequence.
"""
import numpy as np
import pytest

from culbm_b200 import scenes as S

pytestmark = pytest.mark.gpu


def scene(dims):
    nx, ny, nz = dims
    r = max(1.0, min(nx, ny, nz) / 4)
    return S.sphere_channel(nx, ny, nz, 0.05, [(nx / 2, ny / 2, nz / 2)], [r])


def sequential(culbm, dims, arrs, nsteps, **kw):
    with culbm.Simulation(dims, inv_tau=0.6, **kw) as sim:
        sim.load_state(*arrs)
        sim.step(nsteps)
        sim.moments()
        return sim.fields()


def overlapped(culbm, dims, arrs, nsteps, run_slabs=16, **kw):
    with culbm.Simulation(dims, inv_tau=0.6, run_slabs=run_slabs, **kw) as sim:
        out = sim.run_host(nsteps, *arrs)
        assert sim.step_count == nsteps
        return out


def assert_fields_equal(got, want, what):
    for name, g, w in zip(("rho", "vx", "vy", "vz"), got, want):
        gb, wb = g.view(np.uint32), w.view(np.uint32)
        if not np.array_equal(gb, wb):
            bad = np.flatnonzero(gb != wb)
            raise AssertionError(f"{what} {name}: {bad.size} of {gb.size} values differ, first at {bad[:5]}")


DOMAINS = [(19, 13, 1), (21, 9, 3), (33, 17, 5), (16, 8, 9), (40, 12, 37), (24, 10, 40)]


@pytest.mark.parametrize("dims", DOMAINS)
@pytest.mark.parametrize("sp", [0, 1])
@pytest.mark.parametrize("nsteps", [7, 8, 41])
def test_run_host_equals_sequential_fp32(culbm, dims, sp, nsteps):
    arrs = scene(dims).arrays()
    want = sequential(culbm, dims, arrs, nsteps, stream_policy=sp)
    got = overlapped(culbm, dims, arrs, nsteps, stream_policy=sp)
    assert_fields_equal(got, want, f"{dims} sp={sp} steps={nsteps}")


@pytest.mark.parametrize("storage", ["fp16sr", "bf16", "fp64"])
@pytest.mark.parametrize("sp", [0, 1])
def test_run_host_equals_sequential_other_storage(culbm, storage, sp):
    dims = (40, 12, 37)
    arrs = scene(dims).arrays()
    want = sequential(culbm, dims, arrs, 9, stream_policy=sp, storage=storage)
    got = overlapped(culbm, dims, arrs, 9, stream_policy=sp, storage=storage)
    assert_fields_equal(got, want, f"{storage} sp={sp}")


@pytest.mark.parametrize("sp", [0, 1])
def test_run_host_default_inputs_and_zero_steps(culbm, sp):
    dims = (24, 10, 40)
    for nsteps in (0, 3):
        want = sequential(culbm, dims, [None] * 5, nsteps, stream_policy=sp)
        got = overlapped(culbm, dims, [None] * 5, nsteps, stream_policy=sp)
        assert_fields_equal(got, want, f"defaults sp={sp} steps={nsteps}")
    # Only the flags given: rho and u take their defaults.
    f = scene(dims).arrays()[0]
    want = sequential(culbm, dims, [f, None, None, None, None], 5, stream_policy=sp)
    got = overlapped(culbm, dims, [f, None, None, None, None], 5, stream_policy=sp)
    assert_fields_equal(got, want, f"flags only sp={sp}")


def test_run_host_page_locked_buffers_and_repeat(culbm):
    import torch

    dims = (48, 20, 44)
    arrs = scene(dims).arrays()
    n = dims[0] * dims[1] * dims[2]
    pinned_in = []
    for a in arrs:
        t = torch.empty(n, dtype=torch.int32 if a.dtype == np.uint32 else torch.float32, pin_memory=True)
        v = t.numpy().view(a.dtype)
        v[:] = a.reshape(-1)
        pinned_in.append((t, v))
    pinned_out = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(4)]
    outs = tuple(t.numpy() for t in pinned_out)
    want = sequential(culbm, dims, arrs, 11, stream_policy=1)
    with culbm.Simulation(dims, stream_policy=1, inv_tau=0.6, run_slabs=16) as sim:
        for _ in range(2):
            for o in outs:
                o[:] = np.nan
            sim.run_host(11, *[v for _, v in pinned_in], out=outs)
            assert_fields_equal(outs, want, "page-locked")
        # The simulation carries on from the run like after the four calls.
        sim.step(3)
        sim.moments()
        cont = sim.fields()
    with culbm.Simulation(dims, stream_policy=1, inv_tau=0.6) as ref:
        ref.load_state(*arrs)
        ref.step(14)
        ref.moments()
        assert_fields_equal(cont, ref.fields(), "continued after the run")


@pytest.mark.parametrize("run_slabs", [0, 5, 32])
@pytest.mark.parametrize("nsteps", [12, 45])
def test_run_host_slab_counts(culbm, run_slabs, nsteps):
    """The automatic count (5 slabs for 12 steps, 2 for 45 here) and explicit ones."""
    dims = (128, 64, 160)
    arrs = scene(dims).arrays()
    for sp in (0, 1):
        want = sequential(culbm, dims, arrs, nsteps, stream_policy=sp)
        got = overlapped(culbm, dims, arrs, nsteps, run_slabs=run_slabs, stream_policy=sp)
        assert_fields_equal(got, want, f"run_slabs={run_slabs} sp={sp} steps={nsteps}")


def test_run_host_sequential_configurations(culbm):
    """The tile engine and the staged 16-bit kernels run the four calls in order."""
    for dims, kw in (((37, 29, 23), dict(stream_policy=1, opt_policy=3, inner_loop=3, tile=(16, 12, 10))),
                     ((32, 12, 20), dict(stream_policy=0, storage="fp16sr", kernel_variant=1))):
        arrs = scene(dims).arrays()
        want = sequential(culbm, dims, arrs, 6, **kw)
        got = overlapped(culbm, dims, arrs, 6, **kw)
        assert_fields_equal(got, want, str(kw))


def test_run_host_rejects_null_outputs(culbm):
    import ctypes as C

    from culbm_b200 import _capi
    with culbm.Simulation((8, 8, 8)) as sim:
        out = np.empty(512, np.float32)
        p = out.ctypes.data_as(C.c_void_p)
        st = _capi.lib().culbm_run_host(sim._h, None, None, None, None, None, 1, p, p, None, p)
        assert _capi.STATUS_NAMES[st] == "CULBM_ERR_INVALID_ARGUMENT"
