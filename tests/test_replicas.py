"""The multi-GPU form of the benchmark is N independent replicas (one per
rank, no data-path exchange): the host-side plumbing it uses - process group,
barrier, max over ranks of the device time, whole-job aggregate - run here as
two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench
    got_ws, got_rank = bench.dist()
    tdist = bench.dist_init(got_ws)
    bench.barrier(tdist)
    ms = 100.0 + 50.0 * rank          # rank 1 is the slower replica
    ms_max = bench.max_over_ranks(tdist, ms)
    value = bench.aggregate_mlups(got_ws, 1_000_000, 10, ms_max)
    bench.barrier(tdist)
    tdist.destroy_process_group()
    out.put((got_rank, got_ws, ms_max, value))


def test_two_replicas_report_the_slowest_rank_and_the_whole_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ws, ms_max, value in res:
        assert ws == 2 and ms_max == 150.0
        # two replicas of 1e6 cells x 10 steps in 150 ms
        assert value == pytest.approx(2 * 1e6 * 10 / 0.150 / 1e6)


def test_single_process_needs_no_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init(1) is None
    assert bench.max_over_ranks(None, 3.5) == 3.5
    assert bench.aggregate_mlups(1, 2_000_000, 5, 10.0) == pytest.approx(1000.0)
