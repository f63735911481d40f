"""The bench's multi-rank path on CPU: two gloo ranks, as torchrun launches one rank per GPU.
Replicas over independent atoms (each rank its own seed, no data-path collective); the only
collectives are the barrier and the max of the per-rank times, which the whole-job rate uses."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from lsms_b200 import workloads as W
        ms = 10.0 + 5.0 * rank                      # this rank's time per step
        dist.barrier()
        ms_max = bench.rank_max(ms, dist, "cpu")
        rate = bench.whole_job_rate(31, world, ms_max)
        # the replicas solve different atoms: the bench seeds rank r's atom with 2 + r
        prob = W.config_n2160(seed=2 + rank, npts=2)
        q.put((rank, ms_max, rate, float(abs(prob.tmat_store).sum())))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_report_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]      # every rank reports the slowest rank's time
    assert all(abs(o[2] - 2 * 31 / 15e-3) < 1e-9 for o in out)
    assert out[0][3] != out[1][3]                   # independent atoms per rank


def test_single_rank_is_its_own_max():
    import bench
    assert bench.rank_max(12.5) == 12.5
    assert bench.whole_job_rate(31, 1, 15.0) == pytest.approx(31 / 15e-3)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun the reference arm's rank 0 alone runs and prints; the others exit at once."""
    import bench
    assert bench.run_reference(None, 2, 1) is None
    assert capsys.readouterr().out == ""
