"""The N > 1 host logic of bench.py on CPU: two gloo ranks (replicas only, no data-path
collective) agree on the job time as the slowest rank's and on the whole-job rate; the
reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    secs = bench.max_over_ranks(1.0 + rank, dist, device="cpu")     # rank r took 1 + r seconds
    rate = bench.job_rate(world, 40, 10, secs)

    class Args:
        steps, warmup, gpus = 1, 0, world
    ref = bench.run_reference(Args, rank) if rank != 0 else "skipped"
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, secs, rate, ref))


def test_two_gloo_ranks_agree_on_the_slowest_replica():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, secs, rate, ref in got:
        assert secs == pytest.approx(2.0)                  # the slower rank's time on every rank
        assert rate == pytest.approx(2 * 40 * 10 / 2.0)   # both replicas' sites over that time
        if rank != 0:
            assert ref is None                             # the reference arm: rank 0 only


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.job_rate(1, 40, 10, 2.0) == 200.0
