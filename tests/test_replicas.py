"""Multi-GPU mode of bench.py is replicas only: every rank runs its own box (seed 1234 + rank)
and the job's time is the slowest rank's.  The rank logic runs here as two gloo processes on
the CPU (no GPU, no data-path collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    per_rank_ms = [0.50, 0.62][rank]
    got = bench.max_over_ranks(per_rank_ms, dist, "cpu")
    # a second collective in the same order on every rank (as the bench's legs do)
    got2 = bench.max_over_ranks(10.0 + rank, dist, "cpu")
    value = world * bench.ns_per_day(got)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, got2, value))


def test_slowest_rank_sets_the_job_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import bench
    for rank, got, got2, value in out:
        assert got == pytest.approx(0.62) and got2 == pytest.approx(11.0)
        assert value == pytest.approx(2 * bench.ns_per_day(0.62))


def test_replica_workloads_differ_by_rank():
    import numpy as np

    from protomol3_b200 import waterbox as W
    a, b = W.water_box(64, seed=1234), W.water_box(64, seed=1235)
    assert a["pos"].shape == b["pos"].shape and not np.allclose(a["pos"], b["pos"])
