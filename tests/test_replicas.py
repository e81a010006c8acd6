"""Host logic of multi-GPU runs (replicas only: each rank evolves its own
realisation, no data exchange), checked with two gloo ranks on the CPU:
the replica seeds differ, the step time is the maximum over ranks, and the
whole-job rate counts every rank's particles over that maximum."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world)
    try:
        w, r, _ = bench.setup_dist()
        own_ms = 10.0 + 5.0 * r          # rank 1 is the slower replica
        slowest = bench.max_over_ranks(own_ms, device="cpu")
        rate = bench.whole_job_rate(w, 1000, 4, slowest)
        q.put((r, w, bench.replica_seed(7, r), slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert out[0][2] != out[1][2]
    assert all(o[3] == pytest.approx(15.0) for o in out)
    assert all(o[4] == pytest.approx(2 * 1000 * 4 / 15e-3) for o in out)
