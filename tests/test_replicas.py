"""The benchmark's multi-GPU plumbing (xkblas_b200/replicas.py) with two
ranks on CPU (gloo): barrier, maximum over ranks, the whole-job aggregate,
rank-0-only reporting, and the reference arm's non-zero ranks exiting
without work."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from xkblas_b200.replicas import Replicas
    r = Replicas(backend="gloo", timeout_s=60)
    r.barrier()
    seconds = 0.5 + rank  # rank 1 is the slowest
    value, slowest = r.aggregate(units_per_rank=1e12, seconds_per_rank=seconds)
    out.put((rank, r.leader, value, slowest, r.max(10 * rank)))
    r.close()


def test_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(i, world, port, q)) for i in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, lead0, v0, s0, m0), (r1, lead1, v1, s1, m1) = res
    assert lead0 and not lead1
    assert s0 == s1 == 1.5               # both ranks see the slowest rank's time
    assert v0 == v1 == 2 * 1e12 / 1.5    # all ranks' units over that time
    assert m0 == m1 == 10.0


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from xkblas_b200.replicas import Replicas
    r = Replicas(backend="gloo")
    assert r.world == 1 and r.leader and r.dist is None
    assert r.aggregate(3.0, 2.0) == (1.5, 2.0)
    r.close()


def test_reference_arm_only_rank0_works(capsys):
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=3)
    assert bench.run_reference(args, rank=1, world=2) is None
    assert capsys.readouterr().out == ""
