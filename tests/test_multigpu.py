"""The multi-GPU owner-computes plan (xkblas_b200/multigpu.py) on CPU: the
GPU grid and tile owners against the reference's 2D block-cyclic formula
(blas/xkblas.c:2608-2626, :891), and the panel exchange with 2 and 4 gloo
ranks -- every rank ends with exactly the A row panels and B column panels
of its tiles, and the tiles computed from them assemble C = A B.  The local
contraction here is numpy (a stand-in for the device GEMM, which needs a
GPU per rank); the exchange is the code the GPU path runs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from xkblas_b200.multigpu import DistPlan, OwnerMap, grid_shape, tile_owner


def _ref_grid(n):
    """blas/xkblas.c:2608-2626, step by step."""
    gm = int(np.sqrt(n))
    gn = gm
    if gm == 0:
        return 1, n
    g = gm + 1
    while g > 0:
        if n % g == 0:
            break
        g -= 1
    return (n, 1) if g == 0 else (g, n // g)


@pytest.mark.parametrize("n", list(range(1, 17)) + [24, 32, 64])
def test_grid_shape_matches_reference(n):
    assert grid_shape(n) == _ref_grid(n)
    gm, gn = grid_shape(n)
    assert gm * gn == n


def test_known_grids():
    assert [grid_shape(n) for n in (1, 2, 3, 4, 6, 8, 9, 12, 16)] == \
        [(1, 1), (2, 1), (1, 3), (2, 2), (3, 2), (2, 4), (3, 3), (4, 3), (4, 4)]


@pytest.mark.parametrize("ngpus,mt,nt", [(1, 3, 4), (2, 5, 7), (4, 8, 8), (6, 7, 9), (8, 16, 16)])
def test_owner_map_is_block_cyclic_partition(ngpus, mt, nt):
    om = OwnerMap(mt, nt, ngpus)
    seen = np.zeros((mt, nt), int)
    for r in range(ngpus):
        tiles = om.tiles(r)
        for i, j in tiles:
            assert om.owner[i, j] == r == tile_owner(i, j, om.gm, om.gn)
            seen[i, j] += 1
        # the tiles of a rank are the cross product of its rows and columns
        assert sorted(tiles) == sorted((i, j) for i in om.row_panels(r) for j in om.col_panels(r))
    assert (seen == 1).all()
    counts = np.bincount(om.owner.ravel(), minlength=ngpus)
    if mt % om.gm == 0 and nt % om.gn == 0:
        assert counts.min() == counts.max()


def test_transfers_and_bytes():
    p = DistPlan(M=1000, N=700, K=300, nb=128, world=4)
    t = p.transfers()
    assert all(src != dst for _, _, src, dst in t)
    # every panel a rank needs and does not hold arrives exactly once
    for dst in range(4):
        got_a = sorted(i for k, i, _, d in t if k == "A" and d == dst)
        need_a = [i for i in p.map.row_panels(dst) if p.a_home[i] != dst]
        assert got_a == need_a
    assert p.bytes_moved() == sum(
        ((p.rows(i).stop - p.rows(i).start) if k == "A" else (p.cols(i).stop - p.cols(i).start))
        * 300 * 8 for k, i, _, _ in t)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, M, N, K, nb, out):
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(7)
        A = rng.uniform(-0.5, 0.5, (M, K))
        B = rng.uniform(-0.5, 0.5, (K, N))
        plan = DistPlan(M, N, K, nb, world)
        held_a = {i: torch.from_numpy(A[plan.rows(i)].copy())
                  for i in range(plan.mt) if plan.a_home[i] == rank}
        held_b = {j: torch.from_numpy(B[:, plan.cols(j)].copy())
                  for j in range(plan.nt) if plan.b_home[j] == rank}
        a, b = plan.exchange(rank, held_a, held_b)
        ok = sorted(a) == plan.map.row_panels(rank) and sorted(b) == plan.map.col_panels(rank)
        ok = ok and all(np.array_equal(a[i].numpy(), A[plan.rows(i)]) for i in a)
        ok = ok and all(np.array_equal(b[j].numpy(), B[:, plan.cols(j)]) for j in b)
        tiles = plan.compute(rank, a, b, lambda x, y: x @ y)
        gathered = [None] * world
        dist.all_gather_object(gathered, {k: v.numpy() for k, v in tiles.items()})
        if rank == 0:
            C = np.zeros((M, N))
            for part in gathered:
                for (i, j), t in part.items():
                    C[plan.rows(i), plan.cols(j)] = t
            err = float(np.abs(C - A @ B).max())
            out.put((rank, ok, err, sum(len(g) for g in gathered), plan.mt * plan.nt))
        else:
            out.put((rank, ok, 0.0, 0, 0))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_panel_exchange_gloo(world):
    M, N, K, nb = 520, 390, 200, 64
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, M, N, K, nb, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _, _, _ in res)
    _, _, err, ntiles, total = res[0]
    assert ntiles == total and err < 1e-12
