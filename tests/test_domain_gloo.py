"""Host logic of the row-slab decomposition on CPU: partitioning, the halo
exchange and the totals combine of DistExchange over gloo (world size 2 and 3),
against a single global array."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mantlepar_b200.domain import DistExchange, combine_totals, partition

NX, NY = 7, 11


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _layout(rows, ny):
    b, e = rows
    hb, ht = min(2, b), min(2, ny - e)
    return b - hb, hb, hb + (e - b), (e - b) + hb + ht   # row0, own0, own1, local_rows


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rows = partition(NY, world)
        g = np.arange(NX * NY, dtype=np.float64).reshape(NY, NX)
        row0, own0, own1, lr = _layout(rows[rank], NY)
        loc = np.full((lr, NX), np.nan)
        loc[own0:own1] = g[rows[rank][0]:rows[rank][1]]
        H = torch.from_numpy(loc.ravel().copy())
        C = torch.from_numpy(-loc.ravel().copy())
        ex = DistExchange(rank, world, rows, NX)
        ex.exchange(H, C, row0, own0, own1, lr)
        okH = np.array_equal(H.numpy().reshape(lr, NX), g[row0:row0 + lr])
        okC = np.array_equal(C.numpy().reshape(lr, NX), -g[row0:row0 + lr])
        # totals: maxRate, divergence, bH, bC, HI, CI, Hmin, Cmin, Cmax, nonfinite
        tot = np.array([rank + 1.0, 0.5 * rank, 1.0, 2.0, 10.0 * (rank + 1), 3.0, -rank, 5.0 - rank, rank, 0.0, 0.25 * rank])
        st = [(rank << 8) | 63 if rank == world - 1 else (1 << 64) - 1]
        ex.combine(tot, st)
        q.put((rank, okH, okC, tot.tolist(), st[0]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_dist_exchange_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = [np.array([r + 1.0, 0.5 * r, 1.0, 2.0, 10.0 * (r + 1), 3.0, -r, 5.0 - r, r, 0.0, 0.25 * r]) for r in range(world)]
    want, _ = combine_totals(parts, [0] * world)
    for rank, okH, okC, tot, st in res:
        assert okH and okC, rank
        assert np.allclose(tot, want)
        assert st == (((world - 1) << 8) | 63)


def test_partition_and_combine():
    assert partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert all(e - b >= 2 for b, e in partition(2560, 8))
    with pytest.raises(ValueError):
        partition(5, 3)
    a = np.array([1.0, 2, 3, 4, 5, 6, 7, 8, 9, 0, 0.5])
    b = np.array([2.0, 1, 3, 4, 5, 6, 6, 9, 8, 1, 0.25])
    tot, st = combine_totals([a, b], [5, 3])
    assert tot.tolist() == [2, 2, 6, 8, 10, 12, 6, 8, 9, 1, 0.75] and st == 3
