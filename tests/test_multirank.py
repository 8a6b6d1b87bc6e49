"""Multi-rank host logic on CPU: two gloo ranks shard the cells by
contiguous, group-aligned ranges, integrate them independently (the CPU
oracle stands in for the per-GPU solve here), take the MAX of their timings
and gather the ranges; the result equals one process solving all cells."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from odevec_b200 import dist as D


def test_cell_range_partitions():
    for n, w, a in [(4096, 2, 32), (4096, 3, 32), (1000, 7, 1), (96, 4, 32), (64, 8, 32)]:
        rs = [D.cell_range(n, r, w, a) for r in range(w)]
        assert rs[0][0] == 0 and rs[-1][1] == n
        for (a0, b0), (a1, b1) in zip(rs, rs[1:]):
            assert b0 == a1
        for s, e in rs:
            assert s % a == 0 and e % a == 0
        sizes = [e - s for s, e in rs]
        assert max(sizes) - min(sizes) <= a
    with pytest.raises(ValueError):
        D.cell_range(100, 0, 2, 32)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as O
    from odevec_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = W.rober(ncells=256)
        a, b = D.cell_range(wl.ncells, rank, world, wl.group)
        y, t, dt, st, _ = O.solve(wl.network, wl.y[:, a:b], wl.t0[a:b], wl.dt0[a:b], wl.t_stop[a:b],
                                  wl.rtol, wl.atol, wl.dt_min, group=wl.group, nthreads=1)
        elapsed = 0.5 + rank  # stand-in timings: the reduction must return the larger
        m = D.max_over_ranks(elapsed)
        full = D.gather_cells(y, wl.ncells, wl.group)
        stat = D.gather_cells(st[None, :].astype(np.int64), wl.ncells, wl.group)[0]
        if rank == 0:
            out.put((m, full, stat))
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one_process():
    from oracle import oracle as O
    from odevec_b200 import workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    m, full, stat = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert m == 1.5
    wl = W.rober(ncells=256)
    ref = O.solve(wl.network, wl.y, wl.t0, wl.dt0, wl.t_stop, wl.rtol, wl.atol, wl.dt_min, group=wl.group)
    assert np.array_equal(full, ref[0])
    assert np.all(stat == 0)
