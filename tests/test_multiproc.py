"""Multi-process (gloo, world size 2) coverage of the column sharding used to
spread one step over several GPUs: each rank solves its shard (with the CPU
oracle standing in for the device), the shards are gathered, and the result
must equal the single-process solve column for column."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_shard_columns_cover_exactly_once(pkg):
    sc = pkg.batch.shard_columns
    ncols, weights = [10368, 333, 1, 700], [57, 56, 113, 114]
    for world in (1, 2, 3, 4, 8):
        seen = [np.zeros(n, int) for n in ncols]
        loads = []
        for r in range(world):
            load = 0
            for i, c0, c1 in sc(ncols, weights, world, r):
                seen[i][c0:c1] += 1
                load += (c1 - c0) * weights[i]
            loads.append(load)
        assert all(np.all(s == 1) for s in seen)
        assert max(loads) - min(loads) <= 2 * max(weights)


def test_aligned_shards_start_on_tiles(pkg):
    """With align=32 every cut inside a segment falls on a 32-column tile
    boundary; still every column exactly once and the loads balanced to
    within one aligned block of columns."""
    sc = pkg.batch.shard_columns
    ncols, weights = [10368, 6969, 2072, 333, 1], [57, 57, 114, 56, 113]
    for world in (1, 2, 3, 4, 8):
        seen = [np.zeros(n, int) for n in ncols]
        loads = []
        for r in range(world):
            load = 0
            for i, c0, c1 in sc(ncols, weights, world, r, align=32):
                assert c0 % 32 == 0 and (c1 % 32 == 0 or c1 == ncols[i])
                seen[i][c0:c1] += 1
                load += (c1 - c0) * weights[i]
            loads.append(load)
        assert all(np.all(s == 1) for s in seen)
        assert max(loads) - min(loads) <= 2 * 32 * max(weights)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import __graft_entry__ as ge
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pkg, orc = ge.load_package(), ge.load_oracle()
        systems = [pkg.synth.scalar_system(29, n, 0.5, 40 + n) for n in (700, 131, 64)]
        ncols = [s[0].shape[1] for s in systems]
        mine = pkg.batch.shard_columns(ncols, [29] * 3, world, rank)
        out = [np.zeros((29, n)) for n in ncols]
        for i, c0, c1 in mine:
            a, b, c, f = (np.asfortranarray(v[:, c0:c1]) for v in systems[i])
            out[i][:, c0:c1] = orc.trsolv_ng(a, b, c, f, 29)
        # combine the shards (each column is owned by exactly one rank)
        for i in range(3):
            t = torch.from_numpy(out[i])
            dist.all_reduce(t)
            out[i] = t.numpy()
        t_local = torch.tensor([float(rank + 1)])
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)  # max-over-ranks timing reduction
        if rank == 0:
            ok = all(np.array_equal(out[i], orc.trsolv_ng(*systems[i], 29)) for i in range(3))
            q.put((ok, float(t_local.item())))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_match_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    ok, tmax = q.get(timeout=5)
    assert ok and tmax == 2.0
