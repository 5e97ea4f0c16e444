"""World-size-2 process groups on the CPU (gloo): the multi-rank host logic.

Each rank takes its share of an ensemble (physgpu.dist.shard_systems), steps
it, and the shares are gathered and compared with the single-process result;
the per-rank compute here is the CPU oracle (test stand-in: no GPU in this
test), the plumbing is the product's.  Also checks max-over-ranks timing."""
import os
import socket

import numpy as np
import pytest

import oracle
import physgpu.dist as pd
import physgpu.ics as ics


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, pos, vel, m = ics.ensemble(40, seed=8)
        mine = pd.shard_systems(off, rank, world)
        sub, body = pd.subset_csr(off, mine)
        x, v, _ = oracle.ensemble_run(sub, pos[body], vel[body], m[body], 1.0, 1e-3, 1e-4, 5,
                                      nthreads=1)
        rows = np.concatenate([body[:, None].astype(np.float64), x, v], axis=1)
        every = pd.gather_rows(rows)
        t = pd.max_over_ranks(1.0 + rank)
        if rank == 0:
            q.put((np.concatenate(every), t))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_shards_cover_every_system_once_and_balance():
    off, _, _, _ = ics.ensemble(1000, seed=1)
    ns = np.diff(off)
    cost = ns * (ns - 1)
    parts = [pd.shard_systems(off, r, 4) for r in range(4)]
    allp = np.sort(np.concatenate(parts))
    assert np.array_equal(allp, np.arange(1000))
    loads = [cost[p].sum() for p in parts]
    assert max(loads) / min(loads) < 1.01


def test_two_rank_gloo_ensemble_matches_single_process():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        rows, t = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert t == 2.0  # max over ranks of (1 + rank)
    off, pos, vel, m = ics.ensemble(40, seed=8)
    x, v, _ = oracle.ensemble_run(off, pos, vel, m, 1.0, 1e-3, 1e-4, 5, nthreads=1)
    idx = rows[:, 0].astype(np.int64)
    assert np.array_equal(np.sort(idx), np.arange(len(m)))
    assert np.array_equal(rows[:, 1:4], x[idx]) and np.array_equal(rows[:, 4:7], v[idx])
