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


# ---- one system split by targets (physgpu.dist.SharedEvaluation) ----------

class _FakeShareCtx:
    """Stand-in for physgpu.Context on the CPU (no GPU in this test): the same
    share / unshare / Verlet calls, computed with a plain f64 direct sum, so
    that the exchange's plumbing (chunking, all-gather, scatter, ordering)
    runs for real over gloo."""

    def __init__(self, pos, vel, m, eps=0.05):
        self.x, self.v, self.m = pos.copy(), vel.copy(), m.copy()
        self.a = np.zeros_like(pos)
        self.prev = np.zeros_like(pos)
        self.n, self.device, self.stream, self.eps = len(m), 0, None, eps

    def _accel(self, i):
        r = self.x - self.x[i]
        s2 = np.einsum("ij,ij->i", r, r) + self.eps ** 2
        w = self.m / (s2 * np.sqrt(s2))
        w[i] = 0.0
        return (r * w[:, None]).sum(axis=0)

    @staticmethod
    def _view(ptr, count):
        import ctypes
        return np.ctypeslib.as_array((ctypes.c_double * count).from_address(ptr))

    def gravity_accel_share(self, params, rank, world, ptr):
        import physgpu
        c = physgpu.share_chunk(self.n, world)
        lo, hi = min(self.n, rank * c), min(self.n, (rank + 1) * c)
        out = self._view(ptr, 3 * c)
        out[:] = 0.0
        for i in range(lo, hi):
            a = self._accel(i)
            for k in range(3):
                out[k * c + i - lo] = a[k]

    def gravity_accel_unshare(self, world, ptr):
        import physgpu
        c = physgpu.share_chunk(self.n, world)
        g = self._view(ptr, world * 3 * c)
        for i in range(self.n):
            r, j = divmod(i, c)
            self.a[i] = [g[r * 3 * c + k * c + j] for k in range(3)]

    def vv_position_step(self, dt):
        self.prev = self.a.copy()
        self.x = self.x + (self.v * dt + self.a * (0.5 * dt * dt))

    def vv_velocity_step(self, dt):
        self.v = self.v + (self.prev + self.a) * (0.5 * dt)


def _share_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pos, vel, m = ics.plummer(300, seed=3)
        fake = _FakeShareCtx(pos, vel, m)
        ex = pd.SharedEvaluation(fake, device="cpu")
        assert (ex.rank, ex.world) == (rank, world)
        pd.verlet_steps_shared(fake, None, 1e-3, 4, exchange=ex)
        q.put((rank, fake.x, fake.v, fake.a))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_gloo_target_shares_match_single_process():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_share_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = dict((r, (x, v, a)) for r, x, v, a in (q.get(timeout=120) for _ in range(2)))
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    pos, vel, m = ics.plummer(300, seed=3)
    ref = _FakeShareCtx(pos, vel, m)
    pd.verlet_steps_shared(ref, None, 1e-3, 4, exchange=pd.SharedEvaluation(ref, device="cpu"))
    for r in range(2):  # every rank holds the whole, identical state
        for got_k, want in zip(got[r], (ref.x, ref.v, ref.a)):
            assert np.array_equal(got_k, want)


def test_share_chunk_rule():
    import physgpu
    assert physgpu.share_chunk(1000, 3) == 384  # ceil(1000 / 3) = 334 -> 3 tiles of 128
    assert physgpu.share_chunk(1 << 20, 8) == 131072
    assert physgpu.share_chunk(5, 1) == 128
    assert physgpu.share_chunk(10, 0) == -1 and physgpu.share_chunk(-1, 2) == -1
