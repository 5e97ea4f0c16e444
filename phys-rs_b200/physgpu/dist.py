"""Multi-process plumbing (one process per GPU, torch.distributed).

Three ways to use several GPUs:

* replicas: one independent system per rank, no collective;
* a batched ensemble split across ranks by system (shard_systems), no
  collective on the data path;
* one system split by targets (verlet_steps_shared): every rank holds the
  whole state and integrates every body, evaluates its share of the targets
  (phys_gravity_accel_share), and one all-gather of the shares'
  accelerations per evaluation (24 bytes per body, NCCL over NVLink)
  completes it.  The trajectory equals the one-GPU run bit for bit.

The rest is host logic: which systems a rank owns, the max-over-ranks timing
that the benchmark reports, and gathering per-rank results for checking.
"""
import numpy as np


def shard_systems(offsets, rank, world):
    """Systems owned by `rank` when the ensemble in CSR `offsets` is split
    over `world` ranks, balancing the O(N^2) pair work: longest systems first,
    each to the rank with the least work so far (ties to the lower rank).
    Returns the sorted system indices."""
    off = np.asarray(offsets, dtype=np.int64)
    ns = np.diff(off)
    cost = ns * np.maximum(ns - 1, 1)
    order = np.argsort(-cost, kind="stable")
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(ns), dtype=np.int64)
    for s in order:
        r = int(np.argmin(load))
        owner[s] = r
        load[r] += cost[s]
    return np.nonzero(owner == rank)[0]


def subset_csr(offsets, systems):
    """CSR offsets and body indices of a subset of systems."""
    off = np.asarray(offsets, dtype=np.int64)
    systems = np.asarray(systems, dtype=np.int64)
    sizes = off[systems + 1] - off[systems]
    sub = np.zeros(len(systems) + 1, dtype=np.int64)
    sub[1:] = np.cumsum(sizes)
    body = np.concatenate([np.arange(off[s], off[s + 1]) for s in systems]) if len(systems) \
        else np.zeros(0, dtype=np.int64)
    return sub, body


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (the benchmark's job time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(local, device=None):
    """All-gather a (k_r, c) float64 array whose row count differs per rank;
    returns the list of every rank's array (same on all ranks)."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local, dtype=np.float64)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [local]
    world = dist.get_world_size()
    cols = local.shape[1] if local.ndim == 2 else 1
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(counts, n)
    counts = [int(c.item()) for c in counts]
    cap = max(counts)
    buf = torch.zeros((cap, cols), dtype=torch.float64, device=device)
    buf[:local.shape[0]] = torch.from_numpy(local.reshape(-1, cols)).to(buf.device)
    outs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf)
    return [o[:c].cpu().numpy().reshape((c,) + local.shape[1:]) for o, c in zip(outs, counts)]


class SharedEvaluation:
    """The exchange of a target-shared force evaluation on one context.

    `ctx` is a physgpu.Context whose state every rank of `group` uploaded
    identically.  Buffers: this rank's block (3 * c float64) and the
    gathered blocks (world * 3 * c), c = physgpu.share_chunk(n, world), on
    the context's device.  The all-gather runs on the context's stream, so
    it is ordered after the share's kernels and before the scatter."""

    def __init__(self, ctx, group=None, device=None):
        import torch
        import torch.distributed as dist
        from . import share_chunk
        self.ctx = ctx
        self.group = group
        on = dist.is_available() and dist.is_initialized()
        self.world = dist.get_world_size(group) if on else 1
        self.rank = dist.get_rank(group) if on else 0
        self.chunk = share_chunk(ctx.n, self.world)
        self.device = torch.device(device) if device is not None else \
            torch.device("cuda", ctx.device)
        self.send = torch.zeros(3 * self.chunk, dtype=torch.float64, device=self.device)
        self.recv = torch.zeros(self.world * 3 * self.chunk, dtype=torch.float64,
                                device=self.device)
        self.stream = (torch.cuda.ExternalStream(ctx.stream, device=self.device)
                       if self.device.type == "cuda" else None)

    def evaluate(self, params):
        """a(x) of all bodies into the context, this rank computing its share."""
        import contextlib
        import torch
        import torch.distributed as dist
        self.ctx.gravity_accel_share(params, self.rank, self.world, self.send.data_ptr())
        scope = torch.cuda.stream(self.stream) if self.stream is not None \
            else contextlib.nullcontext()
        with scope:
            if self.world > 1:
                dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
            else:
                self.recv.copy_(self.send)
        self.ctx.gravity_accel_unshare(self.world, self.recv.data_ptr())


def verlet_steps_shared(ctx, params, dt, nsteps, group=None, exchange=None):
    """nsteps Velocity-Verlet ticks (phys_verlet_steps) of one system split by
    targets over the ranks of `group`: a(x_0), then per tick the position
    step, a shared evaluation and the velocity step, every rank integrating
    all bodies.  Returns the SharedEvaluation (reusable for more ticks)."""
    ex = exchange or SharedEvaluation(ctx, group)
    ex.evaluate(params)
    for _ in range(int(nsteps)):
        ctx.vv_position_step(dt)
        ex.evaluate(params)
        ctx.vv_velocity_step(dt)
    return ex
