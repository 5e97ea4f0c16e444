"""Multi-process plumbing (one process per GPU, torch.distributed).

The gravity path has no exchange step that would need a collective on the
data path: Barnes-Hut runs one independent system per rank (replicas), and a
batched ensemble splits its independent systems across ranks.  What is
shared is host logic: which systems a rank owns, the max-over-ranks timing
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
