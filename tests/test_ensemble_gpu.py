"""Batched ensemble (K8) parity through the C ABI.

Bar: F64_EXACT is bit-identical to the oracle's per-system reference tick
loop for every group size and chunking; F32C stays within 1e-9 relative of
F64_EXACT positions over a short run (chaotic systems diverge later)."""
import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import F32C, F64_EXACT, make_params

pytestmark = pytest.mark.gpu


def small_ensemble(nsys, seed):
    off, pos, vel, m = ics.ensemble(nsys, seed=seed)
    return off, pos, vel, m


def edge_ensemble():
    """Systems of 1, 2, 3, 8, 9, 16, 17, 31, 32, 33, 63 and 64 bodies."""
    rng = np.random.default_rng(4)
    sizes = [1, 2, 3, 8, 9, 16, 17, 31, 32, 33, 63, 64, 5]
    off = np.concatenate([[0], np.cumsum(sizes)])
    n = off[-1]
    pos = rng.uniform(-1, 1, (n, 3))
    vel = rng.normal(0, 0.3, (n, 3))
    m = np.exp(rng.uniform(np.log(0.1), np.log(10), n))
    return off, pos, vel, m


@pytest.mark.parametrize("group", [8, 16, 32, physgpu.ENS_BY_SIZE,
                                   32 | physgpu.ens_warps(4),
                                   physgpu.ENS_BY_SIZE | physgpu.ens_warps(4)])
def test_exact_bitexact_vs_oracle(ctx, group):
    off, pos, vel, m = edge_ensemble()
    ctx.ensemble_load(off, pos, vel, m)
    p = make_params(1.0, 1e-3, precision=F64_EXACT)
    ctx.ensemble_run(p, 1e-4, 15, group=group)
    x, v, a = ctx.ensemble_download()
    rx, rv, ra = oracle.ensemble_run(off, pos, vel, m, 1.0, 1e-3, 1e-4, 15)
    assert np.array_equal(x, rx) and np.array_equal(v, rv) and np.array_equal(a, ra)


def test_exact_random_systems_bitexact(ctx):
    off, pos, vel, m = small_ensemble(300, seed=1)
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(make_params(1.0, 1e-3, precision=F64_EXACT), 1e-4, 10, group=16)
    x, v, _ = ctx.ensemble_download()
    rx, rv, _ = oracle.ensemble_run(off, pos, vel, m, 1.0, 1e-3, 1e-4, 10)
    assert np.array_equal(x, rx) and np.array_equal(v, rv)


def test_chunked_graph_equals_single_launch(ctx):
    """The step loop split into graph-captured chunks (7 steps each), and
    runs split across calls, give the same trajectory as one launch."""
    off, pos, vel, m = small_ensemble(200, seed=2)
    p = make_params(1.0, 1e-3, precision=F64_EXACT)
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(p, 1e-4, 30, group=8, chunk=0)
    x1, v1, _ = ctx.ensemble_download()
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(p, 1e-4, 30, group=8, chunk=7)
    x2, v2, _ = ctx.ensemble_download()
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(p, 1e-4, 13, group=32)
    ctx.ensemble_run(p, 1e-4, 17, group=32)
    x3, v3, _ = ctx.ensemble_download()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert np.array_equal(x1, x3) and np.array_equal(v1, v3)


def test_f32c_close_to_exact(ctx):
    off, pos, vel, m = small_ensemble(1024, seed=3)
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(make_params(1.0, 1e-3, precision=F64_EXACT), 1e-4, 50, group=16)
    x64, _, a64 = ctx.ensemble_download()
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(make_params(1.0, 1e-3, precision=F32C), 1e-4, 50, group=16)
    x32, _, a32 = ctx.ensemble_download()
    dx = np.linalg.norm(x32 - x64, axis=1) / np.linalg.norm(x64, axis=1)
    da = np.linalg.norm(a32 - a64, axis=1) / np.linalg.norm(a64, axis=1)
    assert np.median(dx) < 1e-9
    assert np.median(da) < 1e-6


def test_autotune_and_default_group(ctx):
    off, pos, vel, m = small_ensemble(2048, seed=5)
    ctx.ensemble_load(off, pos, vel, m)
    p = make_params(1.0, 1e-3, precision=F32C)
    best, ms = ctx.ensemble_autotune(p, 1e-4, probe_steps=5)
    assert best in physgpu.ENS_CANDIDATES and all(t > 0 for t in ms.values())
    assert ms[best] == min(ms.values())
    x0, v0, _ = ctx.ensemble_download()
    assert np.array_equal(x0[:, 0], pos[:, 0])  # probes leave the state untouched
    ctx.ensemble_run(p, 1e-4, 5, group=0)
    x, _, _ = ctx.ensemble_download()
    assert np.all(np.isfinite(x)) and not np.array_equal(x, pos)


def test_oversized_system_rejected(ctx):
    off = np.array([0, 65])
    with pytest.raises(physgpu.PhysError) as ei:
        ctx.ensemble_load(off, np.zeros((65, 3)), None, np.ones(65))
    assert ei.value.status == physgpu.ERR_ARG


@pytest.mark.parametrize("config", [8, 16, 32, physgpu.ENS_BY_SIZE,
                                    physgpu.ENS_BY_SIZE | physgpu.ens_warps(4)])
def test_f32c_every_configuration_close_to_exact(ctx, config):
    """Every launch shape the autotuner may pick (lanes per system, lanes by
    size, the split layout of 33-64-body systems on 32 lanes, 2 or 4 warps
    per block) on systems of every size 1..64."""
    rng = np.random.default_rng(9)
    sizes = np.concatenate([np.arange(1, 65), rng.integers(3, 65, 200)])
    off = np.concatenate([[0], np.cumsum(sizes)])
    n = int(off[-1])
    pos = rng.uniform(-1, 1, (n, 3))
    vel = rng.normal(0, 0.3, (n, 3))
    m = np.exp(rng.uniform(np.log(0.1), np.log(10), n))
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(make_params(1.0, 1e-3, precision=F64_EXACT), 1e-4, 1, group=8)
    _, _, a64 = ctx.ensemble_download()
    ctx.ensemble_load(off, pos, vel, m)
    ctx.ensemble_run(make_params(1.0, 1e-3, precision=F32C), 1e-4, 1, group=config)
    _, _, a32 = ctx.ensemble_download()
    nz = np.linalg.norm(a64, axis=1) > 0
    da = np.linalg.norm(a32 - a64, axis=1)[nz] / np.linalg.norm(a64, axis=1)[nz]
    assert np.median(da) < 1e-6 and da.max() < 1e-4, (np.median(da), da.max())
    assert np.all(a32[~nz] == 0)


def test_bad_configuration_rejected(ctx):
    off, pos, vel, m = small_ensemble(10, seed=1)
    ctx.ensemble_load(off, pos, vel, m)
    for bad in (7, 64, 32 | physgpu.ens_warps(3), 1 << 20):
        with pytest.raises(physgpu.PhysError) as ei:
            ctx.ensemble_run(make_params(1.0, 1e-3, precision=F32C), 1e-4, 1, group=bad)
        assert ei.value.status == physgpu.ERR_ARG
