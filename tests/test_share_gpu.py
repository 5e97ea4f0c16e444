"""Target shares through the C ABI (phys_gravity_accel_share / _unshare): one
system split over GPUs that each hold the whole state.

On one GPU the ranks run one after another (each share evaluated, the
blocks concatenated as an all-gather would, then scattered), which is the
multi-GPU data path without any kernel waiting on another.  Every share
layout gives the accelerations of a one-GPU evaluation bit for bit (direct
sum in all three precisions, Barnes-Hut with both walks), and a two-context
Verlet run whose evaluations are split this way keeps the one-GPU
trajectory bit for bit."""
import numpy as np
import pytest
import torch

import physgpu
import physgpu.dist as pd
import physgpu.ics as ics
from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, GROUP_WALK, make_params

pytestmark = pytest.mark.gpu

CASES = [
    ("direct_exact", make_params(1.0, 0.01, method=DIRECT, precision=F64_EXACT)),
    ("direct_f64", make_params(1.0, 0.01, method=DIRECT, precision=F64)),
    ("direct_f32c", make_params(1.0, 0.01, method=DIRECT, precision=F32C)),
    ("bh_exact", make_params(1.0, 0.01, 0.5, BARNES_HUT, F64_EXACT, 1)),
    ("bh_f64_body", make_params(1.0, 0.01, 0.5, BARNES_HUT, F64, 8)),
    ("bh_f32c_body", make_params(1.0, 0.01, 0.5, BARNES_HUT, F32C, 8)),
    ("bh_f64_group", make_params(1.0, 0.01, 0.5, BARNES_HUT, F64, 8, GROUP_WALK)),
    ("bh_f32c_group", make_params(1.0, 0.01, 0.5, BARNES_HUT, F32C, 8, GROUP_WALK)),
]


def shared_accel(ctx, p, world):
    """All shares of one evaluation on one context, gathered and scattered."""
    c = physgpu.share_chunk(ctx.n, world)
    blocks = [torch.empty(3 * c, dtype=torch.float64, device="cuda") for _ in range(world)]
    for r in range(world):
        ctx.gravity_accel_share(p, r, world, blocks[r].data_ptr())
    gathered = torch.cat(blocks)
    ctx.gravity_accel_unshare(world, gathered.data_ptr())
    torch.cuda.synchronize()
    _, _, a = ctx.download()
    return a


@pytest.mark.parametrize("name,p", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("world", [2, 3, 8])
def test_shares_equal_one_gpu_evaluation(ctx, name, p, world):
    n = 9000 if name.startswith("direct") else 70001
    pos, vel, m = ics.plummer(n, seed=11)
    ctx.upload(pos, vel, m)
    full = ctx.gravity_accel(p)
    got = shared_accel(ctx, p, world)
    assert np.array_equal(got, full)


def test_share_blocks_hold_their_targets(ctx):
    """Block r holds targets [r c, (r+1) c) in order, zero-padded."""
    pos, vel, m = ics.plummer(1000, seed=2)
    ctx.upload(pos, vel, m)
    p = make_params(1.0, 0.01, method=DIRECT, precision=F64)
    full = ctx.gravity_accel(p)
    world, c = 3, physgpu.share_chunk(1000, 3)
    blk = torch.empty(3 * c, dtype=torch.float64, device="cuda")
    ctx.gravity_accel_share(p, 2, world, blk.data_ptr())
    b = blk.cpu().numpy().reshape(3, c)
    lo = 2 * c
    assert np.array_equal(b[:, :1000 - lo].T, full[lo:])
    assert not b[:, 1000 - lo:].any()


def test_shares_with_halo(ctx):
    pos, vel, m = ics.plummer(5000, seed=4)
    ctx.upload(pos, vel, m)
    ctx.set_nfw_halo(physgpu.NfwHaloConfig(rho_0=0.05, scale_radius=2.0, center=(0.1, 0.0, -0.1),
                                           enabled=True))
    try:
        p = make_params(1.0, 0.01, 0.5, BARNES_HUT, F32C, 8, GROUP_WALK)
        full = ctx.gravity_accel(p)
        assert np.array_equal(shared_accel(ctx, p, 4), full)
    finally:
        ctx.set_nfw_halo(None)


@pytest.mark.parametrize("p", [CASES[0][1], CASES[7][1]], ids=["direct_exact", "bh_f32c_group"])
def test_two_context_verlet_keeps_one_gpu_trajectory(ctx, p):
    """Two contexts stand in for two ranks: both integrate every body, each
    evaluates its share, the blocks are concatenated and both scatter them."""
    n, dt, steps = (2048, 1e-3, 6) if p.method == DIRECT else (60000, 1e-3, 3)
    pos, vel, m = ics.plummer(n, seed=9)
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(p, dt, steps)
    want = ctx.download()
    ranks = [physgpu.Context(0), physgpu.Context(0)]
    try:
        world, c = 2, physgpu.share_chunk(n, 2)
        blocks = [torch.empty(3 * c, dtype=torch.float64, device="cuda") for _ in range(world)]
        for r in ranks:
            r.upload(pos, vel, m)

        def evaluate():
            for k, r in enumerate(ranks):
                r.gravity_accel_share(p, k, world, blocks[k].data_ptr())
            g = torch.cat(blocks)
            for r in ranks:
                r.gravity_accel_unshare(world, g.data_ptr())
            torch.cuda.synchronize()

        evaluate()
        for _ in range(steps):
            for r in ranks:
                r.vv_position_step(dt)
            evaluate()
            for r in ranks:
                r.vv_velocity_step(dt)
        for r in ranks:
            for got, w in zip(r.download(), want):
                assert np.array_equal(got, w)
    finally:
        for r in ranks:
            r.close()


def test_driver_with_one_rank_keeps_trajectory(ctx):
    """physgpu.dist.verlet_steps_shared without a process group (world 1)."""
    p = make_params(1.0, 0.01, 0.5, BARNES_HUT, F32C, 8, GROUP_WALK)
    pos, vel, m = ics.plummer(40000, seed=5)
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(p, 1e-3, 3)
    want = ctx.download()
    ctx.upload(pos, vel, m)
    pd.verlet_steps_shared(ctx, p, 1e-3, 3)
    for got, w in zip(ctx.download(), want):
        assert np.array_equal(got, w)


def test_share_errors(ctx):
    pos, vel, m = ics.plummer(1000, seed=1)
    ctx.upload(pos, vel, m)
    p = make_params(1.0, 0.01, method=DIRECT, precision=F64)
    c = physgpu.share_chunk(1000, 2)
    blk = torch.empty(3 * c * 2, dtype=torch.float64, device="cuda")
    with pytest.raises(physgpu.PhysError) as e:
        ctx.gravity_accel_unshare(2, blk.data_ptr())  # no share evaluated
    assert e.value.status == physgpu.ERR_STATE
    for rank, world in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(physgpu.PhysError) as e:
            ctx.gravity_accel_share(p, rank, world, blk.data_ptr())
        assert e.value.status == physgpu.ERR_ARG
    ctx.gravity_accel_share(p, 0, 2, blk.data_ptr())
    with pytest.raises(physgpu.PhysError) as e:
        ctx.gravity_accel_unshare(3, blk.data_ptr())  # another world
    assert e.value.status == physgpu.ERR_ARG
    ctx.gravity_accel(p)  # any other evaluation voids the pending share
    with pytest.raises(physgpu.PhysError) as e:
        ctx.gravity_accel_unshare(2, blk.data_ptr())
    assert e.value.status == physgpu.ERR_STATE
