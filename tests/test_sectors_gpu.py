"""(Sector, LocalPosition) state kept on the device across Verlet ticks.

Bar: bit-identical to the oracle's reference tick loop on sectors
(flatten per force pass, LocalPosition integrated, sector_boundary_system
after the velocity step) for the exact direct sum and the exact Barnes-Hut
walk, including ticks in which bodies change sector; normalize_position's
known answers (coordinates.rs:136-157) hold on the device."""
import numpy as np
import pytest

import oracle
import physgpu
from physgpu import BARNES_HUT, DIRECT, F64_EXACT, make_params

pytestmark = pytest.mark.gpu
SIZE = 1e12  # coordinates.rs test SECTOR_SIZE


def crossing_system(n, seed, size):
    """Bodies spread over a few sectors, local offsets near the sector edges,
    fast enough that several cross a boundary within the run."""
    rng = np.random.default_rng(seed)
    sec = rng.integers(-2, 3, size=(n, 3)).astype(np.int64)
    loc = rng.uniform(-0.5, 0.5, size=(n, 3)) * size
    loc[: n // 4] = np.sign(loc[: n // 4]) * 0.4999 * size
    vel = rng.normal(scale=0.002 * size, size=(n, 3))
    m = rng.uniform(1e24, 1e26, n)
    return sec, loc, vel, m


def test_normalize_known_answers_on_device(ctx):
    """dt = 0: one tick leaves positions alone, then normalises them."""
    loc = np.array([[1.2e12, 0.0, 0.0], [-1.2e12, 0.0, 0.0], [0.5e12, -0.5e12, 0.4e12]])
    sec = np.zeros((3, 3), np.int64)
    m = np.ones(3) * 1e20
    ctx.upload_sector_state(sec, loc, SIZE, m)
    ctx.verlet_steps(make_params(physgpu.G_SI, 1e-4, 0.5, DIRECT, F64_EXACT), 0.0, 1)
    s, l = ctx.download_sector_state()
    rs, rl, _ = oracle.normalize(sec, loc, SIZE)
    assert np.array_equal(s, rs) and np.array_equal(l, rl)
    assert s[0, 0] == 1 and s[1, 0] == -1 and list(s[2]) == [1, -1, 0]


@pytest.mark.parametrize("method", [DIRECT, BARNES_HUT])
def test_run_on_sectors_bit_identical(ctx, method):
    n, steps, dt = 300, 25, 100.0
    sec, loc, vel, m = crossing_system(n, 7 + method, SIZE)
    G, eps = physgpu.G_SI, 1e6
    p = make_params(G, eps, 0.5, method, F64_EXACT)
    ctx.upload_sector_state(sec, loc, SIZE, m, vel)
    ctx.verlet_steps(p, dt, steps)
    s, l = ctx.download_sector_state()
    _, v, a = ctx.download()
    rs, rl, rv, ra, _ = oracle.vv_run_sectors(sec, loc, vel, m, SIZE, G, eps, dt, steps,
                                              method="direct" if method == DIRECT else "bh")
    moved = np.any(rs != sec, axis=1).sum()
    assert moved > 0  # the run exercised sector changes
    assert np.array_equal(s, rs)
    assert np.array_equal(l, rl)
    assert np.array_equal(v, rv)
    assert np.array_equal(a, ra)
    # the POSITION component is LocalPosition in this mode
    assert np.array_equal(ctx.read_component(physgpu.COMP_POSITION), rl)


def test_run_on_sectors_with_halo(ctx):
    """The halo reads LocalPosition, gravity the flattened positions."""
    n, steps, dt = 200, 10, 1e11
    rng = np.random.default_rng(3)
    size = 1e21
    sec = rng.integers(-1, 2, size=(n, 3)).astype(np.int64)
    loc = rng.uniform(-0.5, 0.5, size=(n, 3)) * size
    vel = rng.normal(scale=1e5, size=(n, 3))
    m = rng.uniform(1e30, 1e31, n)
    h = physgpu.NfwHaloConfig(enabled=True)
    G, eps = physgpu.G_SI, 1e17
    ctx.upload_sector_state(sec, loc, size, m, vel)
    ctx.set_nfw_halo(h)
    try:
        ctx.verlet_steps(make_params(G, eps, 0.5, DIRECT, F64_EXACT), dt, steps)
    finally:
        ctx.set_nfw_halo(None)
    s, l = ctx.download_sector_state()
    rs, rl, _, _, _ = oracle.vv_run_sectors(
        sec, loc, vel, m, size, G, eps, dt, steps,
        halo=(h.rho_0, h.scale_radius) + tuple(h.center))
    assert np.array_equal(s, rs)
    assert np.max(np.abs(l - rl)) <= 1e-12 * size


def test_mirror_run_velocity_verlet(ctx):
    """physgpu.run_velocity_verlet (World, UniverseConfig, SimulationTime)
    = the oracle's tick loop on sectors; time advances."""
    sec, loc, vel, m = crossing_system(120, 11, SIZE)
    w = physgpu.World()
    for i in range(120):
        w.spawn(m[i], loc[i], sector=sec[i], velocity=vel[i])
    cfg = physgpu.UniverseConfig(softening_epsilon=1e6, sector_size=SIZE)
    t = physgpu.SimulationTime(dt=100.0)
    physgpu.run_velocity_verlet(w, cfg, t, 12, ctx=ctx)
    rs, rl, rv, ra, rpa = oracle.vv_run_sectors(sec, loc, vel, m, SIZE, physgpu.G_SI, 1e6,
                                                100.0, 12)
    assert np.array_equal(w.sector, rs) and np.array_equal(w.local, rl)
    assert np.array_equal(w.velocity, rv) and np.array_equal(w.acceleration, ra)
    assert np.array_equal(w.prev_acceleration, rpa)
    assert t.tick == 12


def test_plain_upload_leaves_sector_mode(ctx):
    sec, loc, vel, m = crossing_system(50, 2, SIZE)
    ctx.upload_sector_state(sec, loc, SIZE, m, vel)
    ctx.upload(loc, vel, m)
    with pytest.raises(physgpu.PhysError) as ei:
        ctx.download_sector_state()
    assert ei.value.status == physgpu.ERR_STATE
