"""Velocity-Verlet (K7) and diagnostics (K10) parity through the C ABI.

Bar: device-resident trajectories in F64_EXACT are bit-identical to the
oracle's reference tick loop (src/main.rs:103-140); energy/momentum within
1e-12 relative of the oracle's sequential sums."""
import math

import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, make_params

pytestmark = pytest.mark.gpu


def test_plummer_1024_100_steps_bitexact(ctx):
    """Plain direct-sum workload: N = 1024 Plummer, G = 1, eps = 0.01,
    dt = 1e-3, 100 Velocity-Verlet ticks, F64_EXACT."""
    pos, vel, m = ics.plummer(1024, seed=0)
    ctx.upload(pos, vel, m)
    p = make_params(1.0, 0.01, method=DIRECT, precision=F64_EXACT)
    ctx.verlet_steps(p, 1e-3, 100)
    x, v, a = ctx.download()
    rx, rv, ra, _ = oracle.vv_run(pos, vel, m, 1.0, 0.01, 1e-3, 100, method="direct")
    assert np.array_equal(x, rx) and np.array_equal(v, rv) and np.array_equal(a, ra)


def test_split_calls_equal_one_call(ctx):
    """Cached a(x) across calls: 3 + 4 steps == 7 steps."""
    pos, vel, m = ics.plummer(700, seed=3)
    p = make_params(1.0, 0.01, method=DIRECT, precision=F64_EXACT)
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(p, 1e-3, 3)
    ctx.verlet_steps(p, 1e-3, 4)
    x1, v1, _ = ctx.download()
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(p, 1e-3, 7)
    x2, v2, _ = ctx.download()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)


def test_bh_exact_trajectory_bitexact(ctx):
    pos, vel, m = ics.plummer(2048, seed=2)
    ctx.upload(pos, vel, m)
    p = make_params(1.0, 0.01, 0.5, BARNES_HUT, F64_EXACT)
    ctx.verlet_steps(p, 1e-3, 4)
    x, v, a = ctx.download()
    rx, rv, ra, _ = oracle.vv_run(pos, vel, m, 1.0, 0.01, 1e-3, 4, method="bh", theta=0.5)
    assert np.array_equal(x, rx) and np.array_equal(v, rv) and np.array_equal(a, ra)


def test_f32c_bh_trajectory_close(ctx):
    """Mixed precision (f32 pair terms, f64 state) stays close to the f64
    reference over 10 steps of the Barnes-Hut workload shape."""
    pos, vel, m = ics.plummer(16384, seed=6)
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(make_params(1.0, 0.01, 0.5, BARNES_HUT, F32C, 8), 1e-3, 10)
    x32, v32, _ = ctx.download()
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(make_params(1.0, 0.01, 0.5, BARNES_HUT, F64, 8), 1e-3, 10)
    x64, v64, _ = ctx.download()
    dx = np.linalg.norm(x32 - x64, axis=1) / np.linalg.norm(x64, axis=1)
    assert np.median(dx) < 1e-10


def test_vv_systems_mirror_bitexact(ctx):
    """velocity_verlet_position_system / velocity_verlet_velocity_system
    (integrators.rs:63-104) through the ECS mirror vs the oracle."""
    rng = np.random.default_rng(1)
    n = 257
    w = physgpu.World.from_arrays(rng.normal(0, 1, (n, 3)), rng.normal(0, 1, (n, 3)),
                                  rng.uniform(1, 2, n))
    w.acceleration = rng.normal(0, 1, (n, 3))
    w.prev_acceleration = rng.normal(0, 1, (n, 3))
    t = physgpu.SimulationTime.with_dt(0.013)
    X = [w.local[:, k].copy() for k in range(3)]
    V = [w.velocity[:, k].copy() for k in range(3)]
    A = [w.acceleration[:, k].copy() for k in range(3)]
    PA = [w.prev_acceleration[:, k].copy() for k in range(3)]
    L, P = oracle.lib(), oracle._p
    physgpu.velocity_verlet_position_system(w, t, ctx=ctx)
    L.oracle_vv_position(n, 0.013, *[P(a) for a in X + V + A + PA])
    assert np.array_equal(w.local, np.stack(X, 1))
    assert np.array_equal(w.prev_acceleration, np.stack(PA, 1))
    w.acceleration = rng.normal(0, 1, (n, 3))
    A = [w.acceleration[:, k].copy() for k in range(3)]
    physgpu.velocity_verlet_velocity_system(w, t, ctx=ctx)
    L.oracle_vv_velocity(n, 0.013, *[P(a) for a in V + A + PA])
    assert np.array_equal(w.velocity, np.stack(V, 1))


def test_circular_orbit_energy_mirror(ctx):
    """integrators.rs:288-348 through the ECS mirror: GM = 1 circular orbit,
    dt = 1e-3, 6283 ticks with a = -r/|r|^3 set between the two systems;
    energy drift < 1e-4 (run as 300 ticks here, same per-tick bound)."""
    w = physgpu.World()
    w.spawn(1.0, [1.0, 0.0, 0.0], velocity=[0.0, 1.0, 0.0], acceleration=[-1.0, 0, 0],
            prev_acceleration=[-1.0, 0, 0])
    t = physgpu.SimulationTime.with_dt(0.001)
    for _ in range(300):
        physgpu.velocity_verlet_position_system(w, t, ctx=ctx)
        r = w.local[0]
        rm = math.sqrt(float(r @ r))
        w.acceleration = (-r / (rm * rm * rm))[None]
        physgpu.velocity_verlet_velocity_system(w, t, ctx=ctx)
        t.advance_tick()
    v, r = w.velocity[0], w.local[0]
    e = 0.5 * float(v @ v) - 1.0 / math.sqrt(float(r @ r))
    assert abs(e + 0.5) < 1e-4


@pytest.mark.parametrize("n", [2, 100, 3000])
def test_diagnostics_vs_oracle(ctx, n):
    pos, vel, m = ics.plummer(n, seed=n)
    ctx.upload(pos, vel, m)
    out = ctx.diagnostics(1.0)
    ref = oracle.energy(pos, vel, m, 1.0)
    assert abs(out[0] - ref[0]) <= 1e-12 * abs(ref[0])
    assert abs(out[1] - ref[1]) <= 1e-12 * abs(ref[1])
    assert np.all(np.abs(out[2:] - ref[2:]) <= 1e-12 * np.abs(m[:, None] * vel).sum(0) + 1e-300)


def test_energy_mirror_skips_coincident_pairs(ctx):
    """energy.rs:49: pairs with r^2 == 0 contribute no potential energy."""
    w = physgpu.World()
    w.spawn(2.0, [0.0, 0, 0], velocity=[1.0, 0, 0])
    w.spawn(3.0, [0.0, 0, 0])
    w.spawn(1.0, [3.0, 4.0, 0.0], velocity=[0, 2.0, 0])
    ke, pe, p = physgpu.energy_diagnostics(w, physgpu.UniverseConfig(gravitational_constant=1.0),
                                           ctx=ctx)
    assert ke == 0.5 * 2.0 * 1.0 + 0.5 * 1.0 * 4.0
    assert abs(pe - (-(2.0 / 5.0) - (3.0 / 5.0))) < 1e-15
    assert np.allclose(p, [2.0, 2.0, 0.0])


@pytest.mark.parametrize("pinned", [False, True])
def test_tick_host_equals_four_calls(ctx, pinned):
    """phys_verlet_tick_host == upload + set_accel + one tick + download, bit
    for bit, with pageable (numpy) and page-locked (torch) host arrays."""
    import torch
    n = 30000
    pos, vel, m = ics.plummer(n, seed=6)
    acc = np.random.default_rng(6).normal(size=(n, 3)) * 1e-3
    p = make_params(1.0, 0.01, 0.5, physgpu.BARNES_HUT, physgpu.F32C, 8, physgpu.GROUP_WALK)
    ctx.upload(pos, vel, m)
    ctx.set_accel(acc)
    ctx.verlet_steps(p, 1e-3, 1)
    want = ctx.download()

    def arrays(a):
        cols = [np.ascontiguousarray(a[:, k]) for k in range(3)]
        if not pinned:
            return cols
        return [torch.from_numpy(c).pin_memory() for c in cols]
    X, V, A = arrays(pos), arrays(vel), arrays(acc)
    M = torch.from_numpy(m.copy()).pin_memory() if pinned else m.copy()
    ctx.verlet_tick_host(p, 1e-3, X, V, M, A)
    got = [np.stack([np.asarray(c) for c in t], axis=1) for t in (X, V, A)]
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


@pytest.mark.parametrize("prec", [F64_EXACT, F64, F32C])
def test_graph_replayed_ticks_equal_single_ticks(ctx, prec):
    """The direct sum's middle ticks replay a captured graph: a 7-tick run
    equals seven 1-tick runs bit for bit, and the cached graph follows a
    change of dt, of the parameters and of the body count."""
    def run(n, p, dt, ticks, one_by_one):
        pos, vel, m = ics.plummer(n, seed=n)
        ctx.upload(pos, vel, m)
        if one_by_one:
            for _ in range(ticks):
                ctx.verlet_steps(p, dt, 1)
        else:
            ctx.verlet_steps(p, dt, ticks)
        return ctx.download()
    p = make_params(1.0, 0.01, method=DIRECT, precision=prec)
    q = make_params(1.0, 0.02, method=DIRECT, precision=prec)
    for n, pp, dt in ((1000, p, 1e-3), (1000, p, 2e-3), (1000, q, 2e-3), (3000, q, 2e-3),
                      (1000, p, 1e-3)):
        a = run(n, pp, dt, 7, False)
        b = run(n, pp, dt, 7, True)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), (n, dt)
