"""NFW phantom halo (src/physics/nfw.rs:103-139) through the C ABI.

Bar: the device's halo force matches the oracle to 1e-12 relative (the only
operation that may differ is ln(1 + x): CUDA's double log is within 1 ulp of
the host libm's, and M(r) = c (ln(1 + x) - x/(1 + x)) amplifies that for
small x = r/Rs); bodies at the centre are skipped; a disabled halo changes
nothing; accelerations and Verlet runs with the halo set follow the reference
schedule (gravity, then the halo, then a = F/m) to 1e-12; a body on a
circular orbit in the halo alone keeps its radius."""
import numpy as np
import pytest

import oracle
import physgpu
from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, GROUP_WALK, make_params

pytestmark = pytest.mark.gpu
G = physgpu.G_SI
RHO0, RS = 1.4e-21, 6.17e20  # nfw.rs:40-45 defaults


def halo(center=(0.0, 0.0, 0.0), enabled=True, rho_0=RHO0, rs=RS):
    return physgpu.NfwHaloConfig(rho_0=rho_0, scale_radius=rs, center=center, enabled=enabled)


def htuple(h):
    return (h.rho_0, h.scale_radius) + tuple(h.center)


def rel_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def galaxy_like(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.normal(scale=3e20, size=(n, 3))
    vel = rng.normal(scale=2e5, size=(n, 3))
    m = 10 ** rng.uniform(29.5, 31.0, n)
    return pos, vel, m


def test_halo_force_matches_oracle(ctx):
    pos, _, m = galaxy_like(5000, 1)
    pos[7] = (1e19, -2e19, 3e19)  # a displaced centre below
    h = halo(center=(1e19, -2e19, 3e19))
    ctx.upload(pos, None, m)
    f0 = np.random.default_rng(2).normal(size=(5000, 3)) * 1e20
    f = ctx.nfw_forces(h, f0)
    ref = oracle.nfw_forces(pos, m, htuple(h), f0)
    e = rel_err(f - f0, ref - f0)
    assert e.max() < 1e-12, e.max()
    assert np.mean(f == ref) > 0.9  # bit-identical apart from a log ulp here and there
    assert np.array_equal(f[7], f0[7])  # the body at the centre is skipped


def test_disabled_halo_and_bad_arguments(ctx):
    pos, _, m = galaxy_like(100, 3)
    ctx.upload(pos, None, m)
    f0 = np.ones((100, 3))
    assert np.array_equal(ctx.nfw_forces(halo(enabled=False), f0), f0)
    h = physgpu._halo(halo())
    h.reserved = 1
    with pytest.raises(physgpu.PhysError) as ei:
        ctx.nfw_forces(h, f0)
    assert ei.value.status == physgpu.ERR_ARG
    with pytest.raises(physgpu.PhysError):
        ctx.set_nfw_halo(h)


def test_accel_with_halo_follows_the_schedule(ctx):
    """phys_gravity_accel with the halo set = oracle (direct forces, then the
    halo's Force +=, then a = F/m)."""
    pos, _, m = galaxy_like(600, 4)
    h = halo(center=(5e19, 0.0, 0.0))
    p = make_params(G, 1e18, 0.5, DIRECT, F64_EXACT)
    ctx.upload(pos, None, m)
    ctx.set_nfw_halo(h)
    try:
        a = ctx.gravity_accel(p)
    finally:
        ctx.set_nfw_halo(None)
    f = oracle.direct_forces(pos, m, G, 1e18)
    f = oracle.nfw_forces(pos, m, htuple(h), f)
    ref = oracle.accel(f, m)
    assert rel_err(a, ref).max() < 1e-12
    # removing the halo gives the gravity-only accelerations back
    a0 = ctx.gravity_accel(p)
    assert np.array_equal(a0, oracle.accel(oracle.direct_forces(pos, m, G, 1e18), m))


@pytest.mark.parametrize("method,precision,flags,tol", [
    (DIRECT, F64_EXACT, 0, 1e-12),
    (BARNES_HUT, F64, GROUP_WALK, 1e-6),
    (BARNES_HUT, F32C, GROUP_WALK, 1e-6),
])
def test_verlet_steps_with_halo(ctx, method, precision, flags, tol):
    """10 Velocity-Verlet ticks with gravity + halo against the oracle's
    reference tick loop with nfw_gravity_system in both force passes (direct
    f64 sum in the oracle; the Barnes-Hut runs differ from it by the tree
    approximation, hence the looser bar)."""
    n, dt, steps = 512, 3e12, 10
    pos, vel, m = galaxy_like(n, 5)
    h = halo()
    p = make_params(G, 1e18, 0.3, method, precision, 8 if method == BARNES_HUT else 1, flags)
    ctx.upload(pos, vel, m)
    ctx.set_nfw_halo(h)
    try:
        ctx.verlet_steps(p, dt, steps)
    finally:
        ctx.set_nfw_halo(None)
    x, v, _ = ctx.download()
    xr, vr, _, _ = oracle.vv_run(pos, vel, m, G, 1e18, dt, steps, halo=htuple(h))
    dx = np.linalg.norm(x - xr, axis=1) / np.linalg.norm(xr - pos, axis=1)
    assert np.median(dx) < tol, np.median(dx)
    assert rel_err(v, vr).max() < (1e-12 if tol < 1e-9 else 1e-3)


def test_circular_orbit_in_halo_alone(ctx):
    """One body (gravity.rs:49-51 returns early for n < 2; the halo still
    acts) on a circular orbit at 5 Rs with v = nfw_circular_velocity keeps its
    radius over a quarter orbit."""
    r = 5 * RS
    vc = physgpu.nfw_circular_velocity(r, RHO0, RS)
    period = 2 * np.pi * r / vc
    steps = 2000
    dt = period / 4 / steps
    ctx.upload(np.array([[r, 0.0, 0.0]]), np.array([[0.0, vc, 0.0]]), np.array([1e30]))
    ctx.set_nfw_halo(halo())
    try:
        ctx.verlet_steps(make_params(G, 1e18, 0.5, DIRECT, F64_EXACT), dt, steps)
    finally:
        ctx.set_nfw_halo(None)
    x, v, _ = ctx.download()
    assert abs(np.linalg.norm(x[0]) - r) / r < 1e-5
    assert abs(np.linalg.norm(v[0]) - vc) / vc < 1e-5
    assert x[0, 1] > 0.9 * r  # a quarter turn


def test_mirror_system_matches_oracle(ctx):
    """physgpu.nfw_gravity_system (the ECS mirror) = oracle, Force +=."""
    pos, _, m = galaxy_like(300, 6)
    w = physgpu.World()
    for i in range(300):
        w.spawn(m[i], pos[i])
    w.force[:] = 1e21
    before = w.force.copy()
    cfg = halo(center=(-1e20, 0.0, 2e19))
    physgpu.nfw_gravity_system(w, cfg, ctx=ctx)
    ref = oracle.nfw_forces(pos, m, htuple(cfg), before)
    assert rel_err(w.force - before, ref - before).max() < 1e-12
    w2 = physgpu.World()
    w2.spawn(1.0, [1.0, 0.0, 0.0])
    physgpu.nfw_gravity_system(w2, halo(enabled=False), ctx=ctx)
    assert not w2.force.any()
