"""Direct-sum parity (K1) through the C ABI against the oracle.

Bar: F64_EXACT is bit-identical to the reference's arithmetic (oracle of
gravity.rs:53-69); F64 within 1e-12 relative; F32C within 1e-6 median
relative of the f64 result (tolerances stated per test)."""
import math

import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import DIRECT, F32C, F64, F64_EXACT, make_params

pytestmark = pytest.mark.gpu
G_SI = physgpu.G_SI


def rel_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def test_figure_8_stability_mirror(ctx):
    """gravity.rs:81-103 through the ECS mirror."""
    w = physgpu.World()
    for p in ([-0.97000436, 0.24308753, 0.0], [0.97000436, -0.24308753, 0.0], [0.0, 0.0, 0.0]):
        w.spawn(1.0, p)
    cfg = physgpu.UniverseConfig(softening_epsilon=0.0)
    physgpu.brute_force_gravity_system(w, cfg, ctx=ctx)
    f = w.force
    assert np.all(np.isfinite(f))
    assert abs(f[:, 0].sum()) < 1e-10 and abs(f[:, 1].sum()) < 1e-10
    ref = oracle.direct_forces(w.local, w.mass, G_SI, 0.0)
    assert np.array_equal(f, ref)


def test_kepler_orbit_period_mirror(ctx):
    """gravity.rs:106-130 through the ECS mirror."""
    w = physgpu.World()
    w.spawn(1e12, [0.0, 0.0, 0.0])
    small = w.spawn(1.0, [100.0, 0.0, 0.0])
    physgpu.brute_force_gravity_system(w, physgpu.UniverseConfig(softening_epsilon=0.0), ctx=ctx)
    f = w.force[small]
    expected = -(G_SI * 1e12 * 1.0) / (100.0 * 100.0)
    assert abs(f[0] - expected) < 1e-10
    assert f[1] == 0.0 and f[2] == 0.0


@pytest.mark.parametrize("n", [2, 3, 5, 8, 9, 17, 31, 32, 33, 63, 64, 65, 127, 129, 300, 1031])
def test_exact_small_n_bitexact(ctx, n):
    rng = np.random.default_rng(n)
    pos = rng.normal(0, 1, (n, 3))
    m = rng.uniform(0.5, 2.0, n)
    ctx.upload(pos, None, m)
    f = ctx.gravity_forces(make_params(1.0, 0.05, method=DIRECT, precision=F64_EXACT))
    assert np.array_equal(f, oracle.direct_forces(pos, m, 1.0, 0.05))


def test_exact_plummer_1024_bitexact(ctx):
    """Shape of the plain direct-sum workload: N = 1024 Plummer, G = 1, eps = 0.01."""
    pos, vel, m = ics.plummer(1024, seed=1)
    ctx.upload(pos, vel, m)
    p = make_params(1.0, 0.01, method=DIRECT, precision=F64_EXACT)
    f = ctx.gravity_forces(p)
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    assert np.array_equal(f, ref)
    a = ctx.gravity_accel(p)
    assert np.array_equal(a, oracle.accel(ref, m))  # a = F / m (integrators.rs:115)


def test_force_accumulates(ctx):
    """Force += computed (gravity.rs:71-73): existing forces are kept."""
    pos, _, m = ics.plummer(200, seed=2)
    ctx.upload(pos, None, m)
    pre = np.random.default_rng(0).normal(0, 1, (200, 3))
    f = ctx.gravity_forces(make_params(1.0, 0.01, precision=F64_EXACT), pre.copy())
    assert np.array_equal(f, pre + oracle.direct_forces(pos, m, 1.0, 0.01))


@pytest.mark.parametrize("n", [1000, 4096, 20000])
def test_f64_close_to_reference(ctx, n):
    """F64 (FMA + rsqrt, sliced j) vs the reference arithmetic: <= 1e-12 relative."""
    pos, _, m = ics.plummer(n, seed=n)
    ctx.upload(pos, None, m)
    f = ctx.gravity_forces(make_params(1.0, 0.01, precision=F64))
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    assert rel_err(f, ref).max() < 1e-12


@pytest.mark.parametrize("n", [1000, 4096, 20000])
def test_f32c_vs_f64(ctx, n):
    """F32C vs the f64 direct sum: median relative error <= 1e-6 (max <= 1e-4)."""
    pos, _, m = ics.plummer(n, seed=n + 1)
    ctx.upload(pos, None, m)
    f32 = ctx.gravity_forces(make_params(1.0, 0.01, precision=F32C))
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    e = rel_err(f32, ref)
    assert np.median(e) <= 1e-6, np.median(e)
    assert e.max() <= 1e-4, e.max()


def test_f32c_offset_system_keeps_accuracy(ctx):
    """Relative coordinates: a cluster far from the origin loses no accuracy."""
    pos, _, m = ics.plummer(2000, seed=9)
    pos = pos * 1e-3 + np.array([1e4, -2e4, 5e3])
    ctx.upload(pos, None, m)
    f32 = ctx.gravity_forces(make_params(1.0, 1e-5, precision=F32C))
    ref = oracle.direct_forces(pos, m, 1.0, 1e-5)
    assert np.median(rel_err(f32, ref)) <= 1e-6


def test_sector_flattening(ctx):
    """gravity.rs:38-47: bodies in different sectors are measured from the
    first body's sector before the pair law."""
    rng = np.random.default_rng(4)
    n = 64
    sec = rng.integers(-2, 3, (n, 3))
    loc = rng.uniform(-0.5e3, 0.5e3, (n, 3))
    m = rng.uniform(1e20, 1e22, n)
    ctx.upload_sectors(sec, loc, 1e4, m)
    f = ctx.gravity_forces(make_params(G_SI, 1e-4, precision=F64_EXACT))
    x = oracle.flatten(sec, loc, 1e4)
    assert np.array_equal(f, oracle.direct_forces(x, m, G_SI, 1e-4))


def test_n_below_two_returns_early(ctx):
    """gravity.rs:49-51: fewer than two bodies leave Force untouched."""
    ctx.upload(np.zeros((1, 3)), None, np.ones(1))
    pre = np.array([[1.0, 2.0, 3.0]])
    assert np.array_equal(ctx.gravity_forces(make_params(1.0, 0.0), pre.copy()), pre)
    ctx.upload(np.zeros((0, 3)), None, np.zeros(0))
    assert ctx.gravity_forces(make_params(1.0, 0.0)).shape == (0, 3)


def test_nonfinite_input_is_reported(ctx):
    pos = np.array([[0.0, 0, 0], [1.0, math.nan, 0], [2.0, 0, 0]])
    ctx.upload(pos, None, np.ones(3))
    with pytest.raises(physgpu.PhysError) as ei:
        ctx.gravity_forces(make_params(1.0, 0.1, precision=F64))
    assert ei.value.status == physgpu.ERR_NONFINITE
    # the context stays usable
    ctx.upload(np.array([[0.0, 0, 0], [1.0, 0, 0]]), None, np.ones(2))
    f = ctx.gravity_forces(make_params(1.0, 0.0, precision=F64_EXACT))
    assert f[0, 0] == 1.0 and f[1, 0] == -1.0


def test_bad_arguments(ctx):
    ctx.upload(np.zeros((4, 3)) + np.arange(4)[:, None], None, np.ones(4))
    for bad in (make_params(1.0, 0.0, method=7), make_params(1.0, 0.0, precision=9),
                make_params(1.0, 0.0, leaf_cap=0), make_params(1.0, 0.0, theta=-1.0)):
        with pytest.raises(physgpu.PhysError) as ei:
            ctx.gravity_forces(bad)
        assert ei.value.status == physgpu.ERR_ARG


def test_direct_targets_subset(ctx):
    """Direct sum for a list of targets (the f64 reference for BH runs)."""
    pos, _, m = ics.plummer(5000, seed=21)
    ctx.upload(pos, None, m)
    t = np.random.default_rng(0).choice(5000, 300, replace=False)
    ref = oracle.accel(oracle.direct_forces(pos, m, 1.0, 0.01), m)[t]
    a = ctx.direct_accel_targets(make_params(1.0, 0.01, precision=F64_EXACT), t)
    assert np.array_equal(a, ref)
    a64 = ctx.direct_accel_targets(make_params(1.0, 0.01, precision=F64), t)
    assert rel_err(a64, ref).max() < 1e-12
    with pytest.raises(physgpu.PhysError):
        ctx.direct_accel_targets(make_params(1.0, 0.01, precision=F64), np.array([0, 5000]))
