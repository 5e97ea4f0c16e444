"""Group walk (PHYS_FLAG_GROUP_WALK): one Barnes-Hut walk per 64 key-adjacent
bodies with a shared interaction list.

Bar: theta = 0 equals the direct sum up to summation order (1e-12 relative,
f64) and counts exactly n(n-1) pairs; F32C within 1e-6 median relative of
F64 on the same lists; the force error against the direct sum is no larger
than the per-body walk's (the group criterion only opens more cells);
ragged group sizes, coincident bodies, zero masses and eps = 0 run."""
import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, GROUP_WALK, make_params

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def gw(theta=0.5, precision=F64, leaf_cap=8, eps=0.01, G=1.0):
    return make_params(G, eps, theta, BARNES_HUT, precision, leaf_cap, GROUP_WALK)


@pytest.mark.parametrize("n", [2, 3, 63, 64, 65, 1000, 5000])
@pytest.mark.parametrize("leaf_cap", [1, 8])
def test_theta_zero_is_direct_sum(ctx, n, leaf_cap):
    pos, _, m = ics.plummer(n, seed=n + leaf_cap)
    ctx.upload(pos, None, m)
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    f = ctx.gravity_forces(gw(0.0, F64, leaf_cap))
    assert rel_err(f, ref).max() < 1e-12
    assert ctx.timings()["interactions"] == n * (n - 1)
    f32 = ctx.gravity_forces(gw(0.0, F32C, leaf_cap))
    assert np.median(rel_err(f32, ref)) < 1e-6
    assert ctx.timings()["interactions"] == n * (n - 1)


@pytest.mark.parametrize("n", [8, 9, 16, 17, 32, 33, 40, 41, 48, 49])
def test_single_group_layouts_theta_zero(ctx, n):
    """Systems of at most 64 bodies are one group: at theta = 0 every body
    of every target layout (one per lane; a second target shared by 4 lane
    streams at 33-40 bodies or 2 at 41-48; two per lane above) must match the
    direct sum, the in-group pass skipping exactly i == j."""
    pos, _, m = ics.plummer(n, seed=100 + n)
    ctx.upload(pos, None, m)
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    f32 = ctx.gravity_forces(gw(0.0, F32C, 8))
    assert ctx.timings()["interactions"] == n * (n - 1)
    e = rel_err(f32, ref)
    assert np.median(e) < 1e-6 and e.max() < 1e-4


@pytest.mark.parametrize("leaf_cap", [1, 8, 16])
def test_f32c_vs_f64_same_lists(ctx, leaf_cap):
    pos, _, m = ics.plummer(65536, seed=21)
    ctx.upload(pos, None, m)
    a64 = ctx.gravity_accel(gw(0.5, F64, leaf_cap))
    n64 = ctx.timings()["interactions"]
    a32 = ctx.gravity_accel(gw(0.5, F32C, leaf_cap))
    assert ctx.timings()["interactions"] == n64
    e = rel_err(a32, a64)
    assert np.median(e) <= 1e-6, np.median(e)
    assert e.max() <= 1e-4, e.max()


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_error_not_above_per_body_walk(ctx, theta):
    pos, _, m = ics.plummer(20000, seed=5)
    ctx.upload(pos, None, m)
    ref = ctx.gravity_accel(make_params(1.0, 0.01, 0.5, DIRECT, F64))
    body = ctx.gravity_accel(make_params(1.0, 0.01, theta, BARNES_HUT, F64, 8))
    nb = ctx.timings()["interactions"]
    grp = ctx.gravity_accel(gw(theta, F64, 8))
    ng = ctx.timings()["interactions"]
    eb, eg = rel_err(body, ref), rel_err(grp, ref)
    assert ng >= nb
    assert np.median(eg) <= np.median(eb)
    assert np.percentile(eg, 99) <= np.percentile(eb, 99) * 1.05


def test_coincident_zero_mass_and_clusters(ctx):
    rng = np.random.default_rng(3)
    pos = rng.normal(size=(3000, 3))
    pos[100:140] = pos[100]          # a coincident clump (guard-depth leaf)
    pos[500:530] = pos[500] + rng.normal(scale=1e-9, size=(30, 3))
    m = rng.uniform(0.5, 1.5, 3000)
    m[700:720] = 0.0
    ctx.upload(pos, None, m)
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    for cap in (2, 8, 16):
        f0 = ctx.gravity_forces(gw(0.0, F64, cap))
        assert rel_err(f0, ref).max() < 1e-12
        f = ctx.gravity_forces(gw(0.5, F64, cap))
        f32 = ctx.gravity_forces(gw(0.5, F32C, cap))
        assert np.all(np.isfinite(f)) and np.all(np.isfinite(f32))
        assert np.median(rel_err(f, ref)) < 1e-2
        assert np.median(rel_err(f32, f)) < 1e-6


def test_zero_softening_distinct_bodies(ctx):
    pos, _, m = ics.plummer(4000, seed=8)
    ctx.upload(pos, None, m)
    ref = oracle.direct_forces(pos, m, 1.0, 0.0)
    f = ctx.gravity_forces(gw(0.0, F64, 8, eps=0.0))
    assert rel_err(f, ref).max() < 1e-11
    f32 = ctx.gravity_forces(gw(0.5, F32C, 8, eps=0.0))
    assert np.all(np.isfinite(f32))


def test_si_units_sectors(ctx):
    """SI-scale positions (1e11 m) and masses (1e24-1e30 kg), G = 6.674e-11."""
    rng = np.random.default_rng(9)
    pos = rng.normal(scale=1e11, size=(6000, 3))
    m = 10 ** rng.uniform(24, 30, 6000)
    ctx.upload(pos, None, m)
    G = physgpu.G_SI
    ref = oracle.direct_forces(pos, m, G, 1e-4)
    f = ctx.gravity_forces(gw(0.0, F64, 8, eps=1e-4, G=G))
    assert rel_err(f, ref).max() < 1e-12
    a64 = ctx.gravity_accel(gw(0.5, F64, 8, eps=1e-4, G=G))
    a32 = ctx.gravity_accel(gw(0.5, F32C, 8, eps=1e-4, G=G))
    assert np.median(rel_err(a32, a64)) < 1e-6


def test_verlet_steps_with_group_walk(ctx):
    """The accel cache is keyed by the flags: a group-walk run after a
    per-body run recomputes a(x0)."""
    pos, vel, m = ics.plummer(4096, seed=2)
    pb = make_params(1.0, 0.01, 0.5, BARNES_HUT, F64, 8)
    pg = gw(0.5, F64, 8)
    ctx.upload(pos, vel, m)
    ctx.gravity_accel(pb, download=False)
    ctx.verlet_steps(pg, 1e-3, 3)
    xa, va, _ = ctx.download()
    ctx.upload(pos, vel, m)
    ctx.verlet_steps(pg, 1e-3, 3)
    xb, vb, _ = ctx.download()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


@pytest.mark.parametrize("method,precision", [(BARNES_HUT, F64_EXACT), (DIRECT, F64),
                                              (DIRECT, F32C)])
def test_flag_rejected_outside_bh_f64_f32c(ctx, method, precision):
    pos, _, m = ics.plummer(100, seed=1)
    ctx.upload(pos, None, m)
    with pytest.raises(physgpu.PhysError) as ei:
        ctx.gravity_forces(make_params(1.0, 0.01, 0.5, method, precision, 1, GROUP_WALK))
    assert ei.value.status == physgpu.ERR_ARG
    with pytest.raises(physgpu.PhysError):
        ctx.gravity_forces(make_params(1.0, 0.01, 0.5, BARNES_HUT, F64, 1, 2))


def test_mirror_system_group_walk_theta_zero(ctx):
    """barnes_hut_gravity_system(group_walk=True) at theta = 0 adds the direct
    sum to Force (SI units, sector-flattened positions)."""
    rng = np.random.default_rng(12)
    wb, wd = physgpu.World(), physgpu.World()
    for _ in range(300):
        mm, p = 10 ** rng.uniform(20, 26), rng.normal(scale=1e9, size=3)
        wb.spawn(mm, p)
        wd.spawn(mm, p)
    cfg = physgpu.UniverseConfig(softening_epsilon=1e-4, barnes_hut_theta=0.0)
    physgpu.barnes_hut_gravity_system(wb, cfg, precision=F64, leaf_cap=8, ctx=ctx,
                                      group_walk=True)
    physgpu.brute_force_gravity_system(wd, cfg, precision=F64, ctx=ctx)
    assert rel_err(wb.force, wd.force).max() < 1e-12


@pytest.mark.parametrize("leaf_cap", [8, 16])
def test_lists_do_not_depend_on_scheduling(ctx, leaf_cap):
    """At 300 001 bodies a list warp's pool region holds about one group's
    list, so which groups a warp takes decides whether its region fills;
    a warp then continues in a spill region instead of re-queueing, so every
    run builds the same lists: identical forces and interaction counts from
    run to run, and the same count for F32C and F64."""
    pos, _, m = ics.plummer(300001, seed=3)
    ctx.upload(pos, None, m)
    counts = {}
    for prec in (F64, F32C):
        p = make_params(1.0, 0.01, 0.5, BARNES_HUT, prec, leaf_cap, GROUP_WALK)
        a1 = ctx.gravity_accel(p)
        n1 = ctx.timings()["interactions"]
        a2 = ctx.gravity_accel(p)
        n2 = ctx.timings()["interactions"]
        assert np.array_equal(a1, a2) and n1 == n2
        counts[prec] = n1
    assert counts[F64] == counts[F32C]
