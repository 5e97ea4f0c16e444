"""Pins the CPU oracle to the reference's own known-answer tests.

Each test re-runs a unit test of the reference (same bodies, same config,
same tolerance) against the oracle's restatement of that code.  The reference
itself (Rust) cannot be built here, so these tests are the oracle's anchor.
"""
import math

import numpy as np
import pytest

import oracle

G = 6.67430e-11  # src/core/constants.rs:7


def test_figure_8_stability():
    """src/physics/gravity.rs:81-103: three equal masses, eps = 0."""
    pos = np.array([[-0.97000436, 0.24308753, 0.0], [0.97000436, -0.24308753, 0.0], [0, 0, 0]])
    f = oracle.direct_forces(pos, np.ones(3), G, 0.0)
    assert np.all(np.isfinite(f))
    assert abs(f[:, 0].sum()) < 1e-10
    assert abs(f[:, 1].sum()) < 1e-10


def test_kepler_orbit_period():
    """src/physics/gravity.rs:106-130: 1e12 kg and 1 kg at r = 100, eps = 0."""
    pos = np.array([[0.0, 0.0, 0.0], [100.0, 0.0, 0.0]])
    f = oracle.direct_forces(pos, np.array([1e12, 1.0]), G, 0.0)
    expected = -(G * 1e12 * 1.0) / (100.0 * 100.0)
    assert abs(f[1, 0] - expected) < 1e-10
    assert f[1, 1] == 0.0 and f[1, 2] == 0.0


def test_barnes_hut_matches_brute_force_two_bodies():
    """src/physics/gravity_tree.rs:350-416."""
    eps = 1e-4
    pos = np.array([[0.0, 0.0, 0.0], [100.0, 0.0, 0.0]])
    m = np.array([1e10, 2e10])
    f = oracle.bh_forces(pos, m, G, eps, 0.5)
    r2 = 100.0 * 100.0
    s3 = math.sqrt(r2 + eps * eps) * (r2 + eps * eps)
    expected = G * 1e10 * 2e10 * 100.0 / s3
    assert f[0, 0] > 0 and f[1, 0] < 0
    assert abs(f[0, 0] - expected) / expected < 1e-10
    assert np.linalg.norm(f[0] + f[1]) < 1e-20


def test_barnes_hut_theta_zero_equals_brute_force():
    """src/physics/gravity_tree.rs:420-487."""
    pos = np.array([[0.0, 0, 0], [100.0, 0, 0], [0, 200.0, 0], [150.0, 150.0, 0]])
    m = np.array([1e10, 2e10, 3e10, 5e10])
    fb = oracle.bh_forces(pos, m, G, 1e-4, 0.0)
    fd = oracle.direct_forces(pos, m, G, 1e-4)
    for i in range(4):
        rel = np.linalg.norm(fb[i] - fd[i]) / max(np.linalg.norm(fd[i]), 1e-30)
        assert rel < 1e-8


def test_barnes_hut_approximation_bounded_error():
    """src/physics/gravity_tree.rs:491-556: 4x4 grid + distant body."""
    pos = [[i * 10.0, j * 10.0, 0.0] for i in range(4) for j in range(4)] + [[1000.0, 0, 0]]
    m = [1e8] * 16 + [5e10]
    pos, m = np.array(pos), np.array(m)
    f5 = oracle.bh_forces(pos, m, G, 1e-4, 0.5)
    f0 = oracle.bh_forces(pos, m, G, 1e-4, 0.0)
    rel = np.linalg.norm(f5[-1] - f0[-1]) / max(np.linalg.norm(f0[-1]), 1e-30)
    assert rel < 0.05


def test_verlet_energy_conservation_circular_orbit():
    """src/physics/integrators.rs:288-348: GM = 1 circular orbit, dt = 1e-3,
    6283 steps, a = -r/|r|^3 recomputed between the position and velocity
    systems; energy drift < 1e-4."""
    L = oracle.lib()
    p = [np.array([1.0]), np.array([0.0]), np.array([0.0])]
    v = [np.array([0.0]), np.array([1.0]), np.array([0.0])]
    a = [np.array([-1.0]), np.array([0.0]), np.array([0.0])]
    pa = [np.array([-1.0]), np.array([0.0]), np.array([0.0])]
    ptr = oracle._p
    dt = 0.001
    for _ in range(6283):
        L.oracle_vv_position(1, dt, *[ptr(q) for q in p], *[ptr(q) for q in v],
                             *[ptr(q) for q in a], *[ptr(q) for q in pa])
        r = np.array([p[0][0], p[1][0], p[2][0]])
        rm = math.sqrt(float(r @ r))
        acc = -r / (rm * rm * rm)
        for k in range(3):
            a[k][0] = acc[k]
        L.oracle_vv_velocity(1, dt, *[ptr(q) for q in v], *[ptr(q) for q in a],
                             *[ptr(q) for q in pa])
    vv = np.array([v[0][0], v[1][0], v[2][0]])
    rr = np.array([p[0][0], p[1][0], p[2][0]])
    e = 0.5 * float(vv @ vv) - 1.0 / math.sqrt(float(rr @ rr))
    assert abs(e - (-0.5)) < 1e-4


def test_flatten_uses_first_body_sector():
    """gravity.rs:38-47 vs the BH system's per-body origin (gravity_tree.rs:280-291)."""
    sec = np.array([[1, 0, 0], [2, 0, 0], [1, -1, 0]], np.int64)
    loc = np.array([[0.5, 1.0, -2.0], [0.25, 0.0, 0.0], [0.0, 3.0, 1.0]])
    x = oracle.flatten(sec, loc, 1e12)
    assert x[1, 0] == 1e12 + 0.25 and x[2, 1] == -1e12 + 3.0 and x[0, 0] == 0.5
    xq = oracle.flatten(sec, loc, 1e12, bh_quirk=True)
    assert np.array_equal(xq, loc + 0.0)


def test_theta_zero_bh_close_to_direct_plummer():
    """theta = 0 opens every cell: BH equals the direct sum up to summation order."""
    import physgpu.ics as ics
    pos, vel, m = ics.plummer(512, seed=3)
    fb = oracle.bh_forces(pos, m, 1.0, 0.01, 0.0)
    fd = oracle.direct_forces(pos, m, 1.0, 0.01)
    rel = np.linalg.norm(fb - fd, axis=1) / np.linalg.norm(fd, axis=1)
    assert rel.max() < 1e-12


def test_descent_keys_match_tree_paths():
    """The per-level descent (x >= c, c +/- h/2 in f64) reproduces the pointer
    octree's cell membership: bodies sharing a leaf share their key prefix up
    to the leaf depth, and pre-order leaves come in key order."""
    import physgpu.ics as ics
    pos, vel, m = ics.plummer(2000, seed=5)
    ex = oracle.bh_export(pos, m)
    hi, lo = oracle.descent_keys(pos, ex["root"], 40)
    leaves = np.where(ex["leaf_body"] >= 0)[0]
    order = ex["leaf_body"][leaves]
    keys = [(int(hi[b]), int(lo[b])) for b in order]
    assert keys == sorted(keys)
    assert np.all(ex["body_leaf"] >= 0)


def test_energy_diagnostics_oracle():
    """energy.rs:21-56 on two bodies: KE = 1/2 m v^2, PE = -G m1 m2 / r."""
    pos = np.array([[0.0, 0, 0], [3.0, 4.0, 0]])
    vel = np.array([[1.0, 0, 0], [0, 2.0, 0]])
    m = np.array([2.0, 3.0])
    out = oracle.energy(pos, vel, m, 1.0)
    assert out[0] == 0.5 * 2.0 * 1.0 + 0.5 * 3.0 * 4.0
    assert out[1] == -(1.0 * 2.0 * 3.0) / 5.0
    assert np.allclose(out[2:], [2.0, 6.0, 0.0])


def test_guard_leaf_keeps_last_body():
    """Co-located bodies end in a guard leaf that stores the last inserted
    body while its mass counts all of them (gravity_tree.rs:113-126)."""
    pos = np.array([[0.0, 0, 0], [1.0, 1.0, 1.0], [1.0, 1.0, 1.0], [1.0, 1.0, 1.0]])
    m = np.array([1.0, 2.0, 3.0, 4.0])
    ex = oracle.bh_export(pos, m)
    guard = np.where((ex["leaf_body"] >= 0) & (ex["count"] == 3))[0]
    assert len(guard) == 1
    g = guard[0]
    assert ex["leaf_body"][g] == 3 and ex["mass"][g] == 9.0
    assert ex["depth"][g] in (27, 28, 40)


# ---- src/physics/nfw.rs:150-238, against the oracle and the library's host
# scalars (the C ABI's phys_nfw_*; no GPU needed) ----
def _nfw_impls():
    import physgpu
    return [("oracle", oracle.nfw_density, oracle.nfw_enclosed_mass,
             oracle.nfw_circular_velocity),
            ("library", physgpu.nfw_density, physgpu.nfw_enclosed_mass,
             physgpu.nfw_circular_velocity)]


def test_nfw_density_at_scale_radius():
    """nfw.rs:150-162: rho(Rs) = rho_0 / 4."""
    for name, dens, _, _ in _nfw_impls():
        assert abs(dens(1.0, 1.0, 1.0) - 0.25) < 1e-12, name


def test_nfw_inner_profile():
    """nfw.rs:164-182: rho ~ 1/r for r << Rs."""
    for name, dens, _, _ in _nfw_impls():
        ratio = dens(0.01, 1.0, 100.0) / dens(0.02, 1.0, 100.0)
        assert abs(ratio - 2.0) < 0.01, name


def test_nfw_flat_rotation_curve():
    """nfw.rs:184-213: v_c changes by < 30 % between 5, 10, 20, 50, 100 Rs."""
    rho_0, rs = 1e-21, 1e20
    for name, _, _, vc in _nfw_impls():
        v = [vc(k * rs, rho_0, rs) for k in (5.0, 10.0, 20.0, 50.0, 100.0)]
        for i in range(1, len(v)):
            assert abs(v[i] - v[i - 1]) / v[i - 1] < 0.3, name
        assert all(x > 0 for x in v), name


def test_nfw_enclosed_mass_monotonic():
    """nfw.rs:215-237."""
    for name, _, mass, _ in _nfw_impls():
        ms = [mass(r, 1.0, 1.0) for r in (0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 100.0)]
        assert all(b > a for a, b in zip(ms, ms[1:])), name


def test_nfw_scalars_library_equals_oracle():
    """The library's host scalars restate nfw.rs with the same operation
    order as the oracle: identical results, including the r <= 0 and Rs <= 0
    cases."""
    import physgpu
    rng = np.random.default_rng(3)
    for r, rho, rs in zip(10 ** rng.uniform(-3, 3, 200), 10 ** rng.uniform(-25, 2, 200),
                          10 ** rng.uniform(-2, 21, 200)):
        r = r * rs
        assert physgpu.nfw_density(r, rho, rs) == oracle.nfw_density(r, rho, rs)
        assert physgpu.nfw_enclosed_mass(r, rho, rs) == oracle.nfw_enclosed_mass(r, rho, rs)
        assert (physgpu.nfw_circular_velocity(r, rho, rs)
                == oracle.nfw_circular_velocity(r, rho, rs))
    for f in (physgpu.nfw_density, physgpu.nfw_enclosed_mass):
        assert f(0.0, 1.0, 1.0) == 0.0 and f(-1.0, 1.0, 1.0) == 0.0 and f(1.0, 1.0, 0.0) == 0.0


def test_nfw_oracle_force_matches_enclosed_mass():
    """nfw_gravity_system: |F| = G M(r) m / r^2 toward the centre; a body at
    the centre is skipped."""
    pos = np.array([[3e20, 4e20, 0.0], [0.0, 0.0, 0.0], [1.0, 2.0, 2.0]])
    m = np.array([2e30, 1e30, 5.0])
    halo = (1.4e-21, 6.17e20, 0.0, 0.0, 0.0)
    f = oracle.nfw_forces(pos, m, halo)
    r = 5e20
    mag = G * oracle.nfw_enclosed_mass(r, 1.4e-21, 6.17e20) * 2e30 / (r * r)
    assert np.allclose(f[0], [-0.6 * mag, -0.8 * mag, 0.0], rtol=1e-14)
    assert not f[1].any()
    assert np.all(np.isfinite(f[2])) and np.linalg.norm(f[2]) > 0


def test_normalize_wraps_sector_oracle():
    """coordinates.rs:136-157: 1.2e12 -> sector 1, -1.2e12 -> sector -1, local
    within half a sector (sector_size 1e12)."""
    s, l, ch = oracle.normalize(np.zeros((2, 3), np.int64),
                                np.array([[1.2e12, 0, 0], [-1.2e12, 0, 0]]), 1e12)
    assert ch and s[0, 0] == 1 and s[1, 0] == -1
    assert np.all(np.abs(l[:, 0]) < 0.5e12 + 1.0)
    assert l[0, 0] == 1.2e12 - 1e12 and l[1, 0] == -1.2e12 + 1e12
    # half-way rounds away from zero (f64::round); in range: untouched
    s, l, ch = oracle.normalize(np.zeros((2, 3), np.int64),
                                np.array([[0.5e12, -0.5e12, 0.4e12], [1.0, 2.0, 3.0]]), 1e12)
    assert list(s[0]) == [1, -1, 0] and list(s[1]) == [0, 0, 0]
    assert list(l[0]) == [-0.5e12, 0.5e12, 0.4e12]
