"""Barnes-Hut parity (K2-K6) through the C ABI against the oracle's pointer
octree (gravity_tree.rs).

Bar: descent keys, sort order, cell membership, cell mass and centre of
mass and F64_EXACT forces are bit-identical to the oracle; F64 (parallel
centre of mass, FMA, flat sums) within 1e-12 median relative of the
reference; F32C within 1e-6 median relative of F64 on the same tree."""
import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, make_params

pytestmark = pytest.mark.gpu
G_SI = physgpu.G_SI


def rel_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def bh(theta=0.5, precision=F64_EXACT, leaf_cap=1, G=1.0, eps=0.01):
    return make_params(G, eps, theta, BARNES_HUT, precision, leaf_cap)


def dstar_of(half):
    h, d = half, 0
    while not (d >= 40 or h < 1e-8):
        h *= 0.5
        d += 1
    return d


def test_two_bodies_mirror(ctx):
    """gravity_tree.rs:350-416 through the ECS mirror."""
    w = physgpu.World()
    e1 = w.spawn(1e10, [0.0, 0.0, 0.0])
    e2 = w.spawn(2e10, [100.0, 0.0, 0.0])
    cfg = physgpu.UniverseConfig(softening_epsilon=1e-4, barnes_hut_theta=0.5)
    physgpu.barnes_hut_gravity_system(w, cfg, ctx=ctx)
    f1, f2 = w.force[e1], w.force[e2]
    r2 = 1e4
    expected = G_SI * 1e10 * 2e10 * 100.0 / ((r2 + 1e-8) ** 0.5 * (r2 + 1e-8))
    assert f1[0] > 0 and f2[0] < 0
    assert abs(f1[0] - expected) / expected < 1e-10
    assert np.linalg.norm(f1 + f2) < 1e-20
    assert np.array_equal(w.force, oracle.bh_forces(w.local, w.mass, G_SI, 1e-4, 0.5))


def test_theta_zero_equals_brute_force_mirror(ctx):
    """gravity_tree.rs:420-487 through the ECS mirror."""
    pts = [(1e10, [0.0, 0, 0]), (2e10, [100.0, 0, 0]), (3e10, [0, 200.0, 0]),
           (5e10, [150.0, 150.0, 0])]
    wb, wd = physgpu.World(), physgpu.World()
    for mm, p in pts:
        wb.spawn(mm, p)
        wd.spawn(mm, p)
    cfg = physgpu.UniverseConfig(softening_epsilon=1e-4, barnes_hut_theta=0.0)
    physgpu.barnes_hut_gravity_system(wb, cfg, ctx=ctx)
    physgpu.brute_force_gravity_system(wd, cfg, ctx=ctx)
    assert rel_err(wb.force, wd.force).max() < 1e-8


def test_bounded_error_mirror(ctx):
    """gravity_tree.rs:491-556 through the ECS mirror."""
    w5, w0 = physgpu.World(), physgpu.World()
    for i in range(4):
        for j in range(4):
            w5.spawn(1e8, [i * 10.0, j * 10.0, 0.0])
            w0.spawn(1e8, [i * 10.0, j * 10.0, 0.0])
    w5.spawn(5e10, [1000.0, 0, 0])
    w0.spawn(5e10, [1000.0, 0, 0])
    physgpu.barnes_hut_gravity_system(w5, physgpu.UniverseConfig(barnes_hut_theta=0.5), ctx=ctx)
    physgpu.barnes_hut_gravity_system(w0, physgpu.UniverseConfig(barnes_hut_theta=0.0), ctx=ctx)
    assert rel_err(w5.force[-1:], w0.force[-1:])[0] < 0.05


def structure_check(ctx, pos, m):
    ctx.upload(pos, None, m)
    g = ctx.bh_export(bh(precision=F64_EXACT))
    o = oracle.bh_export(pos, m)
    assert np.array_equal(g["root"], o["root"])
    assert g["nnodes"] == len(o["depth"])
    assert np.array_equal(g["depth"], o["depth"])
    assert np.array_equal(g["count"], o["count"])
    assert np.array_equal(g["leaf_body"], o["leaf_body"])
    assert np.array_equal(g["body_leaf"], o["body_leaf"])
    assert np.array_equal(g["mass"], o["mass"])        # insertion-order mass sums
    assert np.array_equal(g["com"], o["com"])          # running-mean centre of mass
    D = dstar_of(o["root"][3])
    hi, lo = oracle.descent_keys(pos, o["root"], D)
    assert np.array_equal(g["keys_hi"], hi) and np.array_equal(g["keys_lo"], lo)
    order = np.lexsort((np.arange(len(m)), lo, hi))
    assert np.array_equal(g["perm"], order)
    return g


@pytest.mark.parametrize("n,seed", [(2, 0), (3, 1), (9, 2), (100, 3), (1000, 4), (20000, 5)])
def test_tree_matches_reference_octree(ctx, n, seed):
    pos, _, m = ics.plummer(n, seed=seed)
    structure_check(ctx, pos, m)


def test_tree_reference_bench_fixture(ctx):
    """The reference bench's golden-angle spiral (tests/gpu_bench.rs:43-62)."""
    pos, _, m = ics.golden_spiral(5000)
    structure_check(ctx, pos, m)


def test_tree_coincident_and_clustered(ctx):
    """Co-located bodies (guard leaves at D*), exact duplicates, bodies on cell
    boundaries, a tight pair forcing a deep chain, unequal masses."""
    rng = np.random.default_rng(7)
    base = rng.normal(0, 1, (300, 3))
    dup = np.repeat(base[:5], 4, axis=0)
    tight = np.array([[0.3, 0.3, 0.3], [0.3 + 1e-12, 0.3, 0.3]])
    grid = np.array([[i, j, k] for i in range(-2, 3) for j in range(-2, 3) for k in range(-2, 3)],
                    float)
    pos = np.concatenate([base, dup, tight, grid])
    m = rng.uniform(0.1, 3.0, len(pos))
    g = structure_check(ctx, pos, m)
    assert (g["count"][g["leaf_body"] >= 0] > 1).any()  # some guard leaves exist


def test_sort_fixup_long_runs(ctx):
    """Many bodies sharing their first 21 octants (equal hi keys): the run
    fixup must order them by the deeper octants, then by index."""
    rng = np.random.default_rng(8)
    far = rng.normal(0, 1e3, (50, 3))
    blob = 1e-4 * rng.uniform(-1, 1, (400, 3)) + 1.0
    pos = np.concatenate([far, blob, blob[:40]])
    m = rng.uniform(0.5, 1.5, len(pos))
    structure_check(ctx, pos, m)


@pytest.mark.parametrize("n", [1 << 20, 300_001])
def test_sort_many_tiles(ctx, n):
    """The key sort over hundreds of 2048-key tiles (every pass is one kernel
    whose tiles take their offsets from the tiles before them): the
    permutation is the stable order of the (hi, lo) descent keys."""
    pos, _, m = ics.plummer(n, seed=11)
    ctx.upload(pos, None, m)
    g = ctx.bh_export(bh(precision=F64))
    hi, lo = g["keys_hi"], g["keys_lo"]
    assert np.array_equal(g["perm"], np.lexsort((np.arange(n), lo, hi)))


@pytest.mark.parametrize("n,theta,seed", [(1000, 0.5, 1), (4096, 0.5, 2), (4096, 0.0, 3),
                                          (4096, 1.0, 4), (30000, 0.5, 5)])
def test_exact_forces_bitexact(ctx, n, theta, seed):
    pos, _, m = ics.plummer(n, seed=seed)
    ctx.upload(pos, None, m)
    f = ctx.gravity_forces(bh(theta, F64_EXACT))
    ref = oracle.bh_forces(pos, m, 1.0, 0.01, theta)
    assert np.array_equal(f, ref)


def test_exact_forces_bitexact_si_fixture(ctx):
    """Reference bench fixture in SI units (G, eps = 1e-4, mass 1e10)."""
    pos, _, m = ics.golden_spiral(3000)
    ctx.upload(pos, None, m)
    f = ctx.gravity_forces(make_params(G_SI, 1e-4, 0.5, BARNES_HUT, F64_EXACT))
    assert np.array_equal(f, oracle.bh_forces(pos, m, G_SI, 1e-4, 0.5))


def test_exact_forces_coincident(ctx):
    rng = np.random.default_rng(3)
    base = rng.normal(0, 1, (500, 3))
    pos = np.concatenate([base, base[:20], base[:3]])
    m = rng.uniform(0.5, 1.5, len(pos))
    ctx.upload(pos, None, m)
    f = ctx.gravity_forces(bh(0.5, F64_EXACT))
    assert np.array_equal(f, oracle.bh_forces(pos, m, 1.0, 0.01, 0.5))


@pytest.mark.parametrize("kind", ["tiny", "mixed"])
def test_exact_com_outside_reciprocal_range(ctx, kind):
    """The centre-of-mass chains divide through a reciprocal while the running
    mass and the numerators lie in [2^-500, 2^501); a cell that leaves that
    range is rerun with the IEEE division.  Masses near 1e-160 send every
    chain there ("tiny"), every other body's ("mixed") only the cells whose
    first inserted body is one of them.  20 000 bodies: cells of more than
    2048 bodies take the warp form, the rest the thread form.  Tree and
    forces stay bit-identical to the oracle (G = 1e300 keeps the tiny
    masses' pair terms normal)."""
    pos, _, m = ics.plummer(20000, seed=21)
    m = m.copy()
    if kind == "tiny":
        m *= 1e-160
        G = 1e300
    else:
        m[::2] *= 1e-160
        G = 1.0
    g = structure_check(ctx, pos, m)
    assert (g["count"] >= 2048).any()
    f = ctx.gravity_forces(bh(0.5, F64_EXACT, G=G))
    ref = oracle.bh_forces(pos, m, G, 0.01, 0.5)
    assert np.isfinite(ref).all() and (ref != 0).any()
    assert np.array_equal(f, ref)


@pytest.mark.parametrize("n", [4096, 65536])
def test_f64_close_to_reference(ctx, n):
    pos, _, m = ics.plummer(n, seed=n)
    ctx.upload(pos, None, m)
    f = ctx.gravity_forces(bh(0.5, F64))
    ref = oracle.bh_forces(pos, m, 1.0, 0.01, 0.5)
    e = rel_err(f, ref)
    assert np.median(e) <= 1e-12, np.median(e)
    assert np.mean(e > 1e-9) < 1e-3  # near-tie opening flips only


@pytest.mark.parametrize("leaf_cap", [1, 8])
def test_f32c_vs_f64_same_tree(ctx, leaf_cap):
    pos, _, m = ics.plummer(65536, seed=17)
    ctx.upload(pos, None, m)
    a64 = ctx.gravity_accel(bh(0.5, F64, leaf_cap))
    a32 = ctx.gravity_accel(bh(0.5, F32C, leaf_cap))
    e = rel_err(a32, a64)
    assert np.median(e) <= 1e-6, np.median(e)


@pytest.mark.parametrize("leaf_cap", [2, 8, 16])
def test_bucket_leaves(ctx, leaf_cap):
    """theta = 0 opens every cell: bucket-leaf BH equals the direct sum up to
    summation order; theta = 0.5 stays within the usual BH error."""
    pos, _, m = ics.plummer(5000, seed=leaf_cap)
    ctx.upload(pos, None, m)
    ref = oracle.direct_forces(pos, m, 1.0, 0.01)
    f0 = ctx.gravity_forces(bh(0.0, F64, leaf_cap))
    assert rel_err(f0, ref).max() < 1e-12
    f5 = ctx.gravity_forces(bh(0.5, F64, leaf_cap))
    assert np.median(rel_err(f5, ref)) < 1e-2


def test_interaction_count(ctx):
    """theta = 0: every lane interacts with every other body exactly once."""
    pos, _, m = ics.plummer(3000, seed=4)
    ctx.upload(pos, None, m)
    ctx.gravity_forces(bh(0.0, F64))
    assert ctx.timings()["interactions"] == 3000 * 2999
    ctx.gravity_forces(bh(0.0, F32C, 8))
    assert ctx.timings()["interactions"] == 3000 * 2999
