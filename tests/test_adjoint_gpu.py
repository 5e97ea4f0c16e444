"""Trajectory gradients (K9) through the C ABI.

Bar: the hand-written adjoint agrees with central finite differences of the
same f64 forward pass to 1e-5 relative, per coordinate (floor: 1e-3 of the
largest entry of that gradient, for entries near zero).  Positions and
velocities use h = 1e-6.  Masses use a relative step of 1e-3: dL/dm is
~1e-7 here, so a 1e-6 relative step moves the loss by less than its own f64
rounding (the difference quotient is then noise at the 1e-3 level), while
the loss is smooth enough in m that the 1e-3 step's truncation error stays
below 1e-5.  The checkpoint interval does not change the result."""
import numpy as np
import pytest

import physgpu
import physgpu.ics as ics
from physgpu import F32C, F64, make_params

pytestmark = pytest.mark.gpu
TOL = 1e-5


def setup_case(ctx, n, seed, nsteps, dt, eps):
    pos, vel, m = ics.plummer(n, seed=seed)
    p = make_params(1.0, eps, precision=F64)
    rng = np.random.default_rng(seed + 100)
    ctx.upload(pos, vel + rng.normal(0.0, 0.01, vel.shape), m)
    _, targets = ctx.trajectory_loss(p, dt, nsteps, np.zeros((n, 3)), final=True)
    ctx.upload(pos, vel, m)
    return pos, vel, m, p, targets


def fd_check(ctx, pos, vel, m, p, dt, nsteps, targets, grads, picks, h=1e-6, hm=1e-3):
    gx, gv, gm = grads
    worst = 0.0
    scale = {"x": np.abs(gx).max(), "v": np.abs(gv).max(), "m": np.abs(gm).max()}
    for kind, i, c in picks:
        P, V, M = pos.copy(), vel.copy(), m.copy()
        hh = hm * M[i] if kind == "m" else h
        arr = {"x": P, "v": V, "m": M}[kind]
        idx = (i, c) if kind != "m" else i
        arr[idx] += hh
        ctx.upload(P, V, M)
        lp = ctx.trajectory_loss(p, dt, nsteps, targets)
        arr[idx] -= 2 * hh
        ctx.upload(P, V, M)
        lm = ctx.trajectory_loss(p, dt, nsteps, targets)
        fd = (lp - lm) / (2 * hh)
        g = {"x": gx[i, c] if kind == "x" else 0, "v": gv[i, c] if kind == "v" else 0,
             "m": gm[i] if kind == "m" else 0}[kind]
        err = abs(fd - g) / max(abs(fd), abs(g), 1e-3 * scale[kind])
        worst = max(worst, err)
    ctx.upload(pos, vel, m)
    return worst


def test_adjoint_matches_finite_differences_small(ctx):
    n, nsteps, dt = 64, 30, 1e-3
    pos, vel, m, p, targets = setup_case(ctx, n, 3, nsteps, dt, 0.01)
    loss, gx, gv, gm = ctx.adjoint(p, dt, nsteps, targets, checkpoint=8)
    assert loss > 0 and np.all(np.isfinite(gx)) and np.all(np.isfinite(gm))
    assert loss == ctx.trajectory_loss(p, dt, nsteps, targets)
    rng = np.random.default_rng(0)
    picks = [("x", int(rng.integers(n)), int(rng.integers(3))) for _ in range(6)]
    picks += [("v", int(rng.integers(n)), int(rng.integers(3))) for _ in range(6)]
    picks += [("m", int(rng.integers(n)), 0) for _ in range(4)]
    assert fd_check(ctx, pos, vel, m, p, dt, nsteps, targets, (gx, gv, gm), picks) < TOL


def test_checkpoint_interval_does_not_change_gradients(ctx):
    n, nsteps, dt = 200, 23, 1e-3
    pos, vel, m, p, targets = setup_case(ctx, n, 4, nsteps, dt, 0.01)
    ref = ctx.adjoint(p, dt, nsteps, targets, checkpoint=1)
    for K in (5, 23, 64):
        out = ctx.adjoint(p, dt, nsteps, targets, checkpoint=K)
        assert out[0] == ref[0]
        for a, b in zip(out[1:], ref[1:]):
            assert np.array_equal(a, b)
    # the uploaded state is left untouched
    x, v, _ = ctx.download()
    assert np.array_equal(x, pos) and np.array_equal(v, vel)


def test_zero_steps_gradient_is_analytic(ctx):
    pos, vel, m = ics.plummer(50, seed=9)
    ctx.upload(pos, vel, m)
    tg = pos + 0.1
    loss, gx, gv, gm = ctx.adjoint(make_params(1.0, 0.01, precision=F64), 1e-3, 0, tg)
    assert np.isclose(loss, np.sum((pos - tg) ** 2))
    assert np.allclose(gx, 2 * (pos - tg)) and not gv.any() and not gm.any()


def test_adjoint_workload_shape_finite_differences(ctx):
    """N = 4096 Plummer, 1000 Verlet steps dt = 1e-3, eps = 0.01, targets from
    a forward run with velocities perturbed by N(0, 0.01), checkpoint every
    32 steps, central differences h = 1e-6 on 64 random coordinates."""
    n, nsteps, dt = 4096, 1000, 1e-3
    pos, vel, m, p, targets = setup_case(ctx, n, 1, nsteps, dt, 0.01)
    loss, gx, gv, gm = ctx.adjoint(p, dt, nsteps, targets, checkpoint=32)
    rng = np.random.default_rng(1)
    picks = [(("x", "v")[k % 2], int(rng.integers(n)), int(rng.integers(3))) for k in range(64)]
    picks += [("m", int(rng.integers(n)), 0) for _ in range(8)]
    assert fd_check(ctx, pos, vel, m, p, dt, nsteps, targets, (gx, gv, gm), picks) < TOL


def test_adjoint_rejects_other_precisions(ctx):
    pos, vel, m = ics.plummer(10, seed=1)
    ctx.upload(pos, vel, m)
    with pytest.raises(physgpu.PhysError) as ei:
        ctx.adjoint(make_params(1.0, 0.01, precision=F32C), 1e-3, 2, pos)
    assert ei.value.status == physgpu.ERR_ARG


def test_adjoint_vs_full_difference_gradient(ctx):
    """Brute-force reference gradient: central differences (h = 1e-6) of the
    f64 GPU forward pass over every position and velocity coordinate of a
    48-body system, compared with the adjoint in the 2-norm."""
    n, nsteps, dt = 48, 20, 1e-3
    pos, vel, m, p, targets = setup_case(ctx, n, 6, nsteps, dt, 0.01)
    _, gx, gv, _ = ctx.adjoint(p, dt, nsteps, targets, checkpoint=6)
    h = 1e-6
    fx, fv = np.zeros_like(gx), np.zeros_like(gv)
    for arr_name, out in (("x", fx), ("v", fv)):
        for i in range(n):
            for c in range(3):
                P, V = pos.copy(), vel.copy()
                arr = P if arr_name == "x" else V
                arr[i, c] += h
                ctx.upload(P, V, m)
                lp = ctx.trajectory_loss(p, dt, nsteps, targets)
                arr[i, c] -= 2 * h
                ctx.upload(P, V, m)
                lm = ctx.trajectory_loss(p, dt, nsteps, targets)
                out[i, c] = (lp - lm) / (2 * h)
    ctx.upload(pos, vel, m)
    assert np.linalg.norm(gx - fx) / np.linalg.norm(fx) < 1e-6
    assert np.linalg.norm(gv - fv) / np.linalg.norm(fv) < 1e-6
