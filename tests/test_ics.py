"""Seeded synthetic inputs: shapes, determinism and the stated statistics."""
import numpy as np

import physgpu.ics as ics


def test_plummer_seeded_and_centered():
    p1, v1, m1 = ics.plummer(4096, seed=11)
    p2, v2, m2 = ics.plummer(4096, seed=11)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert p1.shape == (4096, 3) and np.allclose(m1, 1 / 4096)
    assert np.abs(p1.mean(0)).max() < 1e-12 and np.abs(v1.mean(0)).max() < 1e-12
    r = np.linalg.norm(p1, axis=1)
    # half-mass radius of a Plummer sphere with a = 1 is ~1.305
    assert 1.15 < np.median(r) < 1.45
    assert r.max() < 40.0


def test_ensemble_layout_and_virial_ratio():
    off, pos, vel, m = ics.ensemble(64, seed=2)
    ns = np.diff(off)
    assert off[0] == 0 and off[-1] == len(m) and ns.min() >= 3 and ns.max() <= 64
    assert m.min() >= 0.1 and m.max() <= 10.0
    s = 5
    b, e = off[s], off[s + 1]
    mm, p, v = m[b:e], pos[b:e], vel[b:e]
    K = 0.5 * np.sum(mm * (v * v).sum(1))
    d = p[:, None] - p[None]
    r = np.sqrt((d * d).sum(-1))
    iu = np.triu_indices(e - b, 1)
    W = -np.sum(mm[iu[0]] * mm[iu[1]] / r[iu])
    assert abs(K / abs(W) - 0.5) < 1e-9


def test_galaxy_components():
    pos, vel, m = ics.galaxy(20000, seed=1)
    assert pos.shape == (20000, 3)
    nd = 6000
    assert np.allclose(m[:nd], 0.3 / nd) and np.allclose(m[nd:], 0.7 / 14000)
    assert np.abs(pos[:nd, 2]).mean() < 0.2
    assert np.linalg.norm(pos[nd:], axis=1).max() <= 30.0 + 1e-9
