"""Seeded synthetic initial conditions for the gravity workloads.

The reference ships no scenario generators for these shapes (its scenarios are
hand-placed bodies, src/scenarios/test_demo.rs:9-60), so the particle sets are
defined here.  All generators use numpy's PCG64 (`np.random.default_rng(seed)`)
and return float64 arrays in G = 1 units unless stated.
"""
import math

import numpy as np


def _isotropic(rng, n):
    """Unit vectors uniform on the sphere."""
    cz = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2.0 * math.pi, n)
    sz = np.sqrt(1.0 - cz * cz)
    return np.stack([sz * np.cos(ph), sz * np.sin(ph), cz], axis=1)


def plummer(n, seed=0, a=1.0, total_mass=1.0, G=1.0, mfrac_max=0.999, center=True):
    """Equal-mass Plummer sphere (Aarseth, Henon & Wielen 1974).

    Radii come from the cumulative mass M(<r)/M = r^3 / (r^2 + a^2)^{3/2}
    inverted at a uniform mass fraction X in (0, mfrac_max]; the cut
    mfrac_max = 0.999 keeps r <= 38.7 a.  Speeds are q * v_esc(r) with
    v_esc = sqrt(2 G M) (r^2 + a^2)^{-1/4} and q drawn from
    g(q) ~ q^2 (1 - q^2)^{7/2} by von Neumann rejection; directions are
    isotropic.  With `center` the centre-of-mass position and velocity are
    subtracted.  Returns (pos (n,3), vel (n,3), mass (n,)).
    """
    rng = np.random.default_rng(seed)
    X = rng.uniform(0.0, mfrac_max, n)
    X = np.maximum(X, 1e-300)
    r = a / np.sqrt(X ** (-2.0 / 3.0) - 1.0)
    pos = r[:, None] * _isotropic(rng, n)
    q = np.empty(n)
    filled = 0
    while filled < n:
        k = max(1024, 2 * (n - filled) * 11 // 10)
        qq = rng.uniform(0.0, 1.0, k)
        yy = rng.uniform(0.0, 0.1, k)
        ok = qq[yy < qq * qq * (1.0 - qq * qq) ** 3.5]
        take = min(ok.shape[0], n - filled)
        q[filled:filled + take] = ok[:take]
        filled += take
    vesc = math.sqrt(2.0 * G * total_mass) * (r * r + a * a) ** -0.25
    vel = (q * vesc)[:, None] * _isotropic(rng, n)
    m = np.full(n, total_mass / n)
    if center:
        pos -= np.average(pos, axis=0, weights=m)
        vel -= np.average(vel, axis=0, weights=m)
    return np.ascontiguousarray(pos), np.ascontiguousarray(vel), m


def golden_spiral(n, sigma=100.0, mass=1e10):
    """The deterministic body set of the reference bench
    (tests/gpu_bench.rs:43-62): golden-angle spiral, radius sigma * i^0.333,
    mass 1e10 each, zero velocity (SI units, G = 6.67430e-11)."""
    i = np.arange(n, dtype=np.float64)
    th = i * 2.0 * math.pi * 0.618033988749895
    ph = np.arccos(np.cos(i * math.pi * 0.618033988749895))
    r = sigma * np.power(i, 0.333)
    pos = np.stack([r * np.sin(ph) * np.cos(th), r * np.sin(ph) * np.sin(th), r * np.cos(ph)],
                   axis=1)
    return np.ascontiguousarray(pos), np.zeros((n, 3)), np.full(n, mass)


def ensemble(nsys, seed=0, nmin=3, nmax=64, mmin=0.1, mmax=10.0, G=1.0, Q=0.5):
    """Independent small systems in CSR layout.

    Per system: N ~ U{nmin..nmax}; masses log-uniform in [mmin, mmax];
    positions uniform in the unit ball; velocities isotropic Gaussian, then in
    the system's centre-of-mass frame (positions and velocities) scaled so the
    virial ratio Q = K / |W| equals `Q`, with K = sum 1/2 m v^2 and
    W = -sum_{i<j} G m_i m_j / r_ij (unsoftened).
    Returns (offsets (nsys+1,), pos, vel, mass).
    """
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, nsys)
    off = np.zeros(nsys + 1, np.int64)
    off[1:] = np.cumsum(ns)
    n = int(off[-1])
    m = np.exp(rng.uniform(math.log(mmin), math.log(mmax), n))
    u = rng.uniform(0.0, 1.0, n) ** (1.0 / 3.0)
    pos = u[:, None] * _isotropic(rng, n)
    vel = rng.normal(0.0, 1.0, (n, 3))
    for s in range(nsys):
        b, e = off[s], off[s + 1]
        mm = m[b:e]
        p = pos[b:e]
        v = vel[b:e]
        p -= np.average(p, axis=0, weights=mm)
        v -= np.average(v, axis=0, weights=mm)
        d = p[:, None, :] - p[None, :, :]
        r = np.sqrt((d * d).sum(-1))
        iu = np.triu_indices(e - b, 1)
        W = -G * np.sum(mm[iu[0]] * mm[iu[1]] / r[iu])
        K = 0.5 * np.sum(mm * (v * v).sum(1))
        v *= math.sqrt(Q * abs(W) / K)
    return off, np.ascontiguousarray(pos), np.ascontiguousarray(vel), m


def _inverse_cdf(cdf, x, u):
    return np.interp(u, cdf, x)


def galaxy(n, seed=0, disk_frac=0.3, Rd=1.0, z0=0.1, c=10.0, rs=3.0, rcut_rs=10.0,
           total_mass=1.0, G=1.0):
    """Disk + NFW halo galaxy model.

    disk_frac of the mass in an exponential disk (scale length Rd, sech^2
    vertical profile of scale z0), the rest in an NFW halo of scale radius rs
    truncated at rcut_rs * rs (concentration c sets r_200 = c * rs, used only
    to name the model).  Particle counts follow the mass split, so particles
    are equal-mass within each component.  The halo radius comes from
    M(<r) ~ ln(1 + r/rs) - (r/rs)/(1 + r/rs) (the enclosed-mass form of the
    reference's nfw_enclosed_mass, src/physics/nfw.rs:76-83), inverted
    numerically.  Disk bodies move on circular orbits with
    v_c^2 = G M(<r) / r from the spherically averaged enclosed mass of both
    components; halo velocities are isotropic Gaussian with
    sigma^2 = v_c^2 / 3.  Returns (pos, vel, mass).
    """
    del c
    rng = np.random.default_rng(seed)
    nd = int(round(n * disk_frac))
    nh = n - nd
    Md, Mh = total_mass * disk_frac, total_mass - total_mass * disk_frac
    # Disk radii: M(<R)/Md = 1 - (1 + R/Rd) exp(-R/Rd), tabulated to 40 Rd.
    Rt = np.linspace(0.0, 40.0 * Rd, 200001)
    cdf_d = 1.0 - (1.0 + Rt / Rd) * np.exp(-Rt / Rd)
    R = _inverse_cdf(cdf_d, Rt, rng.uniform(0.0, cdf_d[-1], nd))
    phi = rng.uniform(0.0, 2.0 * math.pi, nd)
    zz = z0 * np.arctanh(rng.uniform(-1.0, 1.0, nd) * (1.0 - 1e-12))
    dpos = np.stack([R * np.cos(phi), R * np.sin(phi), zz], axis=1)
    # Halo radii from the truncated NFW enclosed mass.
    xt = np.linspace(0.0, rcut_rs, 200001)
    mx = np.log1p(xt) - xt / (1.0 + xt)
    cdf_h = mx / mx[-1]
    rh = rs * _inverse_cdf(cdf_h, xt, rng.uniform(0.0, 1.0, nh))
    hpos = rh[:, None] * _isotropic(rng, nh)

    def menc(r):
        md = Md * np.interp(r, Rt, cdf_d)
        mh = Mh * np.interp(r / rs, xt, cdf_h)
        return md + mh

    rdisk = np.sqrt((dpos * dpos).sum(1))
    vc_d = np.sqrt(G * menc(rdisk) / np.maximum(rdisk, 1e-6))
    dvel = np.stack([-vc_d * np.sin(phi), vc_d * np.cos(phi), np.zeros(nd)], axis=1)
    vc_h = np.sqrt(G * menc(rh) / np.maximum(rh, 1e-6))
    hvel = rng.normal(0.0, 1.0, (nh, 3)) * (vc_h / math.sqrt(3.0))[:, None]
    pos = np.concatenate([dpos, hpos])
    vel = np.concatenate([dvel, hvel])
    m = np.concatenate([np.full(nd, Md / max(nd, 1)), np.full(nh, Mh / max(nh, 1))])
    return np.ascontiguousarray(pos), np.ascontiguousarray(vel), m
