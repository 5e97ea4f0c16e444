"""ctypes wrapper around the C++ oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py.  The product (phys-rs_b200/) never
imports it.  Every function restates the reference's f64 arithmetic; the C++
source cites the reference file:line each one follows.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)
_U64 = ctypes.POINTER(ctypes.c_uint64)


def build():
    """Compile liboracle.so with the committed Makefile (no-op when fresh)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        i64, dbl, cint = ctypes.c_int64, ctypes.c_double, ctypes.c_int
        L.oracle_flatten.argtypes = [i64, _I64, _I64, _I64, _D, _D, _D, dbl, cint, _D, _D, _D]
        L.oracle_direct_forces.argtypes = [i64, _D, _D, _D, _D, dbl, dbl, cint, _D, _D, _D]
        L.oracle_direct_forces_targets.argtypes = [i64, _D, _D, _D, _D, dbl, dbl, i64, _I64,
                                                   cint, _D, _D, _D]
        L.oracle_bh_forces.argtypes = [i64, _D, _D, _D, _D, dbl, dbl, dbl, cint, _D, _D, _D, _D]
        L.oracle_bh_forces_targets.argtypes = [i64, _D, _D, _D, _D, dbl, dbl, dbl, i64, _I64,
                                               cint, _D, _D, _D, _D]
        L.oracle_bh_export.argtypes = [i64, _D, _D, _D, _D, i64, _I32, _I64, _D, _D, _D, _D,
                                       _I64, _I64, _D]
        L.oracle_bh_export.restype = i64
        L.oracle_descent_keys.argtypes = [i64, _D, _D, _D, _D, cint, _U64, _U64]
        L.oracle_accel.argtypes = [i64, _D, _D, _D, _D, _D, _D, _D]
        L.oracle_vv_position.argtypes = [i64, dbl] + [_D] * 12
        L.oracle_vv_velocity.argtypes = [i64, dbl] + [_D] * 9
        L.oracle_vv_run.argtypes = ([i64] + [_D] * 7 + [dbl, dbl, dbl, cint, dbl, i64, cint]
                                    + [_D] * 6)
        L.oracle_vv_run_halo.argtypes = ([i64] + [_D] * 7 + [dbl, dbl, dbl, cint, dbl, i64, cint]
                                         + [_D] * 7)
        L.oracle_energy.argtypes = [i64] + [_D] * 7 + [dbl, _D]
        for f in ("oracle_nfw_density", "oracle_nfw_enclosed_mass",
                  "oracle_nfw_circular_velocity"):
            getattr(L, f).argtypes = [dbl, dbl, dbl]
            getattr(L, f).restype = dbl
        L.oracle_nfw_forces.argtypes = [i64] + [_D] * 4 + [_D] + [_D] * 3
        L.oracle_normalize.argtypes = [i64, _I64, _I64, _I64, _D, _D, _D, dbl]
        L.oracle_normalize.restype = cint
        L.oracle_vv_run_sectors.argtypes = ([i64, _I64, _I64, _I64] + [_D] * 7
                                            + [dbl, dbl, dbl, dbl, cint, dbl, i64, cint]
                                            + [_D] * 7)
        L.oracle_ensemble_run.argtypes = ([i64, _I64] + [_D] * 7 + [dbl, dbl, dbl, i64, cint]
                                          + [_D] * 3)
        _lib = L
    return _lib


def _p(a, ty=_D):
    return a.ctypes.data_as(ty)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ncpu():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def flatten(sectors, local, sector_size, bh_quirk=False):
    """gravity.rs:38-47 (or gravity_tree.rs:280-291 with bh_quirk)."""
    s = np.ascontiguousarray(sectors, dtype=np.int64)
    l = _f64(local)
    n = s.shape[0]
    sx, sy, sz = (np.ascontiguousarray(s[:, k]) for k in range(3))
    lx, ly, lz = (np.ascontiguousarray(l[:, k]) for k in range(3))
    out = [np.empty(n) for _ in range(3)]
    lib().oracle_flatten(n, _p(sx, _I64), _p(sy, _I64), _p(sz, _I64), _p(lx), _p(ly), _p(lz),
                         sector_size, int(bh_quirk), *[_p(o) for o in out])
    return np.stack(out, axis=1)


def direct_forces(pos, m, G, eps, nthreads=None):
    """Forces of brute_force_gravity_system (gravity.rs:53-69), shape (n, 3)."""
    pos, m = _f64(pos), _f64(m)
    n = m.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    f = [np.zeros(n) for _ in range(3)]
    lib().oracle_direct_forces(n, _p(x), _p(y), _p(z), _p(m), G, eps, nthreads or ncpu(),
                               *[_p(a) for a in f])
    return np.stack(f, axis=1)


def direct_forces_targets(pos, m, G, eps, targets, nthreads=None):
    pos, m = _f64(pos), _f64(m)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    n = m.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    f = [np.zeros(t.shape[0]) for _ in range(3)]
    lib().oracle_direct_forces_targets(n, _p(x), _p(y), _p(z), _p(m), G, eps, t.shape[0],
                                       _p(t, _I64), nthreads or ncpu(), *[_p(a) for a in f])
    return np.stack(f, axis=1)


def bh_forces(pos, m, G, eps, theta, nthreads=None, timings=None):
    """Forces of barnes_hut_gravity_system (gravity_tree.rs:305-330), shape (n, 3)."""
    pos, m = _f64(pos), _f64(m)
    n = m.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    f = [np.zeros(n) for _ in range(3)]
    tm = np.zeros(2)
    lib().oracle_bh_forces(n, _p(x), _p(y), _p(z), _p(m), G, eps, theta, nthreads or ncpu(),
                           *[_p(a) for a in f], _p(tm))
    if timings is not None:
        timings[:] = tm
    return np.stack(f, axis=1)


def bh_forces_targets(pos, m, G, eps, theta, targets, nthreads=None):
    """BH forces on a subset of targets; returns (forces, [build_s, walk_s])."""
    pos, m = _f64(pos), _f64(m)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    n = m.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    f = [np.zeros(t.shape[0]) for _ in range(3)]
    tm = np.zeros(2)
    lib().oracle_bh_forces_targets(n, _p(x), _p(y), _p(z), _p(m), G, eps, theta, t.shape[0],
                                   _p(t, _I64), nthreads or ncpu(), *[_p(a) for a in f], _p(tm))
    return np.stack(f, axis=1), tm


def bh_export(pos, m):
    """Pre-order export of the reference octree's non-empty nodes."""
    pos, m = _f64(pos), _f64(m)
    n = m.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    cap = 4 * n + 64
    depth = np.zeros(cap, np.int32)
    count = np.zeros(cap, np.int64)
    mass, cx, cy, cz = (np.zeros(cap) for _ in range(4))
    leaf_body = np.zeros(cap, np.int64)
    body_leaf = np.zeros(n, np.int64)
    root4 = np.zeros(4)
    cnt = lib().oracle_bh_export(n, _p(x), _p(y), _p(z), _p(m), cap, _p(depth, _I32),
                                 _p(count, _I64), _p(mass), _p(cx), _p(cy), _p(cz),
                                 _p(leaf_body, _I64), _p(body_leaf, _I64), _p(root4))
    assert cnt <= cap
    return dict(depth=depth[:cnt], count=count[:cnt], mass=mass[:cnt],
                com=np.stack([cx[:cnt], cy[:cnt], cz[:cnt]], axis=1),
                leaf_body=leaf_body[:cnt], body_leaf=body_leaf, root=root4)


def descent_keys(pos, root4, levels):
    pos = _f64(pos)
    n = pos.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    hi = np.zeros(n, np.uint64)
    lo = np.zeros(n, np.uint64)
    r = _f64(root4)
    lib().oracle_descent_keys(n, _p(x), _p(y), _p(z), _p(r), levels, _p(hi, _U64), _p(lo, _U64))
    return hi, lo


def accel(force, m):
    force, m = _f64(force), _f64(m)
    n = m.shape[0]
    fx, fy, fz = (np.ascontiguousarray(force[:, k]) for k in range(3))
    a = [np.zeros(n) for _ in range(3)]
    lib().oracle_accel(n, _p(fx), _p(fy), _p(fz), _p(m), *[_p(v) for v in a])
    return np.stack(a, axis=1)


def vv_run(pos, vel, m, G, eps, dt, nsteps, method="direct", theta=0.5, acc=None, prev=None,
           nthreads=None, halo=None):
    """The reference's Velocity-Verlet tick loop (src/main.rs:103-140); `halo`
    = (rho_0, Rs, cx, cy, cz) adds nfw_gravity_system to both force passes.

    Returns (pos, vel, acc, prev_acc) after `nsteps` ticks."""
    pos, vel, m = _f64(pos), _f64(vel), _f64(m)
    n = m.shape[0]
    P = [np.ascontiguousarray(pos[:, k]).copy() for k in range(3)]
    V = [np.ascontiguousarray(vel[:, k]).copy() for k in range(3)]
    A = [np.zeros(n) for _ in range(3)] if acc is None else [
        np.ascontiguousarray(acc[:, k], dtype=np.float64).copy() for k in range(3)]
    PA = [np.zeros(n) for _ in range(3)] if prev is None else [
        np.ascontiguousarray(prev[:, k], dtype=np.float64).copy() for k in range(3)]
    H = None if halo is None else _f64(halo)
    lib().oracle_vv_run_halo(n, *[_p(a) for a in P], *[_p(a) for a in V], _p(m), G, eps, theta,
                             0 if method == "direct" else 1, dt, nsteps, nthreads or ncpu(),
                             *[_p(a) for a in A], *[_p(a) for a in PA],
                             None if H is None else _p(H))
    st = lambda L: np.stack(L, axis=1)
    return st(P), st(V), st(A), st(PA)


def energy(pos, vel, m, G):
    """(KE, PE, px, py, pz) per energy.rs:21-56 and integrators.rs:123-129."""
    pos, vel, m = _f64(pos), _f64(vel), _f64(m)
    n = m.shape[0]
    P = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    V = [np.ascontiguousarray(vel[:, k]) for k in range(3)]
    out = np.zeros(5)
    lib().oracle_energy(n, *[_p(a) for a in P], *[_p(a) for a in V], _p(m), G, _p(out))
    return out


def ensemble_run(offsets, pos, vel, m, G, eps, dt, nsteps, nthreads=None):
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    pos, vel, m = _f64(pos), _f64(vel), _f64(m)
    n = m.shape[0]
    P = [np.ascontiguousarray(pos[:, k]).copy() for k in range(3)]
    V = [np.ascontiguousarray(vel[:, k]).copy() for k in range(3)]
    A = [np.zeros(n) for _ in range(3)]
    lib().oracle_ensemble_run(off.shape[0] - 1, _p(off, _I64), *[_p(a) for a in P],
                              *[_p(a) for a in V], _p(m), G, eps, dt, nsteps, nthreads or ncpu(),
                              *[_p(a) for a in A])
    st = lambda L: np.stack(L, axis=1)
    return st(P), st(V), st(A)


def nfw_density(r, rho_0, rs):
    """nfw_density (nfw.rs:61-67)."""
    return lib().oracle_nfw_density(float(r), float(rho_0), float(rs))


def nfw_enclosed_mass(r, rho_0, rs):
    """nfw_enclosed_mass (nfw.rs:76-83)."""
    return lib().oracle_nfw_enclosed_mass(float(r), float(rho_0), float(rs))


def nfw_circular_velocity(r, rho_0, rs):
    """nfw_circular_velocity (nfw.rs:88-91)."""
    return lib().oracle_nfw_circular_velocity(float(r), float(rho_0), float(rs))


def nfw_forces(pos, m, halo, force=None):
    """nfw_gravity_system (nfw.rs:103-139): returns force + the halo's force,
    halo = (rho_0, Rs, cx, cy, cz)."""
    pos, m = _f64(pos), _f64(m)
    n = m.shape[0]
    P = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    F = [np.zeros(n) if force is None else np.ascontiguousarray(force[:, k], dtype=np.float64).copy()
         for k in range(3)]
    H = _f64(halo)
    lib().oracle_nfw_forces(n, *[_p(a) for a in P], _p(m), _p(H), *[_p(a) for a in F])
    return np.stack(F, axis=1)


def normalize(sectors, local, sector_size):
    """sector_boundary_system (origin.rs:16-24): returns (sectors, local,
    changed) after normalize_position on every body."""
    S = [np.ascontiguousarray(sectors[:, k], dtype=np.int64).copy() for k in range(3)]
    L = [np.ascontiguousarray(local[:, k], dtype=np.float64).copy() for k in range(3)]
    n = S[0].shape[0]
    ch = lib().oracle_normalize(n, *[_p(a, _I64) for a in S], *[_p(a) for a in L],
                                float(sector_size))
    return np.stack(S, axis=1), np.stack(L, axis=1), bool(ch)


def vv_run_sectors(sectors, local, vel, m, sector_size, G, eps, dt, nsteps, method="direct",
                   theta=0.5, halo=None, nthreads=None):
    """The reference tick loop on (Sector, LocalPosition): flatten per force
    pass, integrate LocalPosition, sector_boundary_system after the velocity
    step.  Returns (sectors, local, vel, acc, prev_acc)."""
    m = _f64(m)
    n = m.shape[0]
    S = [np.ascontiguousarray(sectors[:, k], dtype=np.int64).copy() for k in range(3)]
    L = [np.ascontiguousarray(local[:, k], dtype=np.float64).copy() for k in range(3)]
    V = [np.ascontiguousarray(vel[:, k], dtype=np.float64).copy() for k in range(3)]
    A = [np.zeros(n) for _ in range(3)]
    PA = [np.zeros(n) for _ in range(3)]
    H = None if halo is None else _f64(halo)
    lib().oracle_vv_run_sectors(n, *[_p(a, _I64) for a in S], *[_p(a) for a in L],
                                *[_p(a) for a in V], _p(m), float(sector_size), G, eps, theta,
                                0 if method == "direct" else 1, dt, nsteps, nthreads or ncpu(),
                                *[_p(a) for a in A], *[_p(a) for a in PA],
                                None if H is None else _p(H))
    st = lambda X: np.stack(X, axis=1)
    return st(S), st(L), st(V), st(A), st(PA)
