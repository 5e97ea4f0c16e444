"""physgpu: Python binding of libphysgpu.so (the B200 gravity library).

Two layers:

* `Context` wraps the C ABI of include/physgpu.h one call per method.
* A mirror of the reference's gravity "plugin API" (bevy_ecs systems over
  components, src/physics/*.rs): `UniverseConfig`, `SimulationTime`, a
  structure-of-arrays `World`, and the systems
  `brute_force_gravity_system`, `barnes_hut_gravity_system`,
  `compute_acceleration_system`, `velocity_verlet_position_system`,
  `velocity_verlet_velocity_system`, `reset_forces`, plus the energy systems.
  Tests written against these read like the reference's own unit tests.

There is no CPU fallback: importing works without a GPU, but any compute call
raises `PhysError` when the CUDA library or a device is missing.
"""
import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libphysgpu.so")

OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_NONFINITE, ERR_TIMEOUT, ERR_STATE = range(7)
DIRECT, BARNES_HUT = 0, 1
F64_EXACT, F64, F32C = 0, 1, 2
GROUP_WALK = 1  # phys_params.flags: Barnes-Hut walk per group of 64 bodies
COMP_POSITION, COMP_VELOCITY, COMP_ACCELERATION, COMP_PREV_ACCELERATION, COMP_MASS = range(5)
# Ensemble launch configurations: lanes per system (8, 16, 32 or ENS_BY_SIZE)
# | ens_warps(warps per block); the autotuner's candidates, in its order.
ENS_BY_SIZE = 1


def ens_warps(w):
    return w << 8


ENS_CANDIDATES = (8 | 2 << 8, 16 | 2 << 8, 32 | 2 << 8, ENS_BY_SIZE | 2 << 8, 32 | 4 << 8,
                  ENS_BY_SIZE | 4 << 8)

PRECISIONS = {"f64_exact": F64_EXACT, "f64": F64, "f32c": F32C}

# Every symbol include/physgpu.h declares.
EXPORTED = [
    "phys_status_string", "phys_last_error", "phys_ctx_create", "phys_ctx_destroy",
    "phys_ctx_stream", "phys_last_timings", "phys_state_upload", "phys_state_upload_sectors",
    "phys_state_set_accel", "phys_state_download", "phys_state_size", "phys_component_write",
    "phys_component_read", "phys_gravity_forces", "phys_gravity_accel", "phys_verlet_steps",
    "phys_vv_position_step", "phys_vv_velocity_step", "phys_verlet_steps_async",
    "phys_diagnostics", "phys_bh_export", "phys_probe_peaks", "phys_direct_accel_targets",
    "phys_ensemble_load", "phys_ensemble_run", "phys_ensemble_download", "phys_ensemble_autotune",
    "phys_direct_accel_noalloc", "phys_adjoint_direct", "phys_trajectory_loss",
    "phys_nfw_density", "phys_nfw_enclosed_mass", "phys_nfw_circular_velocity",
    "phys_nfw_forces", "phys_set_nfw_halo", "phys_state_upload_sector_state",
    "phys_state_download_sector_state", "phys_debug_set_wait_limit", "phys_share_chunk",
    "phys_gravity_accel_share", "phys_gravity_accel_unshare", "phys_verlet_tick_host",
    "phys_debug_divide",
]


class PhysError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


class Params(ctypes.Structure):
    _fields_ = [("G", ctypes.c_double), ("eps", ctypes.c_double), ("theta", ctypes.c_double),
                ("method", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("leaf_cap", ctypes.c_int32), ("flags", ctypes.c_int32)]


class NfwHalo(ctypes.Structure):
    _fields_ = [("rho_0", ctypes.c_double), ("scale_radius", ctypes.c_double),
                ("center", ctypes.c_double * 3), ("enabled", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Timings(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("bbox_ms", ctypes.c_double),
                ("keys_ms", ctypes.c_double), ("sort_ms", ctypes.c_double),
                ("tree_ms", ctypes.c_double), ("walk_ms", ctypes.c_double),
                ("verlet_ms", ctypes.c_double), ("interactions", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("nodes", ctypes.c_int64),
                ("max_depth", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("walk_eval_ms", ctypes.c_double), ("walk_eval_interactions", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)
_U64 = ctypes.POINTER(ctypes.c_uint64)
_VP = ctypes.c_void_p


def load_library(path=None):
    """Load libphysgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("PHYSGPU_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise PhysError(ERR_STATE, "libphysgpu.so not built (%s); run __graft_entry__.build()" % path)
    L = ctypes.CDLL(path)
    i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P = ctypes.POINTER(Params)
    sig = {
        "phys_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "phys_last_error": ([_VP], ctypes.c_char_p),
        "phys_ctx_create": ([ctypes.c_int, ctypes.POINTER(_VP)], ctypes.c_int),
        "phys_ctx_destroy": ([_VP], ctypes.c_int),
        "phys_ctx_stream": ([_VP], _VP),
        "phys_last_timings": ([_VP, ctypes.POINTER(Timings)], ctypes.c_int),
        "phys_state_upload": ([_VP, i64] + [_D] * 7, ctypes.c_int),
        "phys_state_upload_sectors": ([_VP, i64, _I64, _I64, _I64, _D, _D, _D, dbl, i32]
                                      + [_D] * 4, ctypes.c_int),
        "phys_state_set_accel": ([_VP, _D, _D, _D], ctypes.c_int),
        "phys_state_download": ([_VP] + [_D] * 9, ctypes.c_int),
        "phys_state_size": ([_VP], i64),
        "phys_component_write": ([_VP, i32, _D, _D, _D], ctypes.c_int),
        "phys_component_read": ([_VP, i32, _D, _D, _D], ctypes.c_int),
        "phys_gravity_forces": ([_VP, P, _D, _D, _D], ctypes.c_int),
        "phys_gravity_accel": ([_VP, P, _D, _D, _D], ctypes.c_int),
        "phys_verlet_steps": ([_VP, P, dbl, i64], ctypes.c_int),
        "phys_verlet_steps_async": ([_VP, P, dbl, i64], ctypes.c_int),
        "phys_vv_position_step": ([_VP, dbl], ctypes.c_int),
        "phys_vv_velocity_step": ([_VP, dbl], ctypes.c_int),
        "phys_diagnostics": ([_VP, dbl, _D], ctypes.c_int),
        "phys_bh_export": ([_VP, P, i64, _I64, _I32, _I64, _D, _D, _I64, _I64, _U64, _U64, _I64,
                            _D], ctypes.c_int),
        "phys_probe_peaks": ([_VP, _D, _D, _D], ctypes.c_int),
        "phys_direct_accel_targets": ([_VP, P, i64, _I64, _D, _D, _D], ctypes.c_int),
        "phys_ensemble_load": ([_VP, i64, _I64] + [_D] * 7, ctypes.c_int),
        "phys_ensemble_run": ([_VP, P, dbl, i64, i32, i64], ctypes.c_int),
        "phys_ensemble_download": ([_VP] + [_D] * 9, ctypes.c_int),
        "phys_ensemble_autotune": ([_VP, P, dbl, i64, _I32, _D], ctypes.c_int),
        "phys_adjoint_direct": ([_VP, P, dbl, i64, i64] + [_D] * 11, ctypes.c_int),
        "phys_trajectory_loss": ([_VP, P, dbl, i64] + [_D] * 7, ctypes.c_int),
        "phys_direct_accel_noalloc": ([i64, _VP, _VP, _VP, _VP, dbl, dbl, i32, _VP, _VP, _VP, _VP,
                                       ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "phys_nfw_density": ([dbl, dbl, dbl], dbl),
        "phys_nfw_enclosed_mass": ([dbl, dbl, dbl], dbl),
        "phys_nfw_circular_velocity": ([dbl, dbl, dbl], dbl),
        "phys_nfw_forces": ([_VP, ctypes.POINTER(NfwHalo), _D, _D, _D], ctypes.c_int),
        "phys_set_nfw_halo": ([_VP, ctypes.POINTER(NfwHalo)], ctypes.c_int),
        "phys_state_upload_sector_state": ([_VP, i64, _I64, _I64, _I64, _D, _D, _D, dbl]
                                           + [_D] * 4, ctypes.c_int),
        "phys_state_download_sector_state": ([_VP, _I64, _I64, _I64, _D, _D, _D],
                                             ctypes.c_int),
        "phys_debug_set_wait_limit": ([_VP, i64], ctypes.c_int),
        "phys_debug_divide": ([_VP, i64, _D, _D, _D], ctypes.c_int),
        "phys_share_chunk": ([i64, i32], i64),
        "phys_gravity_accel_share": ([_VP, P, i32, i32, _VP], ctypes.c_int),
        "phys_gravity_accel_unshare": ([_VP, i32, _VP], ctypes.c_int),
        "phys_verlet_tick_host": ([_VP, P, dbl, i64] + [_D] * 10, ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _p(a, ty=_D):
    return None if a is None else a.ctypes.data_as(ty)


def _col(a, k):
    return np.ascontiguousarray(a[:, k], dtype=np.float64)


def make_params(G, eps, theta=0.5, method=DIRECT, precision=F64_EXACT, leaf_cap=1, flags=0):
    if isinstance(precision, str):
        precision = PRECISIONS[precision]
    return Params(float(G), float(eps), float(theta), int(method), int(precision), int(leaf_cap),
                  int(flags))


def share_chunk(n, world):
    """Targets per share when n bodies are split into `world` shares
    (phys_share_chunk): a multiple of 128."""
    return int(load_library().phys_share_chunk(int(n), int(world)))


class Context:
    """One device context: a CUDA stream plus device-resident body state."""

    def __init__(self, device=0):
        self.lib = load_library()
        h = _VP()
        st = self.lib.phys_ctx_create(int(device), ctypes.byref(h))
        if st != OK:
            raise PhysError(st, "phys_ctx_create(%d) failed: %s" % (
                device, self.lib.phys_status_string(st).decode()))
        self.h = h
        self.n = 0
        self.device = int(device)

    def close(self):
        if getattr(self, "h", None):
            self.lib.phys_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what):
        if st != OK:
            raise PhysError(st, "%s: %s" % (what, self.lib.phys_last_error(self.h).decode()))

    @property
    def stream(self):
        return self.lib.phys_ctx_stream(self.h)

    def set_wait_limit(self, spins):
        """Bound on each bounded device wait of the radix sorts (tests only);
        a negative value restores the default."""
        self._check(self.lib.phys_debug_set_wait_limit(self.h, int(spins)),
                    "phys_debug_set_wait_limit")

    def debug_divide(self, a, b):
        """a / b through the tree's centre-of-mass division (tests only)."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        if a.shape != b.shape or a.ndim != 1:
            raise ValueError("a and b must be 1-D arrays of one length")
        q = np.empty_like(a)
        self._check(self.lib.phys_debug_divide(self.h, a.shape[0], _p(a), _p(b), _p(q)),
                    "phys_debug_divide")
        return q

    # ---- state ----
    def upload(self, pos, vel, m):
        pos = np.asarray(pos, dtype=np.float64)
        m = np.ascontiguousarray(m, dtype=np.float64)
        n = m.shape[0]
        P = [_col(pos, k) for k in range(3)]
        V = [None] * 3 if vel is None else [_col(np.asarray(vel, np.float64), k) for k in range(3)]
        self._check(self.lib.phys_state_upload(self.h, n, *[_p(a) for a in P],
                                               *[_p(a) for a in V], _p(m)), "phys_state_upload")
        self.n = n

    def upload_sectors(self, sectors, local, sector_size, m, vel=None, bh_quirk=False):
        s = np.ascontiguousarray(sectors, dtype=np.int64)
        local = np.asarray(local, dtype=np.float64)
        m = np.ascontiguousarray(m, dtype=np.float64)
        n = m.shape[0]
        S = [np.ascontiguousarray(s[:, k]) for k in range(3)]
        Lc = [_col(local, k) for k in range(3)]
        V = [None] * 3 if vel is None else [_col(np.asarray(vel, np.float64), k) for k in range(3)]
        self._check(self.lib.phys_state_upload_sectors(
            self.h, n, *[_p(a, _I64) for a in S], *[_p(a) for a in Lc], float(sector_size),
            int(bool(bh_quirk)), *[_p(a) for a in V], _p(m)), "phys_state_upload_sectors")
        self.n = n

    def set_accel(self, acc):
        A = [_col(np.asarray(acc, np.float64), k) for k in range(3)]
        self._check(self.lib.phys_state_set_accel(self.h, *[_p(a) for a in A]),
                    "phys_state_set_accel")

    def upload_sector_state(self, sectors, local, sector_size, m, vel=None):
        """Keep (Sector, LocalPosition) on the device: later force passes
        flatten them and Verlet runs normalise sectors every tick."""
        m = np.ascontiguousarray(m, dtype=np.float64)
        n = m.shape[0]
        S = [np.ascontiguousarray(np.asarray(sectors)[:, k], dtype=np.int64) for k in range(3)]
        L = [_col(np.asarray(local, np.float64), k) for k in range(3)]
        V = [None] * 3 if vel is None else [_col(np.asarray(vel, np.float64), k) for k in range(3)]
        self._check(self.lib.phys_state_upload_sector_state(
            self.h, n, *[_p(a, _I64) for a in S], *[_p(a) for a in L], float(sector_size),
            *[_p(a) for a in V], _p(m)), "phys_state_upload_sector_state")
        self.n = n

    def download_sector_state(self):
        """(sectors int64 (n,3), local positions (n,3))."""
        n = self.n
        S = [np.empty(n, dtype=np.int64) for _ in range(3)]
        L = [np.empty(n) for _ in range(3)]
        self._check(self.lib.phys_state_download_sector_state(
            self.h, *[_p(a, _I64) for a in S], *[_p(a) for a in L]),
            "phys_state_download_sector_state")
        return np.stack(S, axis=1), np.stack(L, axis=1)

    def download(self):
        n = self.n
        out = [np.empty(n) for _ in range(9)]
        self._check(self.lib.phys_state_download(self.h, *[_p(a) for a in out]),
                    "phys_state_download")
        st = lambda a, b, c: np.stack([a, b, c], axis=1)
        return st(*out[0:3]), st(*out[3:6]), st(*out[6:9])

    def write_component(self, comp, arr):
        arr = np.asarray(arr, dtype=np.float64)
        if comp == COMP_MASS:
            a = np.ascontiguousarray(arr)
            self._check(self.lib.phys_component_write(self.h, comp, _p(a), None, None),
                        "phys_component_write")
        else:
            A = [_col(arr, k) for k in range(3)]
            self._check(self.lib.phys_component_write(self.h, comp, *[_p(a) for a in A]),
                        "phys_component_write")

    def read_component(self, comp):
        if comp == COMP_MASS:
            a = np.empty(self.n)
            self._check(self.lib.phys_component_read(self.h, comp, _p(a), None, None),
                        "phys_component_read")
            return a
        out = [np.empty(self.n) for _ in range(3)]
        self._check(self.lib.phys_component_read(self.h, comp, *[_p(a) for a in out]),
                    "phys_component_read")
        return np.stack(out, axis=1)

    # ---- gravity ----
    def gravity_forces(self, params, force=None):
        """Force += gravity (returns the updated (n,3) array)."""
        n = self.n
        f = np.zeros((n, 3)) if force is None else np.asarray(force, np.float64)
        F = [np.ascontiguousarray(f[:, k]) for k in range(3)]
        self._check(self.lib.phys_gravity_forces(self.h, ctypes.byref(params),
                                                 *[_p(a) for a in F]), "phys_gravity_forces")
        return np.stack(F, axis=1)

    def nfw_forces(self, halo, force=None):
        """nfw_gravity_system on the device: Force += the halo's force (returns
        the updated (n,3) array).  `halo` is an NfwHaloConfig or NfwHalo."""
        n = self.n
        f = np.zeros((n, 3)) if force is None else np.asarray(force, np.float64)
        F = [np.ascontiguousarray(f[:, k]) for k in range(3)]
        h = _halo(halo)
        self._check(self.lib.phys_nfw_forces(self.h, ctypes.byref(h), *[_p(a) for a in F]),
                    "phys_nfw_forces")
        return np.stack(F, axis=1)

    def set_nfw_halo(self, halo):
        """Later accelerations (gravity_accel, verlet_steps) include the halo:
        a = (F_gravity + F_nfw) / m.  None removes it."""
        h = None if halo is None else _halo(halo)
        self._check(self.lib.phys_set_nfw_halo(self.h, None if h is None else ctypes.byref(h)),
                    "phys_set_nfw_halo")

    def gravity_accel(self, params, download=True):
        n = self.n
        A = [np.empty(n) for _ in range(3)] if download else [None] * 3
        self._check(self.lib.phys_gravity_accel(self.h, ctypes.byref(params),
                                                *[_p(a) for a in A]), "phys_gravity_accel")
        return np.stack(A, axis=1) if download else None

    # ---- target shares (one system over several GPUs) ----
    def gravity_accel_share(self, params, rank, world, out_ptr):
        """Evaluates share `rank` of `world` of the targets and packs its
        accelerations into the device buffer at address out_ptr (3 *
        share_chunk(n, world) float64 on this context's device)."""
        self._check(self.lib.phys_gravity_accel_share(self.h, ctypes.byref(params), int(rank),
                                                      int(world), _VP(int(out_ptr))),
                    "phys_gravity_accel_share")

    def gravity_accel_unshare(self, world, gathered_ptr):
        """Scatters all shares' blocks (device buffer at gathered_ptr, world *
        3 * share_chunk(n, world) float64) into the acceleration arrays."""
        self._check(self.lib.phys_gravity_accel_unshare(self.h, int(world),
                                                        _VP(int(gathered_ptr))),
                    "phys_gravity_accel_unshare")

    def direct_accel_targets(self, params, targets):
        """f64 direct-sum accelerations for the given targets (all sources)."""
        t = np.ascontiguousarray(targets, dtype=np.int64)
        out = [np.empty(t.shape[0]) for _ in range(3)]
        self._check(self.lib.phys_direct_accel_targets(self.h, ctypes.byref(params), t.shape[0],
                                                       _p(t, _I64), *[_p(a) for a in out]),
                    "phys_direct_accel_targets")
        return np.stack(out, axis=1)

    # ---- batched ensemble ----
    def ensemble_load(self, offsets, pos, vel, m):
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        pos = np.asarray(pos, np.float64)
        m = np.ascontiguousarray(m, dtype=np.float64)
        P = [_col(pos, k) for k in range(3)]
        V = [None] * 3 if vel is None else [_col(np.asarray(vel, np.float64), k) for k in range(3)]
        self._check(self.lib.phys_ensemble_load(self.h, off.shape[0] - 1, _p(off, _I64),
                                                *[_p(a) for a in P], *[_p(a) for a in V], _p(m)),
                    "phys_ensemble_load")
        self.ens_n = m.shape[0]

    def ensemble_run(self, params, dt, nsteps, group=0, chunk=0):
        self._check(self.lib.phys_ensemble_run(self.h, ctypes.byref(params), float(dt),
                                               int(nsteps), int(group), int(chunk)),
                    "phys_ensemble_run")

    def ensemble_download(self):
        out = [np.empty(self.ens_n) for _ in range(9)]
        self._check(self.lib.phys_ensemble_download(self.h, *[_p(a) for a in out]),
                    "phys_ensemble_download")
        st = lambda a, b, c: np.stack([a, b, c], axis=1)
        return st(*out[0:3]), st(*out[3:6]), st(*out[6:9])

    def ensemble_autotune(self, params, dt, probe_steps=8):
        """(best configuration code, {code: ms}) over ENS_CANDIDATES."""
        best = ctypes.c_int32()
        ms = np.zeros(len(ENS_CANDIDATES))
        self._check(self.lib.phys_ensemble_autotune(self.h, ctypes.byref(params), float(dt),
                                                    int(probe_steps), ctypes.byref(best), _p(ms)),
                    "phys_ensemble_autotune")
        return best.value, dict(zip(ENS_CANDIDATES, ms.tolist()))

    # ---- trajectory gradients ----
    def adjoint(self, params, dt, nsteps, targets, checkpoint=32):
        """(loss, dL/dx0 (n,3), dL/dv0 (n,3), dL/dm (n,)) by the hand-written adjoint."""
        t = np.asarray(targets, np.float64)
        T = [_col(t, k) for k in range(3)]
        n = self.n
        gx = [np.empty(n) for _ in range(3)]
        gv = [np.empty(n) for _ in range(3)]
        gm = np.empty(n)
        loss = ctypes.c_double()
        self._check(self.lib.phys_adjoint_direct(
            self.h, ctypes.byref(params), float(dt), int(nsteps), int(checkpoint),
            *[_p(a) for a in T], ctypes.byref(loss), *[_p(a) for a in gx], *[_p(a) for a in gv],
            _p(gm)), "phys_adjoint_direct")
        return loss.value, np.stack(gx, 1), np.stack(gv, 1), gm

    def trajectory_loss(self, params, dt, nsteps, targets, final=False):
        t = np.asarray(targets, np.float64)
        T = [_col(t, k) for k in range(3)]
        loss = ctypes.c_double()
        X = [np.empty(self.n) for _ in range(3)] if final else [None] * 3
        self._check(self.lib.phys_trajectory_loss(self.h, ctypes.byref(params), float(dt),
                                                  int(nsteps), *[_p(a) for a in T],
                                                  ctypes.byref(loss), *[_p(a) for a in X]),
                    "phys_trajectory_loss")
        return (loss.value, np.stack(X, 1)) if final else loss.value

    def verlet_steps(self, params, dt, nsteps):
        self._check(self.lib.phys_verlet_steps(self.h, ctypes.byref(params), float(dt),
                                               int(nsteps)), "phys_verlet_steps")

    def verlet_steps_async(self, params, dt, nsteps):
        self._check(self.lib.phys_verlet_steps_async(self.h, ctypes.byref(params), float(dt),
                                                     int(nsteps)), "phys_verlet_steps_async")

    def verlet_tick_host(self, params, dt, x, v, m, a):
        """One tick on host state in one call (phys_verlet_tick_host): x, v, a
        are lists of three contiguous float64 arrays (numpy, or page-locked
        torch tensors) updated in place; m is read."""
        def ptr(t):
            if hasattr(t, "data_ptr"):
                return ctypes.cast(t.data_ptr(), _D)
            return _p(t)
        n = len(m)
        self._check(self.lib.phys_verlet_tick_host(
            self.h, ctypes.byref(params), float(dt), n, *[ptr(t) for t in x],
            *[ptr(t) for t in v], ptr(m), *[ptr(t) for t in a]), "phys_verlet_tick_host")
        self.n = n

    def vv_position_step(self, dt):
        self._check(self.lib.phys_vv_position_step(self.h, float(dt)), "phys_vv_position_step")

    def vv_velocity_step(self, dt):
        self._check(self.lib.phys_vv_velocity_step(self.h, float(dt)), "phys_vv_velocity_step")

    def diagnostics(self, G):
        out = np.zeros(5)
        self._check(self.lib.phys_diagnostics(self.h, float(G), _p(out)), "phys_diagnostics")
        return out

    def timings(self):
        t = Timings()
        self._check(self.lib.phys_last_timings(self.h, ctypes.byref(t)), "phys_last_timings")
        return t.as_dict()

    def probe_peaks(self):
        """Measured (fp32 FFMA, fp32 packed FFMA2, fp64 DFMA) TFLOP/s."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.phys_probe_peaks(self.h, ctypes.byref(a), ctypes.byref(b),
                                              ctypes.byref(c)), "phys_probe_peaks")
        return a.value, b.value, c.value

    def bh_export(self, params):
        n = self.n
        cap = 4 * n + 64
        nn = ctypes.c_int64()
        depth = np.zeros(cap, np.int32)
        count = np.zeros(cap, np.int64)
        mass = np.zeros(cap)
        com = np.zeros(3 * cap)
        leaf_body = np.zeros(cap, np.int64)
        body_leaf = np.zeros(n, np.int64)
        khi = np.zeros(n, np.uint64)
        klo = np.zeros(n, np.uint64)
        perm = np.zeros(n, np.int64)
        root4 = np.zeros(4)
        self._check(self.lib.phys_bh_export(
            self.h, ctypes.byref(params), cap, ctypes.byref(nn), _p(depth, _I32), _p(count, _I64),
            _p(mass), _p(com), _p(leaf_body, _I64), _p(body_leaf, _I64), _p(khi, _U64),
            _p(klo, _U64), _p(perm, _I64), _p(root4)), "phys_bh_export")
        k = nn.value
        assert k <= cap
        return dict(depth=depth[:k], count=count[:k], mass=mass[:k],
                    com=com[:3 * k].reshape(k, 3), leaf_body=leaf_body[:k], body_leaf=body_leaf,
                    keys_hi=khi, keys_lo=klo, perm=perm, root=root4, nnodes=k)


# ---------------------------------------------------------------------------
# Mirror of the reference's gravity plugin API (bevy_ecs systems).
# ---------------------------------------------------------------------------
G_SI = 6.67430e-11  # src/core/constants.rs:7


@dataclass
class UniverseConfig:
    """src/core/config.rs:26-79 (fields on the gravity path, same defaults)."""
    gravitational_constant: float = G_SI
    softening_epsilon: float = 1e-4
    barnes_hut_theta: float = 0.5
    sector_size: float = 1e12


@dataclass
class NfwHaloConfig:
    """src/physics/nfw.rs:24-47 (same defaults: a Milky-Way-like halo, off)."""
    rho_0: float = 1.4e-21
    scale_radius: float = 6.17e20
    center: tuple = (0.0, 0.0, 0.0)
    enabled: bool = False


def _halo(cfg):
    if isinstance(cfg, NfwHalo):
        return cfg
    h = NfwHalo()
    h.rho_0 = float(cfg.rho_0)
    h.scale_radius = float(cfg.scale_radius)
    for k in range(3):
        h.center[k] = float(cfg.center[k])
    h.enabled = 1 if cfg.enabled else 0
    h.reserved = 0
    return h


def nfw_density(r, rho_0, rs):
    """nfw.rs:61-67: rho_0 / ((r/Rs)(1 + r/Rs)^2); 0 for r <= 0 or Rs <= 0."""
    return load_library().phys_nfw_density(float(r), float(rho_0), float(rs))


def nfw_enclosed_mass(r, rho_0, rs):
    """nfw.rs:76-83: 4 pi rho_0 Rs^3 (ln(1 + x) - x / (1 + x)), x = r/Rs."""
    return load_library().phys_nfw_enclosed_mass(float(r), float(rho_0), float(rs))


def nfw_circular_velocity(r, rho_0, rs):
    """nfw.rs:88-91: sqrt(G M(r) / r), G the SI constant."""
    return load_library().phys_nfw_circular_velocity(float(r), float(rho_0), float(rs))


@dataclass
class SimulationTime:
    """src/core/time.rs:16-77 (the fixed dt the integrators read)."""
    dt: float = 1.0 / 60.0
    tick: int = 0
    elapsed: float = 0.0

    @staticmethod
    def with_dt(dt):
        return SimulationTime(dt=dt)

    def advance_tick(self):
        self.tick += 1
        self.elapsed += self.dt


@dataclass
class World:
    """Structure-of-arrays body store holding the components the gravity path
    reads and writes (Force, Mass, Sector, LocalPosition, Velocity,
    Acceleration, PreviousAcceleration; src/components/dynamics.rs:13-37,
    src/core/coordinates.rs:19-26).  Row order is the query order."""
    mass: np.ndarray = field(default_factory=lambda: np.zeros(0))
    local: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    sector: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int64))
    velocity: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    force: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    acceleration: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    prev_acceleration: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))

    def spawn(self, mass, local, sector=(0, 0, 0), velocity=(0.0, 0.0, 0.0),
              acceleration=(0.0, 0.0, 0.0), prev_acceleration=(0.0, 0.0, 0.0)):
        """Add one body; returns its row (the 'entity')."""
        self.mass = np.append(self.mass, float(mass))
        self.local = np.vstack([self.local, np.asarray(local, np.float64)[None]])
        self.sector = np.vstack([self.sector, np.asarray(sector, np.int64)[None]])
        self.velocity = np.vstack([self.velocity, np.asarray(velocity, np.float64)[None]])
        self.force = np.vstack([self.force, np.zeros((1, 3))])
        self.acceleration = np.vstack([self.acceleration, np.asarray(acceleration, np.float64)[None]])
        self.prev_acceleration = np.vstack(
            [self.prev_acceleration, np.asarray(prev_acceleration, np.float64)[None]])
        return self.mass.shape[0] - 1

    @staticmethod
    def from_arrays(pos, vel, m):
        n = len(m)
        return World(mass=np.asarray(m, np.float64).copy(), local=np.asarray(pos, np.float64).copy(),
                     sector=np.zeros((n, 3), np.int64),
                     velocity=np.zeros((n, 3)) if vel is None else np.asarray(vel, np.float64).copy(),
                     force=np.zeros((n, 3)), acceleration=np.zeros((n, 3)),
                     prev_acceleration=np.zeros((n, 3)))

    def __len__(self):
        return int(self.mass.shape[0])


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _gravity_system(world, config, method, precision, leaf_cap, ctx, bh_quirk, flags=0):
    ctx = ctx or default_context()
    if len(world) < 2:  # gravity.rs:49-51
        return
    ctx.upload_sectors(world.sector, world.local, config.sector_size, world.mass,
                       bh_quirk=bh_quirk)
    p = make_params(config.gravitational_constant, config.softening_epsilon,
                    config.barnes_hut_theta, method, precision, leaf_cap, flags)
    world.force = ctx.gravity_forces(p, world.force)


def brute_force_gravity_system(world, config, precision=F64_EXACT, ctx=None):
    """src/physics/gravity.rs:27-74 on the GPU: Force += softened direct sum."""
    _gravity_system(world, config, DIRECT, precision, 1, ctx, bh_quirk=False)


def barnes_hut_gravity_system(world, config, precision=F64_EXACT, leaf_cap=1, ctx=None,
                              group_walk=False):
    """src/physics/gravity_tree.rs:260-338 on the GPU: Force += Barnes-Hut.
    group_walk=True walks the tree once per cell group of at most 64 bodies
    (F64 / F32C only; stricter opening, not the reference's traversal)."""
    _gravity_system(world, config, BARNES_HUT, precision, leaf_cap, ctx, bh_quirk=True,
                    flags=GROUP_WALK if group_walk else 0)


def nfw_gravity_system(world, halo_config, ctx=None):
    """src/physics/nfw.rs:103-139 on the GPU: Force += -G M(r) m / r^2 r_hat
    about the halo centre, from LocalPosition (the reference ignores Sector
    here); nothing when the halo is disabled."""
    if not halo_config.enabled or len(world) == 0:
        return
    ctx = ctx or default_context()
    ctx.upload(world.local, None, world.mass)
    world.force = ctx.nfw_forces(halo_config, world.force)


def reset_forces(world):
    """src/physics/forces.rs:15-19."""
    world.force[:] = 0.0


def _state_to_ctx(world, ctx):
    # The integrators update LocalPosition itself (integrators.rs:80): local
    # coordinates go to the device unflattened.
    ctx.upload(world.local, world.velocity, world.mass)
    ctx.write_component(COMP_ACCELERATION, world.acceleration)
    ctx.write_component(COMP_PREV_ACCELERATION, world.prev_acceleration)


def compute_acceleration_system(world, ctx=None):
    """src/physics/integrators.rs:110-118: a = F / m (IEEE division)."""
    world.acceleration = world.force / world.mass[:, None]


def run_velocity_verlet(world, config, time, ticks, method=DIRECT, precision=F64_EXACT,
                        leaf_cap=1, flags=0, ctx=None, halo=None):
    """`ticks` ticks of the reference's Velocity-Verlet schedule
    (src/main.rs:103-150: gravity [+ nfw_gravity_system], a = F/m, position
    and velocity steps, sector_boundary_system) on the device, the World's
    Sector and LocalPosition kept there between ticks.  One upload, one
    download; advances `time`.  The first tick recomputes a(x) as the
    schedule's first force pass does (the Acceleration and
    PreviousAcceleration components are overwritten before they are read)."""
    ctx = ctx or default_context()
    ctx.upload_sector_state(world.sector, world.local, config.sector_size, world.mass,
                            world.velocity)
    p = make_params(config.gravitational_constant, config.softening_epsilon,
                    config.barnes_hut_theta, method, precision, leaf_cap, flags)
    if halo is not None:
        ctx.set_nfw_halo(halo)
    try:
        ctx.verlet_steps(p, time.dt, ticks)
    finally:
        if halo is not None:
            ctx.set_nfw_halo(None)
    world.sector, world.local = ctx.download_sector_state()
    _, world.velocity, world.acceleration = ctx.download()
    world.prev_acceleration = ctx.read_component(COMP_PREV_ACCELERATION)
    for _ in range(ticks):
        time.advance_tick()


def velocity_verlet_position_system(world, time, ctx=None):
    """src/physics/integrators.rs:63-83 on the device."""
    ctx = ctx or default_context()
    _state_to_ctx(world, ctx)
    ctx.vv_position_step(time.dt)
    world.local = ctx.read_component(COMP_POSITION)
    world.prev_acceleration = ctx.read_component(COMP_PREV_ACCELERATION)


def velocity_verlet_velocity_system(world, time, ctx=None):
    """src/physics/integrators.rs:92-104 on the device."""
    ctx = ctx or default_context()
    _state_to_ctx(world, ctx)
    ctx.vv_velocity_step(time.dt)
    world.velocity = ctx.read_component(COMP_VELOCITY)


def energy_diagnostics(world, config, ctx=None):
    """src/physics/energy.rs:21-56 + integrators.rs:123-129 on the device:
    returns (kinetic, potential, momentum (3,))."""
    ctx = ctx or default_context()
    ctx.upload_sectors(world.sector, world.local, config.sector_size, world.mass,
                       vel=world.velocity)
    out = ctx.diagnostics(config.gravitational_constant)
    return out[0], out[1], out[2:5]
