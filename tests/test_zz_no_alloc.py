"""phys_direct_accel_noalloc through the C ABI (collected last on purpose).

Some callers cannot allocate device memory once they are running: an
engine's fixed-step loop that set up all its buffers at start-up and forbids
cudaMalloc / cudaFree afterwards (they can synchronise the device and stall
a tick), or a host application that lends the library only memory from its
own pool.  They pass their own device buffers and the entry point keeps its
scratch in a fixed device array.  These tests compare it with the oracle's
direct sum (the reference's arithmetic) and with the regular entry point
(phys_gravity_accel, direct sum) on two calls in a row, with the tolerances
the other direct-sum tests use, check that the calls after the first one
leave the device's free memory unchanged, and check that a problem larger
than the fixed scratch is refused with a message.
"""
import ctypes

import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import DIRECT, F32C, F64, make_params

pytestmark = pytest.mark.gpu


def _dev(torch, pos, m):
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    n = len(m)
    X = [dev(pos[:, k]) for k in range(3)]
    A = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
    return X, dev(m), A


def _call(lib, n, X, M, A, G, eps, precision, stream):
    err = ctypes.create_string_buffer(512)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    st = lib.phys_direct_accel_noalloc(n, *[vp(t) for t in X], vp(M), G, eps, precision,
                                       *[vp(t) for t in A], ctypes.c_void_p(stream), err, 512)
    return st, err.value.decode()


def rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


@pytest.mark.parametrize("precision", [F64, F32C])
def test_noalloc_matches_oracle_and_regular_entry_point_twice(precision):
    torch = pytest.importorskip("torch")
    lib = physgpu.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    with physgpu.Context(0) as ctx:
        # two calls in a row, different sizes: the shared scratch keeps the
        # first call's contents when the second one starts
        for n, seed in ((4096, 11), (1000, 12)):
            pos, _, m = ics.plummer(n, seed=seed)
            X, M, A = _dev(torch, pos, m)
            torch.cuda.synchronize()
            st, err = _call(lib, n, X, M, A, 1.0, 0.01, precision, stream)
            assert st == physgpu.OK, err
            a = torch.stack(A, 1).cpu().numpy()
            ref = oracle.accel(oracle.direct_forces(pos, m, 1.0, 0.01), m)
            ctx.upload(pos, None, m)
            reg = ctx.gravity_accel(make_params(1.0, 0.01, method=DIRECT, precision=precision))
            for e in (rel(a, ref), rel(a, reg)):
                if precision == F64:
                    assert e.max() < 1e-12, e.max()
                else:
                    assert np.median(e) <= 1e-6 and e.max() <= 1e-4, (np.median(e), e.max())


def test_noalloc_allocates_nothing():
    """After the first call on the device (which looks up the scratch array's
    address), calls leave the device's free memory exactly as it was."""
    torch = pytest.importorskip("torch")
    lib = physgpu.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    pos, _, m = ics.plummer(32768, seed=5)  # the largest size the scratch holds
    X, M, A = _dev(torch, pos, m)
    torch.cuda.synchronize()
    st, err = _call(lib, len(m), X, M, A, 1.0, 0.01, F32C, stream)
    assert st == physgpu.OK, err
    first = torch.stack(A, 1).cpu().numpy()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for precision in (F64, F32C, F32C):
        st, err = _call(lib, len(m), X, M, A, 1.0, 0.01, precision, stream)
        assert st == physgpu.OK, err
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.array_equal(torch.stack(A, 1).cpu().numpy(), first)


def test_noalloc_refuses_more_than_its_scratch_holds():
    torch = pytest.importorskip("torch")
    lib = physgpu.load_library()
    n = 32769
    pos, _, m = ics.plummer(n, seed=3)
    X, M, A = _dev(torch, pos, m)
    torch.cuda.synchronize()
    st, err = _call(lib, n, X, M, A, 1.0, 0.01, F64, torch.cuda.current_stream().cuda_stream)
    assert st == physgpu.ERR_ARG
    assert "32768" in err
