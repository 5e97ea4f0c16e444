"""Failure paths on the device, made without faulting the GPU.

* A bounded device wait that runs out: the radix sort's look-back waits are
  given a bound of 0 re-reads (phys_debug_set_wait_limit), so the first tile
  that finds a predecessor still ranking gives up, as a stalled predecessor
  would after the default bound.  The evaluation must stop before any kernel
  builds on the unfinished order, return PHYS_ERR_TIMEOUT, and leave the
  context able to compute the same forces as before.
* Two contexts used at once from two threads: contexts share no state (the
  kernels' shared-memory limits and occupancies are kept per context), so
  each computes what it computes alone."""
import threading

import numpy as np
import pytest

import oracle
import physgpu
import physgpu.ics as ics
from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, GROUP_WALK, make_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flags,leaf_cap,precision", [(GROUP_WALK, 8, F32C), (0, 1, F64)])
def test_sort_wait_timeout_is_reported_and_context_recovers(flags, leaf_cap, precision):
    n = 1 << 21  # 1024 tiles per sort pass, 8 passes
    pos, _, m = ics.plummer(n, seed=21)
    p = make_params(1.0, 0.01, 0.5, BARNES_HUT, precision, leaf_cap, flags)
    with physgpu.Context(0) as ctx:
        ctx.upload(pos, None, m)
        ref = ctx.gravity_accel(p)
        ctx.set_wait_limit(0)
        timeouts = 0
        for _ in range(20):
            try:
                a = ctx.gravity_accel(p)
            except physgpu.PhysError as e:
                assert e.status == physgpu.ERR_TIMEOUT, e
                timeouts += 1
                if timeouts >= 3:
                    break
            else:  # no wait happened: the result is the normal one
                assert np.array_equal(a, ref)
        assert timeouts > 0, "no look-back wait occurred in 20 sorts of 2^21 keys"
        ctx.set_wait_limit(-1)
        assert np.array_equal(ctx.gravity_accel(p), ref)
        # the direct sum has no bounded wait and is unaffected
        small, _, ms = ics.plummer(2048, seed=3)
        ctx.upload(small, None, ms)
        d = make_params(1.0, 0.01, 0.5, DIRECT, F64_EXACT)
        assert np.array_equal(ctx.gravity_forces(d), oracle.direct_forces(small, ms, 1.0, 0.01))


def test_two_contexts_from_two_threads():
    pos, _, m = ics.plummer(65536, seed=31)
    pos2, _, m2 = ics.plummer(4096, seed=32)
    pg = make_params(1.0, 0.01, 0.5, BARNES_HUT, F32C, 8, GROUP_WALK)
    pd = make_params(1.0, 0.01, 0.5, DIRECT, F64)
    with physgpu.Context(0) as c0:
        c0.upload(pos, None, m)
        ref_g = c0.gravity_accel(pg)
        c0.upload(pos2, None, m2)
        ref_d = c0.gravity_accel(pd)
    out = {}
    errors = []

    def run(key, P, params, reps):
        try:
            with physgpu.Context(0) as c:
                c.upload(*P)
                for r in range(reps):
                    out[(key, r)] = c.gravity_accel(params)
        except Exception as e:  # reported below
            errors.append(e)

    ts = [threading.Thread(target=run, args=("g", (pos, None, m), pg, 4)),
          threading.Thread(target=run, args=("d", (pos2, None, m2), pd, 8))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    for r in range(4):
        assert np.array_equal(out[("g", r)], ref_g)
    for r in range(8):
        assert np.array_equal(out[("d", r)], ref_d)
