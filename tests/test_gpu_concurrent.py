"""Concurrent solve-phase calls on one setup, from several host threads.

Each call holds its own workspace (stream, work vectors, Krylov basis), so the same call gives the
same bits alone and in the mix: the reductions use a fixed grid and order, and the shared factors
are only read.  Compared bit for bit with the results of the same calls made one after another.
"""
import threading

import numpy as np
import pytest

from conftest import small_setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from s2l_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def _run_threads(fns):
    out = [None] * len(fns)
    err = []

    def body(k):
        try:
            out[k] = fns[k]()
        except Exception as e:  # reported on the main thread
            err.append(e)

    ts = [threading.Thread(target=body, args=(k,)) for k in range(len(fns))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if err:
        raise err[0]
    return out


@pytest.mark.parametrize("name,pou", [("bubbles3d", "boolean"), ("poisson2d", "multiplicity")])
def test_concurrent_gmres_same_bits_as_alone(ctx, name, pou):
    from s2l_b200.capi import GpuSetup
    _, st = small_setup(name, pou=pou)
    g = GpuSetup(ctx, st)
    rng = np.random.default_rng(77)
    bs = [rng.uniform(-1, 1, st.n) for _ in range(4)]
    alone = [g.gmres(b, restart=30, rtol=1e-9) for b in bs]
    bytes_alone = g.device_bytes()
    for _ in range(2):
        mixed = _run_threads([lambda b=b: g.gmres(b, restart=30, rtol=1e-9) for b in bs])
        for (xa, ra), (xm, rm) in zip(alone, mixed):
            assert ra["converged"] and rm["converged"]
            assert ra["iterations"] == rm["iterations"]
            assert np.array_equal(xa, xm)
            assert np.array_equal(ra["history"], rm["history"])
    assert g.device_bytes() >= bytes_alone
    g.close()


def test_concurrent_mixed_calls(ctx):
    """GMRES, BiCGStab, apply and SpMV on one setup at once, each equal to its lone result."""
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("convdiff3d")
    g = GpuSetup(ctx, st)
    rng = np.random.default_rng(78)
    b = rng.uniform(-1, 1, st.n)
    r = rng.standard_normal(st.n)
    calls = [lambda: g.gmres(b, restart=20, rtol=1e-9)[0],
             lambda: g.bicgstab(b, rtol=1e-9)[0],
             lambda: g.apply(r),
             lambda: g.spmv(r),
             lambda: g.one_level_apply(r)]
    alone = [c() for c in calls]
    mixed = _run_threads(calls + calls)
    for k, m in enumerate(mixed):
        assert np.array_equal(m, alone[k % len(calls)])
    g.close()
