"""Batched and asynchronous solves (s2l_gpu_solve_batch, s2l_gpu_submit / poll / wait / cancel).

Every solve runs on a workspace of its own, so a solve gives the same bits alone, in a batch and
through the worker threads when continuous batching is off (s2l_gpu_serve_batching 0; the batched
serving path is tested in test_gpu_serving_batching.py); cancellation stops a queued solve before it
starts and a running one before its next iteration; a setup with queued or running solves refuses to
be destroyed.
"""
import time

import numpy as np
import pytest

from conftest import small_setup

pytestmark = pytest.mark.gpu


def _rhs(n, k, seed=11):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-1.0, 1.0, n) for _ in range(k)]


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
def test_batch_same_bits_as_single_solves(method):
    from s2l_b200 import capi
    ctx = capi.Context(0)
    w, st = small_setup("bubbles3d")
    g = capi.GpuSetup(ctx, st)
    bs = _rhs(st.n, 3)
    kw = dict(rtol=1e-9) if method == "bicgstab" else dict(restart=w.restart, rtol=1e-9)
    single = [(g.gmres(b, **kw) if method == "gmres" else g.bicgstab(b, **kw)) for b in bs]
    out = g.solve_batch(bs, method=method, **kw)
    for (xs, rs), (xb, rb, status) in zip(single, out):
        assert status == 0 and rb["converged"]
        assert rb["iterations"] == rs["iterations"]
        assert np.array_equal(xs, xb)
    g.close()
    ctx.close()


def test_submit_across_setups_same_bits():
    from s2l_b200 import capi
    ctx = capi.Context(0)
    ctx.serve_start(3, batching=0)
    w1, st1 = small_setup("bubbles3d")
    w2, st2 = small_setup("poisson2d")
    g1, g2 = capi.GpuSetup(ctx, st1), capi.GpuSetup(ctx, st2)
    jobs = [(g1, b, "gmres") for b in _rhs(st1.n, 3)] + [(g2, b, "bicgstab") for b in _rhs(st2.n, 2, 12)]
    alone = [(g.gmres(b, rtol=1e-9) if m == "gmres" else g.bicgstab(b, rtol=1e-9)) for g, b, m in jobs]
    tickets = [g.submit(b, method=m, rtol=1e-9) for g, b, m in jobs]
    for t, (xa, ra) in zip(tickets, alone):
        x, r, status = t.wait(120.0)
        assert status == 0 and t.state() == capi.JOB_DONE, t.info()["error"]
        assert r["iterations"] == ra["iterations"] and np.array_equal(x, xa)
        info = t.info()
        assert info["queue_ms"] >= 0.0 and info["run_ms"] > 0.0 and info["error"] == ""
        t.free()
    g1.close()
    g2.close()
    ctx.close()


@pytest.mark.parametrize("batching", [0, -1])
def test_cancel_queued_and_running(batching):
    from s2l_b200 import capi
    ctx = capi.Context(0)
    ctx.serve_start(1, batching=batching)
    w, st = small_setup("bubbles3d")
    g = capi.GpuSetup(ctx, st)
    b = _rhs(st.n, 1)[0]
    # rtol 0 with the L2 test never converges: the first solve runs until it is canceled
    long = g.submit(b, restart=w.restart, rtol=0.0, maxit=10**7, history_cap=0)
    queued = g.submit(b, restart=w.restart, rtol=1e-8)
    queued.cancel()
    deadline = time.time() + 30.0
    while long.state() != capi.JOB_RUNNING and time.time() < deadline:
        time.sleep(0.01)
    assert long.state() == capi.JOB_RUNNING
    with pytest.raises(TimeoutError):
        long.wait(0.05)
    # the setup refuses to be destroyed while a solve is queued or running
    assert g.lib.s2l_gpu_setup_destroy(g.h) == 7
    long.cancel()
    _, _, st_long = long.wait(60.0)
    _, _, st_queued = queued.wait(60.0)
    assert st_long == capi.ERR_CANCELED and long.state() == capi.JOB_CANCELED
    assert st_queued == capi.ERR_CANCELED and queued.state() == capi.JOB_CANCELED
    assert "canceled" in long.info()["error"]
    if batching == 0:  # (a block runner may have given it a slot before the cancel)
        assert queued.info()["run_ms"] == 0.0
    # the worker and the setup stay usable
    x, r, status = g.submit(b, restart=w.restart, rtol=1e-8).wait(60.0)
    assert status == 0 and r["converged"]
    assert np.linalg.norm(st.b - st.A @ x) >= 0.0
    long.free()
    queued.free()
    g.close()
    ctx.close()


def test_submit_needs_workers_and_reports_errors():
    from s2l_b200 import capi
    ctx = capi.Context(0)
    w, st = small_setup("poisson2d")
    g = capi.GpuSetup(ctx, st)
    with pytest.raises(capi.S2LError) as e:
        g.submit(st.b)
    assert e.value.code == 7
    ctx.serve_start(2)
    t = g.submit(st.b, atol=1e-6)  # an absolute tolerance needs the OpenFOAM norm: fails in the worker
    _, _, status = t.wait(60.0)
    assert status == 1 and "OpenFOAM" in t.info()["error"]
    t.free()
    g.close()
    ctx.close()


def test_hbm_admission_waits_for_memory_instead_of_failing():
    """With a budget that fits one solve's buffers but not two, concurrent solves on one setup are
    admitted one after another as workspaces come free (each result the same as alone); with a
    budget below one solve's buffers the call fails with S2L_ERR_OOM instead of waiting."""
    from s2l_b200 import capi
    w, st = small_setup("bubbles3d")
    probe = capi.Context(0)
    g0 = capi.GpuSetup(probe, st)
    d0 = g0.device_bytes()
    bs = _rhs(st.n, 4, 31)
    alone = [g0.gmres(b, restart=w.restart, rtol=1e-9) for b in bs]
    d1 = g0.device_bytes()  # setup + one workspace with its Krylov basis
    g0.close()
    probe.close()
    assert d1 > d0
    ctx = capi.Context(0, hbm_budget=d1 + (d1 - d0) // 2)
    ctx.serve_start(4, batching=0)
    g = capi.GpuSetup(ctx, st)
    tickets = [g.submit(b, restart=w.restart, rtol=1e-9) for b in bs]
    for t, (xa, ra) in zip(tickets, alone):
        x, r, status = t.wait(300.0)
        assert status == 0, t.info()["error"]
        assert r["iterations"] == ra["iterations"] and np.array_equal(x, xa)
        t.free()
    assert g.device_bytes() <= d1 + (d1 - d0) // 2
    g.close()
    ctx.close()
    tight = capi.Context(0, hbm_budget=d0 + (d1 - d0) // 4)
    g = capi.GpuSetup(tight, st)
    with pytest.raises(capi.S2LError) as e:
        g.gmres(bs[0], restart=w.restart, rtol=1e-9)
    assert e.value.code == 2 and "budget" in str(e.value)
    g.close()
    tight.close()


def test_engine_caches_setups_and_evicts_idle_ones_under_the_budget():
    """Setups are cached per matrix (a repeated request builds nothing); with a budget that holds two
    of the three setups, a request on the third evicts the least recently used idle one; every
    result equals the same solve on a context of its own."""
    from s2l_b200 import capi
    from s2l_b200.serving import Engine
    cases = {"a": small_setup("bubbles3d")[1], "b": small_setup("poisson2d")[1], "c": small_setup("convdiff3d")[1]}
    probe = capi.Context(0)
    size, alone = {}, {}
    for key, st in cases.items():
        g = capi.GpuSetup(probe, st)
        alone[key] = g.gmres(st.b, restart=30, rtol=1e-9)
        size[key] = g.device_bytes()
        g.close()
    probe.close()
    pair = max(size["a"] + size["b"], size["b"] + size["c"], size["a"] + size["c"])
    budget = pair + min(size.values()) // 4
    assert budget < sum(size.values())
    eng = Engine(0, hbm_budget=budget, workers=2, batching=0)
    made = []

    def maker(key):
        def make():
            made.append(key)
            return cases[key]
        return make

    for key in ("a", "b", "a", "c", "b", "a"):
        t = eng.submit(key, maker(key), cases[key].b, restart=30, rtol=1e-9)
        x, r, status = t.wait(120.0)
        assert status == 0, t.info()["error"]
        assert r["iterations"] == alone[key][1]["iterations"] and np.array_equal(x, alone[key][0])
        t.free()
    assert made[:2] == ["a", "b"] and "c" in made  # the repeated "a" hit the cache
    assert eng.evictions >= 1 and len(eng.resident()) <= 2
    eng.close()


def test_engine_sequence_update_levels():
    """Engine.update along a sequence: "refactorize" gives the solve of the oracle refactorized on
    the new values (iterations +-1), "reuse" the oracle with the old preconditioner."""
    import dataclasses
    import scipy.sparse as sp
    from oracle.oracle import OracleSetup, refactor_setup
    from s2l_b200.serving import Engine
    w, st = small_setup("bubbles3d")
    eng = Engine(0, workers=1)
    eng.setup("m", lambda: st, options={"refactor": 1})
    rng = np.random.default_rng(12)
    for level in ("refactorize", "reuse"):
        d = 1.0 + 0.1 * rng.uniform(-1.0, 1.0, st.n)
        A = st.A.tocsr()
        rows = np.repeat(np.arange(st.n), np.diff(A.indptr))
        A2 = sp.csr_matrix((A.data * d[rows] * d[A.indices], A.indices, A.indptr), shape=A.shape)
        eng.update("m", A2.data, level=level)
        ref = refactor_setup(st, A2) if level == "refactorize" else None
        if ref is None:  # reuse: the preconditioner of the last refactorization, the new operator
            ref = dataclasses.replace(last, A=A2)
        o = OracleSetup(ref)
        t = eng.submit("m", lambda: st, st.b, restart=w.restart, rtol=1e-8)
        x, r, status = t.wait(120.0)
        t.free()
        _, ro = o.gmres(st.b, restart=w.restart, rtol=1e-8)
        assert status == 0 and r["converged"] and abs(r["iterations"] - ro["iterations"]) <= 1
        assert np.linalg.norm(st.b - A2 @ x) <= 1.1e-8 * np.linalg.norm(st.b)
        o.close()
        if level == "refactorize":
            last = ref
    eng.close()
