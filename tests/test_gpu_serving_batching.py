"""Continuous batching of the asynchronous GMRES solves (s2l_gpu_serve_batching, on by default).

A worker runs a block runner per setup (and restart length, variant): up to K requests at once, each
in a column of one block, every Arnoldi step shared, each column with its own GMRES recurrence,
restart cycle and convergence test (src/solver/gmres.cpp:18-161).  Requests that arrive while
others run take a free slot at the next step; a converged request returns at once.

The contract tested here: a request's result does not depend on which other requests share its
block, when they arrived or where its cycle sits in the basis ring; it is bitwise the result of the
same request alone in the engine.  Against the unbatched solve of the same request (s2l_gpu_gmres)
the iterations agree to +-1 and both reach the FP64 true residual (the block reductions group the
sums differently, so the bits differ).
"""
import time

import numpy as np
import pytest

from conftest import small_setup

pytestmark = pytest.mark.gpu


def _rhs(n, k, seed):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-1.0, 1.0, n) for _ in range(k)]


def _alone(g, bs, **kw):
    """Each request alone through the engine (a runner with one occupied slot)."""
    out = []
    for b in bs:
        t = g.submit(b, **kw)
        x, r, status = t.wait(300.0)
        assert status == 0, t.info()["error"]
        out.append((x, r))
        t.free()
    return out


def _mix(g, bs, first, **kw):
    """`first` requests, then (once one of them runs) the others, while the first ones run."""
    tickets = [g.submit(b, **kw) for b in bs[:first]]
    t_sub = [time.perf_counter()] * first
    deadline = time.time() + 60.0
    from s2l_b200 import capi
    while all(t.state() == capi.JOB_QUEUED for t in tickets) and time.time() < deadline:
        time.sleep(0.0005)
    for b in bs[first:]:
        tickets.append(g.submit(b, **kw))
        t_sub.append(time.perf_counter())
    out = []
    for t, ts in zip(tickets, t_sub):
        x, r, status = t.wait(300.0)
        assert status == 0, t.info()["error"]
        info = t.info()
        out.append((x, r, ts + 1e-3 * info["queue_ms"], ts + 1e-3 * (info["queue_ms"] + info["run_ms"])))
        t.free()
    return out


@pytest.mark.parametrize("case", ["bubbles_fp64", "convdiff_fp32_flexible", "bubbles_short_restart"])
def test_a_request_gives_the_same_bits_alone_and_in_the_mix(case):
    from s2l_b200 import capi
    if case == "convdiff_fp32_flexible":
        w, st = small_setup("convdiff3d", precision="single")
        kw = dict(restart=w.restart, rtol=1e-10, flexible=True, strict=True)
    elif case == "bubbles_short_restart":
        # cycles of 4 steps in a ring of 5 blocks: columns restart at different steps, so their
        # windows wrap around the ring
        w, st = small_setup("bubbles3d")
        kw = dict(restart=4, rtol=1e-10, maxit=2000)
    else:
        w, st = small_setup("bubbles3d")
        kw = dict(restart=w.restart, rtol=1e-11)
    ctx = capi.Context(0)
    ctx.serve_start(2)  # continuous batching on (automatic slots)
    g = capi.GpuSetup(ctx, st)
    bs = _rhs(st.n, 7, 5)
    bs[3] = bs[3] * 1e3  # a different scale: its own norms and convergence
    alone = _alone(g, bs, **kw)
    mix = _mix(g, bs, 3, **kw)
    overlap = any(s2 < e1 and s1 < e2 for i, (_, _, s1, e1) in enumerate(mix) for (_, _, s2, e2) in mix[i + 1:])
    assert overlap, "no two requests ran at the same time"
    for (xa, ra), (xm, rm, _, _) in zip(alone, mix):
        assert rm["converged"] and rm["iterations"] == ra["iterations"] and rm["restarts"] == ra["restarts"]
        assert np.array_equal(xm, xa)
    # against the unbatched solve of each request
    for b, (xa, ra) in zip(bs, alone):
        xs, rs = g.gmres(b, **kw)
        assert abs(ra["iterations"] - rs["iterations"]) <= 1
        assert np.linalg.norm(b - st.A @ xa) <= 1.1 * kw["rtol"] * np.linalg.norm(b)
    g.close()
    ctx.close()


def test_setups_variants_and_methods_served_together():
    """Requests on two setups (FP64 factors, FP32 factors with flexible GMRES) and BiCGStab requests
    (never batched) submitted together: every GMRES result is the bits of the same request alone in
    the engine, every BiCGStab result the bits of s2l_gpu_bicgstab."""
    from s2l_b200 import capi
    w1, st1 = small_setup("bubbles3d")
    w2, st2 = small_setup("convdiff3d", precision="single")
    ctx = capi.Context(0)
    ctx.serve_start(4)
    g1, g2 = capi.GpuSetup(ctx, st1), capi.GpuSetup(ctx, st2)
    kw1 = dict(restart=w1.restart, rtol=1e-10)
    kw2 = dict(restart=w2.restart, rtol=1e-10, flexible=True, strict=True)
    b1, b2 = _rhs(st1.n, 4, 21), _rhs(st2.n, 4, 22)
    a1, a2 = _alone(g1, b1, **kw1), _alone(g2, b2, **kw2)
    bic = [g1.bicgstab(b, rtol=1e-9) for b in b1[:2]]
    jobs = [(g1, b, kw1, "gmres") for b in b1] + [(g2, b, kw2, "gmres") for b in b2] + \
           [(g1, b, dict(rtol=1e-9), "bicgstab") for b in b1[:2]]
    order = np.random.default_rng(3).permutation(len(jobs))
    tickets = {int(i): jobs[i][0].submit(jobs[i][1], method=jobs[i][3], **jobs[i][2]) for i in order}
    want = [a for a in a1] + [a for a in a2] + bic
    for i in range(len(jobs)):
        x, r, status = tickets[i].wait(300.0)
        assert status == 0, tickets[i].info()["error"]
        assert r["iterations"] == want[i][1]["iterations"] and np.array_equal(x, want[i][0]), i
        tickets[i].free()
    g1.close()
    g2.close()
    ctx.close()


def test_cancel_and_a_failing_request_leave_the_others_untouched():
    """In one runner: a request that never converges (rtol 0) is canceled while it runs, a request
    with a non-finite right-hand side fails alone (S2L_ERR_NUMERIC); the other requests keep the bits
    of their solves alone, and a request that takes a freed slot afterwards too."""
    from s2l_b200 import capi
    w, st = small_setup("bubbles3d")
    ctx = capi.Context(0)
    ctx.serve_start(1)
    g = capi.GpuSetup(ctx, st)
    kw = dict(restart=w.restart, rtol=1e-10)
    good = _rhs(st.n, 4, 41)
    alone = _alone(g, good, **kw)
    long = g.submit(good[0], restart=w.restart, rtol=0.0, maxit=10**7, history_cap=0)
    deadline = time.time() + 30.0
    while long.state() != capi.JOB_RUNNING and time.time() < deadline:
        time.sleep(0.001)
    bad_b = good[1].copy()
    bad_b[5] = np.nan
    bad = g.submit(bad_b, **kw)
    others = [g.submit(b, **kw) for b in good[:3]]
    _, _, st_bad = bad.wait(120.0)
    assert st_bad == 4 and "non-finite" in bad.info()["error"]
    for t, (xa, ra) in zip(others, alone[:3]):
        x, r, status = t.wait(120.0)
        assert status == 0 and np.array_equal(x, xa) and r["iterations"] == ra["iterations"]
        t.free()
    assert long.state() == capi.JOB_RUNNING
    # while the long request still runs: the lowest free slot is the one the failed request held
    t3 = g.submit(good[3], **kw)
    x, r, status = t3.wait(120.0)
    assert status == 0 and np.array_equal(x, alone[3][0])
    t3.free()
    long.cancel()
    _, _, st_long = long.wait(60.0)
    assert st_long == capi.ERR_CANCELED and long.state() == capi.JOB_CANCELED
    long.free()
    bad.free()
    g.close()
    ctx.close()


def test_serve_batching_off_runs_every_request_alone():
    """slots = 0: the first-in-first-out path, each request bitwise the unbatched solve."""
    from s2l_b200 import capi
    w, st = small_setup("bubbles3d")
    ctx = capi.Context(0)
    ctx.serve_start(2, batching=0)
    g = capi.GpuSetup(ctx, st)
    bs = _rhs(st.n, 3, 51)
    single = [g.gmres(b, restart=w.restart, rtol=1e-9) for b in bs]
    tickets = [g.submit(b, restart=w.restart, rtol=1e-9) for b in bs]
    for t, (xs, rs) in zip(tickets, single):
        x, r, status = t.wait(120.0)
        assert status == 0 and np.array_equal(x, xs) and r["iterations"] == rs["iterations"]
        t.free()
    with pytest.raises(capi.S2LError):
        ctx.serve_batching(17)
    g.close()
    ctx.close()


def test_runner_fits_the_hbm_budget_with_fewer_slots():
    """A budget that holds the setup and a block of a few columns but not the automatic width: the
    runner halves its slots until its block fits, and every request still converges like alone."""
    from s2l_b200 import capi
    w, st = small_setup("bubbles3d")
    probe = capi.Context(0)
    g0 = capi.GpuSetup(probe, st)
    d0 = g0.device_bytes()
    width = int(g0.stat("block_width"))
    g0.gmres_block(np.stack(_rhs(st.n, width, 61)), restart=w.restart, rtol=1e-9)
    d2 = g0.device_bytes()  # the setup and one workspace with a block of `width` columns
    g0.close()
    probe.close()
    assert width >= 4
    budget = d0 + (d2 - d0) // 3  # room for a block of about a third of the width
    ctx = capi.Context(0, hbm_budget=budget)
    ctx.serve_start(1, batching=width)  # runners of the full width: they must halve to fit
    g = capi.GpuSetup(ctx, st)
    bs = _rhs(st.n, 5, 62)
    tickets = [g.submit(b, restart=w.restart, rtol=1e-9) for b in bs]
    for t, b in zip(tickets, bs):
        x, r, status = t.wait(300.0)
        assert status == 0, t.info()["error"]
        assert r["converged"] and np.linalg.norm(b - st.A @ x) <= 1.1e-9 * np.linalg.norm(b)
        t.free()
    assert g.device_bytes() <= budget
    g.close()
    ctx.close()
