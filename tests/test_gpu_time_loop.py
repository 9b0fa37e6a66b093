"""Sequences of solves with setup reuse on the device (the reference's time loop, ``--steps``).

The loop of s2l_b200.time_loop runs on the device setup (Rebuild = a new setup, Refactorize =
s2l_gpu_refactor, Reuse = the setup kept) and, as the checker, on the oracle (Refactorize =
oracle.refactor_setup).  Every solve must take the oracle's iterations +-1, converge, and the
levels must be the reference's ("201010" refactor, "222222" off, "20101010" one-level auto); refactor
and off must give the same iterations on the first step, as in the reference's test
(``test/test_reuse.cpp:424-444``).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.oracle import OracleSetup, refactor_setup
from s2l_b200 import workloads as W
from s2l_b200.time_loop import TimeLoopConfig, UpdateLevel, levels, run_time_loop

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from s2l_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


class OracleSolver:
    """The oracle behind the loop's solver interface (the checker)."""

    def __init__(self, st, refactor):
        self.st, self.o = st, OracleSetup(st)

    def refactor(self, vals):
        A2 = sp.csr_matrix((np.asarray(vals), self.st.A.indices, self.st.A.indptr), shape=self.st.A.shape)
        self.o.close()
        self.st = refactor_setup(self.st, A2)
        self.o = OracleSetup(self.st)

    def gmres(self, b, **kw):
        return self.o.gmres(b, **kw)

    def bicgstab(self, b, **kw):
        return self.o.bicgstab(b, **kw)

    def close(self):
        self.o.close()


def small_bubbles(coarse="deflated"):
    w = W.bubbles3d(12, 8, nbubbles=6, overlap=1)
    w.opts.nev = 8
    w.opts.coarse = coarse
    return w


def both(ctx, w, **kw):
    cfg = TimeLoopConfig(**kw)
    g = run_time_loop(w, cfg, ctx=ctx, workers=1)
    o = run_time_loop(w, TimeLoopConfig(**kw), make_solver=OracleSolver, workers=1)
    assert levels(g) == levels(o)
    for rg, ro in zip(g, o):
        assert rg.converged and ro.converged
        assert abs(rg.iterations - ro.iterations) <= 1, (rg.step, rg.corrector, rg.iterations, ro.iterations)
        assert rg.true_rel_residual <= 1.1 * w.rtol
    return g


def test_time_loop_refactor_and_off_match_oracle(ctx):
    w = small_bubbles()
    ra = both(ctx, w, steps=3, correctors=2, reuse="refactor")
    assert levels(ra) == "201010"
    ro = both(ctx, w, steps=3, correctors=2, reuse="off")
    assert levels(ro) == "222222"
    assert ra[0].iterations == ro[0].iterations and ra[1].iterations == ro[1].iterations


def test_time_loop_auto_and_one_level(ctx):
    w = small_bubbles()
    rb = run_time_loop(w, TimeLoopConfig(steps=3, correctors=2, reuse="auto"), ctx=ctx, workers=1)
    assert rb[0].level == UpdateLevel.REBUILD and all(r.converged for r in rb)
    assert all(rb[k].level == UpdateLevel.REUSE for k in (1, 3, 5))
    assert all(rb[k].level != UpdateLevel.REUSE for k in (2, 4))
    r1 = both(ctx, small_bubbles("none"), steps=4, correctors=2, reuse="auto")
    assert levels(r1) == "20101010"


def test_time_loop_warm_start_final_tolerances_match_oracle(ctx):
    w = small_bubbles()
    recs = both(ctx, w, steps=2, correctors=3, reuse="refactor", warm_start=True, final_rtol=1e-10)
    assert [r.final_corrector for r in recs] == [False, False, True] * 2


@pytest.mark.parametrize("reuse", [False, True])
def test_time_loop_amg_local_solvers_match_oracle(ctx, reuse):
    """AMG local solvers along the sequence: each Refactorize sets the hierarchies up again on the
    host (new, or with kept transfer operators) and uploads them; every solve matches the oracle's."""
    w = small_bubbles()
    w.opts.local_approx = "amg"
    w.opts.amg_coarse_enough = 100
    w.opts.amg_reuse = reuse
    recs = both(ctx, w, steps=3, correctors=1, reuse="refactor")
    assert levels(recs) == "211"
