"""Sequences of solves with setup reuse (the reference's time loop and reuse policy), host side.

* ReusePolicy against the reference's own known answers (``test/test_reuse.cpp:50-110``);
* the right-hand side of solve (step, corrector) bit for bit against libstdc++'s
  ``std::mt19937_64(std::seed_seq{seed, step, corrector, 0x5eed})`` (tests/golden/seed_seq_rhs.json,
  made by tests/golden/make_seed_seq_golden.py);
* the loop's levels and calls with a recording stand-in for the device setup: the level strings of
  the reference's time-loop test (``test/test_reuse.cpp:424-444``: "201010" refactor, "222222" off,
  "20101010" one-level auto), refactorization values in the setup's order, warm start and final
  tolerances.
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from s2l_b200 import sequence as seqmod
from s2l_b200 import workloads as W
from s2l_b200.rng import random_rhs_step
from s2l_b200.time_loop import ReusePolicy, TimeLoopConfig, UpdateLevel, levels, run_time_loop

HERE = os.path.dirname(os.path.abspath(__file__))
RB, RF, RU = UpdateLevel.REBUILD, UpdateLevel.REFACTORIZE, UpdateLevel.REUSE


def test_policy_iterations_per_decade():
    P = ReusePolicy
    assert abs(P.per_decade(10, 1e-5) - 2.0) < 1e-12
    assert P.per_decade(0, 1e-5) == 0.0 and P.per_decade(5, 1.0) == 0.0


def test_policy_auto_break_even():
    # rebuild 2.0 s, refactorize 0.2 s: premium 1.8 s; q_ref = 10 its / 8 decades; 0.1 s per iteration
    a = ReusePolicy("auto", 0.0, 0)
    a.record(RB, 10, 1e-8, True, 2.0, 1.0)
    assert a.decide(False) == RU and a.decide(True) == RF and a.wasted == 0.0
    a.record(RF, 15, 1e-8, True, 0.2, 1.5)  # 5 extra iterations: 0.5 s
    assert abs(a.wasted - 0.5) < 1e-12 and a.decide(True) == RF
    a.record(RU, 15, 1e-8, True, 0.0, 1.5)
    a.record(RF, 19, 1e-8, True, 0.2, 1.9)  # 1.9 s > 1.8 s
    assert abs(a.wasted - 1.9) < 1e-12 and abs(a.rebuild_premium() - 1.8) < 1e-12
    assert a.decide(True) == RB and a.decide(False) == RU
    a.record(RB, 12, 1e-8, True, 2.5, 1.2)  # new reference 1.5, counter reset
    assert a.decide(True) == RF and a.wasted == 0.0 and abs(a.reference() - 1.5) < 1e-12


def test_policy_auto_safety_nets():
    g = ReusePolicy("auto", 1.5, 0)
    g.record(RB, 10, 1e-8, True, 1e9, 1.0)
    g.record(RF, 16, 1e-8, True, 0.1, 1.6)  # q = 2.0 > 1.5 * 1.25
    assert g.decide(True) == RB
    n = ReusePolicy("auto", 0.0, 0)
    n.record(RB, 10, 1e-8, True, 1e9, 1.0)
    n.record(RF, 500, 1e-3, False, 0.1, 50.0)  # not converged
    assert n.decide(True) == RB
    b = ReusePolicy("auto", 0.0, 2)
    b.record(RB, 10, 1e-8, True, 1e9, 1.0)
    assert b.decide(True) == RF
    b.record(RF, 10, 1e-8, True, 0.1, 1.0)
    assert b.decide(True) == RF
    b.record(RF, 10, 1e-8, True, 0.1, 1.0)
    assert b.decide(True) == RB


def test_policy_robust_costs():
    P = ReusePolicy
    assert P.lower_median([]) == 0.0 and P.lower_median([3.0]) == 3.0 and P.lower_median([5.0, 1.0]) == 1.0
    assert P.lower_median([4.0, 1.0, 2.0]) == 2.0 and P.lower_median([4.0, 1.0, 2.0, 3.0]) == 2.0
    s = P("auto", 0.0, 0)
    s.record(RB, 10, 1e-8, True, 2.0, 1.0)
    s.record(RF, 10, 1e-8, True, 0.2, 1.0)
    s.record(RB, 10, 1e-8, True, 30.0, 1.0)  # stalled rebuild
    assert abs(s.rebuild_premium() - 1.8) < 1e-12
    s.record(RF, 10, 1e-8, True, 9.0, 1.0)   # stalled refactorization
    assert abs(s.rebuild_premium() - 1.8) < 1e-12


def test_policy_off_and_refactor_modes():
    c = ReusePolicy("off", 0.0, 0)
    assert c.decide(False) == RB and c.decide(True) == RB
    r = ReusePolicy("refactor", 0.0, 0)
    r.record(RB, 10, 1e-8, True, 2.0, 1.0)
    r.record(RF, 900, 1e-3, False, 0.1, 90.0)
    assert r.decide(False) == RU and r.decide(True) == RF
    with pytest.raises(ValueError):
        ReusePolicy("sometimes")


def test_policy_kinds_have_their_own_reference():
    p = ReusePolicy("auto", 0.0, 0)
    p.record(RB, 10, 1e-8, True, 2.0, 1.0, kind=0)  # q_ref(0) = 1.25
    p.record(RU, 4, 1e-4, True, 0.0, 0.4, kind=1)   # q_ref(1) = 1.0: its own reference, nothing wasted
    assert p.wasted == 0.0 and abs(p.reference(1) - 1.0) < 1e-12
    p.record(RF, 6, 1e-4, True, 0.2, 0.6, kind=1)   # 2 extra iterations of kind 1: 0.2 s
    assert abs(p.wasted - 0.2) < 1e-12 and abs(p.reference(0) - 1.25) < 1e-12


def test_random_rhs_step_matches_libstdcxx():
    with open(os.path.join(HERE, "golden", "seed_seq_rhs.json")) as f:
        d = json.load(f)
    for c in d["cases"]:
        ref = np.array([float.fromhex(v) for v in c["values_hex"]])
        got = random_rhs_step(d["n"], c["seed"], c["step"], c["corrector"])
        assert np.array_equal(got, ref), (c["seed"], c["step"], c["corrector"])


class Recorder:
    """Stand-in for the device setup: solves exactly with scipy, records what the loop asks."""
    log = []

    def __init__(self, st, refactor):
        self.st, self.A, self.can_refactor = st, st.A.tocsr(), refactor
        Recorder.log.append(("build", st))

    def refactor(self, vals):
        assert self.can_refactor
        self.A = sp.csr_matrix((np.asarray(vals), self.st.A.indices, self.st.A.indptr), shape=self.st.A.shape)
        Recorder.log.append(("refactor", np.array(vals)))

    def gmres(self, b, x0=None, restart=30, rtol=1e-8, maxit=1000, flexible=False, strict=False, stop_norm="l2",
              atol=0.0):
        Recorder.log.append(("gmres", np.array(x0), rtol, atol, stop_norm, np.array(b)))
        x = sp.linalg.spsolve(self.A.tocsc(), b)
        r0 = np.linalg.norm(b - self.A @ x0) / np.linalg.norm(b)
        return x, {"converged": True, "iterations": 10, "true_rel_residual": 1e-9, "history": np.array([r0]),
                   "initial_residual_of": 1.0, "final_residual_of": 1e-9}

    def close(self):
        Recorder.log.append(("close",))


def small_bubbles(coarse="deflated"):
    w = W.bubbles3d(10, 4, nbubbles=4, overlap=1)
    w.opts.nev = 6
    w.opts.coarse = coarse
    return w


def run(w, **kw):
    Recorder.log = []
    recs = run_time_loop(w, TimeLoopConfig(**kw), make_solver=Recorder, workers=1)
    return recs, list(Recorder.log)


def test_time_loop_levels_of_the_reference_test():
    w = small_bubbles()
    ra, log = run(w, steps=3, correctors=2, reuse="refactor")
    assert levels(ra) == "201010" and all(r.converged for r in ra)
    assert [e[0] for e in log if e[0] != "gmres"] == ["build", "refactor", "refactor", "close"]
    ro, log = run(w, steps=3, correctors=2, reuse="off")
    assert levels(ro) == "222222"
    assert [e[0] for e in log].count("build") == 6 and [e[0] for e in log].count("close") == 6
    rb, _ = run(w, steps=3, correctors=2, reuse="auto")
    assert len(rb) == 6 and rb[0].level == RB
    assert all(rb[k].level == RU for k in (1, 3, 5)) and all(rb[k].level != RU for k in (2, 4))
    r1, _ = run(small_bubbles("none"), steps=4, correctors=2, reuse="auto")  # one-level: as refactor
    assert levels(r1) == "20101010"


def test_time_loop_refactorizes_with_the_step_matrix_in_setup_order():
    import dataclasses
    w = small_bubbles()
    recs, log = run(w, steps=3, correctors=1, reuse="refactor")
    st = log[0][1]
    vals = [e[1] for e in log if e[0] == "refactor"]
    for step, v in zip((1, 2), vals):
        A = W.make_problem(dataclasses.replace(w, time=float(step))).A
        want, _ = seqmod.values_in_setup_order(A, st)
        assert np.array_equal(v, want)
    # the right-hand sides are the reference's randomRhs of (step, corrector), in the setup's order
    solves = [e for e in log if e[0] == "gmres"]
    for k, r in enumerate(recs):
        assert (r.step, r.corrector) == (k, 0)
        assert np.array_equal(solves[k][5], random_rhs_step(st.n, w.seed, k, 0)[st.new_to_old])


def test_time_loop_warm_start_and_final_tolerances():
    w = small_bubbles()
    recs, log = run(w, steps=2, correctors=3, reuse="refactor", warm_start=True, final_rtol=1e-6, final_atol=1e-12)
    solves = [e for e in log if e[0] == "gmres"]
    assert not np.any(solves[0][1])                 # the first solve starts from 0
    assert all(np.any(s[1]) for s in solves[1:])    # the next ones from the previous solution
    assert [s[2] for s in solves] == [w.rtol, w.rtol, 1e-6] * 2
    assert [s[3] for s in solves] == [0.0, 0.0, 1e-12] * 2
    assert [r.final_corrector for r in recs] == [False, False, True] * 2


def test_time_loop_rejects_bad_options():
    w = small_bubbles()
    for kw in ({"correctors": 0}, {"reuse": "never"}, {"rebuild_growth": -1.0}, {"rebuild_every": -2},
               {"stop_norm": "linf"}, {"steps": 0}):
        with pytest.raises(ValueError):
            run_time_loop(w, TimeLoopConfig(**kw), make_solver=Recorder, workers=1)


@pytest.mark.parametrize("reuse", [False, True])
def test_time_loop_amg_refactorizes_on_the_host(reuse):
    """AMG local solvers: Refactorize sets the hierarchies up again on the host (new, or with the
    transfer operators kept under amg_reuse) with the coarse basis kept, and uploads a new setup."""
    w = small_bubbles()
    w.opts.local_approx = "amg"
    w.opts.amg_coarse_enough = 100
    w.opts.amg_reuse = reuse
    recs, log = run(w, steps=3, correctors=2, reuse="refactor")
    assert levels(recs) == "201010"
    builds = [e[1] for e in log if e[0] == "build"]
    assert len(builds) == 3 and not any(e[0] == "refactor" for e in log)
    assert [e[0] for e in log].count("close") == 3
    st0, st1 = builds[0], builds[1]
    assert st1.subdomains[0].V is st0.subdomains[0].V                 # the coarse basis is kept
    same = [a.P is b.P for a, b in zip(st0.subdomains[0].amg.levels, st1.subdomains[0].amg.levels)]
    assert all(same) if reuse else not any(same)
    import dataclasses
    A1 = W.make_problem(dataclasses.replace(w, time=1.0)).A
    want, _ = seqmod.values_in_setup_order(A1, st0)
    assert np.array_equal(st1.A.data, want)


def test_time_loop_from_matrix_market_files_matches_the_generator(tmp_path):
    """The reference's --matrix p_%02d.mtx sequence (test/test_reuse.cpp:446-471): the same
    sequence read from Matrix Market files gives the same setups and refactorizations."""
    import dataclasses
    import scipy.io
    w = small_bubbles()
    for s in range(3):
        scipy.io.mmwrite(str(tmp_path / f"p_{s:02d}.mtx"), W.make_problem(dataclasses.replace(w, time=float(s))).A)
    gen, log_gen = run(w, steps=3, correctors=1, reuse="refactor")
    Recorder.log = []
    files = run_time_loop(w, TimeLoopConfig(steps=3, correctors=1, reuse="refactor"), make_solver=Recorder, workers=1,
                          matrix=lambda s: seqmod.read_mtx(str(tmp_path / f"p_{s:02d}.mtx")))
    log_files = list(Recorder.log)
    assert levels(files) == levels(gen) == "211"
    ref_gen = [e[1] for e in log_gen if e[0] == "refactor"]
    ref_files = [e[1] for e in log_files if e[0] == "refactor"]
    assert len(ref_gen) == len(ref_files) == 2
    for a, b in zip(ref_gen, ref_files):
        assert np.array_equal(a, b)


def test_time_loop_summary_counts_levels_after_the_initial_setup():
    from s2l_b200.time_loop import summary
    w = small_bubbles()
    recs, _ = run(w, steps=3, correctors=2, reuse="refactor")
    s = summary(recs)
    assert s["solves"] == 6 and s["converged"] == 6
    assert (s["reuse"], s["refactorize"], s["rebuild"]) == (3, 2, 0)
    assert s["initial_setup_s"] == recs[0].t_update and s["iterations_max"] == 10
    assert abs(s["total_s"] - (s["initial_setup_s"] + s["updates_s"] + s["solves_s"])) < 1e-12
    assert s["last_corrector"]["iterations_mean"] == 10.0 and summary([]) == {}


def test_command_line_maps_the_reference_flags():
    from s2l_b200.time_loop import parse_args
    w, cfg, dev = parse_args(["--workload", "poisson2d", "--nx", "40", "--nsub", "4", "--steps", "5", "--correctors",
                              "2", "--reuse", "refactor", "--rebuild-every", "3", "--warm-start", "--final-rtol",
                              "1e-6", "--stop-norm", "openfoam", "--atol", "1e-12", "--local-approx", "amg",
                              "--amg-coarsening", "rs", "--amg-reuse", "1"])
    assert (w.name, w.nx, w.nsub) == ("poisson2d", 40, 4)
    assert (cfg.steps, cfg.correctors, cfg.reuse, cfg.rebuild_every, cfg.warm_start) == (5, 2, "refactor", 3, True)
    assert cfg.final_rtol == 1e-6 and cfg.final_atol is None and cfg.stop_norm == "openfoam" and cfg.atol == 1e-12
    assert w.opts.local_approx == "amg" and w.opts.amg_coarsening == "rs" and w.opts.amg_reuse and dev == 0
    with pytest.raises(ValueError):
        parse_args(["--correctors", "0"])
    w, _, _ = parse_args(["--workload", "reference_coupled2d", "--nx", "16", "--ncomp", "2", "--pulse", "0.5"])
    assert w.kind == "reference_coupled2d" and w.extra == {"nu": 1.0, "ncomp": 2, "pulse": 0.5, "pulse_period": 20}


def test_time_loop_on_the_reference_pulsating_convection():
    """The reference's own nonsymmetric sequence (convdiff2d, pulse 0.5, period 10, as its reuse
    test): every step refactorizes with new values on the same pattern."""
    w = W.reference_generator("reference_convdiff2d", nx=16, nsub=4, pulse=0.5, pulse_period=10)
    recs, log = run(w, steps=3, correctors=1, reuse="refactor")
    assert levels(recs) == "211"
    vals = [e[1] for e in log if e[0] == "refactor"]
    assert len(vals) == 2 and not np.array_equal(vals[0], vals[1])
