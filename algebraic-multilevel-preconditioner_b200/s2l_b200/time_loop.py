"""Sequences of solves with setup reuse: the reference's time loop and reuse policy on the device.

The reference emulates the pressure equation of a PISO/PIMPLE loop (``runTimeLoop``,
``src/solver/time_loop.cpp:57-195``): every step has new matrix values on the same pattern, every
corrector of a step a new right-hand side; before each solve a ``ReusePolicy``
(``include/preconditioner/reuse_policy.hpp``, ``src/preconditioner/reuse_policy.cpp``) chooses the
``UpdateLevel`` and the preconditioner performs it.  Here the three levels map onto the device
setup:

* ``Reuse``: the setup is kept as it is (the policy only asks for it when the matrix did not change);
* ``Refactorize``: ``GpuSetup.refactor`` (``s2l_gpu_refactor``: the local factors refactorized on their
  kept patterns, E recomputed with the kept coarse basis, on the device); with AMG local solvers
  the hierarchies are set up again on the host (``setup_phase.refactor_amg_setup``, new or with
  kept transfer operators as ``--amg-reuse``) and the setup is uploaded anew;
* ``Rebuild``: a new host setup of the current matrix on the same partition, uploaded as a new
  device setup (the reference's full ``TwoLevelSchwarz`` construction).

``ReusePolicy`` restates the reference's decision arithmetic (iterations per decade, time wasted by
the aging coarse basis, the rebuild premium from lower medians of the measured times, the safety nets
on growth, age and non-convergence); its known answers are the reference's own
(``test/test_reuse.cpp:50-110``).  The right-hand side of solve (step, corrector) is the reference's
``randomRhs`` (``rng.random_rhs_step``).  With the C++ drop-in the reference's own time loop and
policy drive ``GpuTwoLevelSchwarz::update`` instead; this module is the stand-alone loop.
"""
from __future__ import annotations

import dataclasses
import enum
import math
import time
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from . import sequence as seqmod
from . import workloads as W
from .rng import random_rhs_step
from .setup_phase import build_setup, refactor_amg_setup


class UpdateLevel(enum.IntEnum):
    """``prec::UpdateLevel`` (``include/preconditioner/preconditioner.hpp:30``)."""
    REUSE = 0
    REFACTORIZE = 1
    REBUILD = 2


class ReusePolicy:
    """Chooses the update level before each solve of a sequence (``reuse_policy.hpp:63-132``).

    Modes ``off`` (rebuild before every solve), ``refactor`` (never rebuild after the first setup)
    and ``auto`` (reuse on an unchanged matrix, refactorize on a changed one, rebuild once the time
    lost to the aging coarse basis since the last rebuild reaches the extra cost of a rebuild over a
    refactorization, or when a safety net trips).
    """
    OFF, REFACTOR, AUTO = "off", "refactor", "auto"

    def __init__(self, mode: str, growth: float = 4.0, max_age: int = 0):
        self.mode = self.parse_mode(mode)
        self.growth = float(growth)
        self.max_age = int(max_age)
        self._ref: list[float] = []   # per kind: q of its first solve after the last rebuild (0: none yet)
        self.last = 0.0                # q of the last solve
        self._last_ref = 0.0           # q_ref of the kind of the last solve
        self.age = 0                   # refactorizations since the last rebuild
        self._converged = True
        self.wasted = 0.0              # seconds lost to the old basis since the last rebuild
        self._t_rebuild: list[float] = []
        self._t_refactor: list[float] = []

    @classmethod
    def parse_mode(cls, s: str) -> str:
        """``ReusePolicy::parseMode`` (``reuse_policy.cpp:13-19``); ValueError like its invalid_argument."""
        if s in (cls.OFF, cls.REFACTOR, cls.AUTO):
            return s
        raise ValueError(f"unknown reuse mode '{s}' (off|refactor|auto)")

    @staticmethod
    def per_decade(iterations: int, reduction: float) -> float:
        """Iterations per decade of residual reduction, 0 when undefined (``reuse_policy.cpp:21-25``)."""
        if iterations <= 0 or not (reduction > 0.0) or not (reduction < 1.0):
            return 0.0
        return iterations / math.log10(1.0 / reduction)

    @staticmethod
    def lower_median(v) -> float:
        """The element of rank floor((n - 1) / 2) in increasing order, 0 if empty (``reuse_policy.cpp:27-33``)."""
        if len(v) == 0:
            return 0.0
        return float(sorted(v)[(len(v) - 1) // 2])

    def rebuild_premium(self) -> float:
        """Extra cost of a rebuild over a refactorization from the lower medians of the measured
        times, 0 while unknown (``reuse_policy.cpp:35-39``)."""
        reb = self.lower_median(self._t_rebuild)
        return max(0.0, reb - self.lower_median(self._t_refactor)) if reb > 0.0 else 0.0

    def reference(self, kind: int = 0) -> float:
        return self._ref[kind] if 0 <= kind < len(self._ref) else 0.0

    def decide(self, matrix_changed: bool) -> UpdateLevel:
        """Level to perform before the next solve (``reuse_policy.cpp:41-52``)."""
        if self.mode == self.OFF:
            return UpdateLevel.REBUILD
        if not matrix_changed:
            return UpdateLevel.REUSE
        if self.mode == self.REFACTOR:
            return UpdateLevel.REFACTORIZE
        if not self._converged:
            return UpdateLevel.REBUILD
        if self.max_age > 0 and self.age + 1 > self.max_age:
            return UpdateLevel.REBUILD
        if self.growth > 0.0 and self._last_ref > 0.0 and self.last > self.growth * self._last_ref:
            return UpdateLevel.REBUILD
        premium = self.rebuild_premium()
        if premium > 0.0 and self.wasted >= premium:
            return UpdateLevel.REBUILD
        return UpdateLevel.REFACTORIZE

    def record(self, done: UpdateLevel, iterations: int, reduction: float, converged: bool, t_update: float,
               t_solve: float, kind: int = 0) -> None:
        """Outcome of a solve performed after level `done` (``reuse_policy.cpp:54-82``)."""
        if done == UpdateLevel.REBUILD:
            self.age = 0
            self._ref = [0.0] * len(self._ref)  # a rebuild invalidates the baseline of each level
            self._last_ref = 0.0
            self.wasted = 0.0
            if t_update > 0.0:
                self._t_rebuild.append(float(t_update))
        elif done == UpdateLevel.REFACTORIZE:
            self.age += 1
            if t_update > 0.0:
                self._t_refactor.append(float(t_update))
        self._converged = bool(converged)
        q = self.per_decade(iterations, reduction)
        if q <= 0.0:
            return
        self.last = q
        k = max(0, int(kind))
        if k >= len(self._ref):
            self._ref.extend([0.0] * (k + 1 - len(self._ref)))
        if self._ref[k] <= 0.0:  # first solve of this kind on a fresh basis: the reference, nothing wasted
            self._ref[k] = q
            self._last_ref = q
            return
        self._last_ref = self._ref[k]
        excess = iterations - self._ref[k] * math.log10(1.0 / reduction)
        if excess > 0.0:
            self.wasted += excess * t_solve / iterations


@dataclass
class TimeLoopConfig:
    """The reference's sequence options (``include/core/config.hpp:40-49``, ``--maxit`` and the stopping
    test of ``config.hpp:84-92``); the Krylov method, restart and rtol come from the workload."""
    steps: int = 1
    correctors: int = 3
    reuse: str = "auto"
    rebuild_growth: float = 4.0
    rebuild_every: int = 0
    warm_start: bool = False
    final_rtol: float | None = None   # last corrector of a step (p_rghFinal); None: the workload's rtol
    final_atol: float | None = None   # None: atol
    stop_norm: str = "l2"             # "l2" or "openfoam"
    atol: float = 0.0
    maxit: int = 1000

    def validate(self):
        """The reference's checks of these options (``src/core/config.cpp:240-247``)."""
        if self.steps < 1:
            raise ValueError("steps must be >= 1")
        if self.correctors < 1:
            raise ValueError("--correctors must be >= 1")
        ReusePolicy.parse_mode(self.reuse)
        if self.rebuild_growth < 0.0:
            raise ValueError("--rebuild-growth must be >= 0")
        if self.rebuild_every < 0:
            raise ValueError("--rebuild-every must be >= 0")
        if self.stop_norm not in ("l2", "openfoam"):
            raise ValueError("--stop-norm must be l2|openfoam")


@dataclass
class SolveRecord:
    """``solv::SolveRecord`` (``include/solver/time_loop.hpp:20-36``)."""
    step: int
    corrector: int
    level: UpdateLevel
    t_update: float
    t_solve: float
    iterations: int
    per_decade: float
    converged: bool
    true_rel_residual: float
    n0: int
    wasted: float
    initial_res_of: float
    final_res_of: float
    final_corrector: bool


def levels(records) -> str:
    """The levels of a sequence as digits, e.g. "201010" (the reference's test notation)."""
    return "".join(str(int(r.level)) for r in records)


def _device_solver(ctx, options):
    from . import capi

    def make(st, refactor):
        opts = dict(options or {})
        if refactor:
            opts["refactor"] = 1
        return capi.GpuSetup(ctx, st, options=opts)
    return make


def run_time_loop(w: "W.Workload", cfg: TimeLoopConfig, ctx=None, matrix=None, rhs=None, make_solver=None,
                  options=None, part=None, symmetric=None, workers=None, out=None) -> list:
    """``cfg.steps`` steps of ``cfg.correctors`` solves of workload `w` (``time_loop.cpp:57-195``).

    matrix(step): the matrix of a step (CSR, original ordering; default: the workload's problem at
    time = step, the moving-bubble sequence for bubbles3d; Matrix Market files through
    ``sequence.read_mtx``).  rhs(step, corrector, n): the right-hand side in the original ordering
    (default: the reference's randomRhs with the workload's seed).  part, symmetric: the partition
    and the symmetry of the sequence (default: the workload's, from its problem at time 0).
    make_solver(setup, refactor): the device setup of a host setup (default: ``GpuSetup`` on `ctx`,
    with the option refactor when the policy may refactorize).  Returns one SolveRecord per solve.
    """
    cfg.validate()
    if make_solver is None:
        if ctx is None:
            raise ValueError("run_time_loop needs a device context (ctx) or make_solver")
        make_solver = _device_solver(ctx, options)
    mode = ReusePolicy.parse_mode(cfg.reuse)
    one_level = w.opts.coarse == "none"
    # a one-level preconditioner has no coarse basis to age: auto behaves as refactor
    if one_level and mode == ReusePolicy.AUTO:
        mode = ReusePolicy.REFACTOR
    policy = ReusePolicy(mode, cfg.rebuild_growth, cfg.rebuild_every)
    amg = w.opts.local_approx == "amg"
    # factors are refactorized on the device; AMG hierarchies on the host, then uploaded anew
    refactor = mode != ReusePolicy.OFF and not amg
    if matrix is None:
        def matrix(step):
            return W.make_problem(dataclasses.replace(w, time=float(step))).A
    if rhs is None:
        def rhs(step, corr, n):
            return random_rhs_step(n, w.seed, step, corr)
    final_tols = cfg.final_rtol is not None or cfg.final_atol is not None
    final_rtol = cfg.final_rtol if cfg.final_rtol is not None else w.rtol
    final_atol = cfg.final_atol if cfg.final_atol is not None else cfg.atol
    of_stop = cfg.stop_norm == "openfoam"
    # FP32 factors: converged only at the recomputed FP64 true residual, as the drop-in's solver
    strict = w.opts.local_precision == "single"

    if part is None or symmetric is None:
        prob0 = W.make_problem(dataclasses.replace(w, time=0.0))
        part = W.make_partition(w, prob0) if part is None else part
        symmetric = prob0.symmetric if symmetric is None else symmetric
    A_cur = matrix(0).tocsr()
    records = []
    g = st = None
    current = False  # the device setup holds the current matrix
    x = None
    try:
        for step in range(cfg.steps):
            if step > 0:
                A_cur = matrix(step).tocsr()
                current = False
            for corr in range(cfg.correctors):
                b_orig = np.asarray(rhs(step, corr, A_cur.shape[0]), dtype=np.float64)
                t0 = time.perf_counter()
                if g is None:
                    level = UpdateLevel.REBUILD
                else:
                    level = policy.decide(not current)
                if level == UpdateLevel.REBUILD:
                    st = build_setup(A_cur, b_orig, part, w.nsub, w.opts, symmetric, workers=workers)
                    st.stats["part"] = part
                    if g is not None:
                        g.close()
                        g = None
                    g = make_solver(st, refactor)
                elif level == UpdateLevel.REFACTORIZE:
                    vals, _ = seqmod.values_in_setup_order(A_cur, st)
                    if amg:
                        st = refactor_amg_setup(st, sp.csr_matrix((vals, st.A.indices, st.A.indptr),
                                                                  shape=st.A.shape))
                        g.close()
                        g = None
                        g = make_solver(st, False)
                    else:
                        g.refactor(vals)
                current = True
                t_update = time.perf_counter() - t0
                b = np.ascontiguousarray(b_orig[st.new_to_old])
                if not cfg.warm_start or x is None:
                    x = np.zeros(b.size)
                last = corr == cfg.correctors - 1
                rtol, atol = (final_rtol, final_atol) if (final_tols and last) else (w.rtol, cfg.atol)
                t0 = time.perf_counter()
                if w.krylov == "bicgstab":
                    x, res = g.bicgstab(b, x0=x, rtol=rtol, maxit=cfg.maxit, strict=strict, stop_norm=cfg.stop_norm,
                                        atol=atol)
                else:
                    x, res = g.gmres(b, x0=x, restart=w.restart, rtol=rtol, maxit=cfg.maxit, flexible=w.flexible,
                                     strict=strict, stop_norm=cfg.stop_norm, atol=atol)
                t_solve = time.perf_counter() - t0
                hist = res["history"]
                r0 = res["initial_residual_of"] if of_stop else (float(hist[0]) if len(hist) else 1.0)
                r1 = res["final_residual_of"] if of_stop else res["true_rel_residual"]
                reduction = r1 / r0 if r0 > 0.0 else 0.0
                policy.record(level, res["iterations"], reduction, res["converged"], t_update, t_solve,
                              corr if (cfg.warm_start or final_tols) else 0)
                rec = SolveRecord(step, corr, level, t_update, t_solve, int(res["iterations"]),
                                  ReusePolicy.per_decade(res["iterations"], reduction), bool(res["converged"]),
                                  float(res["true_rel_residual"]), int(st.stats.get("n0", 0)), policy.wasted,
                                  float(res["initial_residual_of"]), float(res["final_residual_of"]), last)
                records.append(rec)
                if out is not None:
                    out.write(f"{step:7d}{corr:5d}  {level.name.lower():<12}{t_update:10.4f}{t_solve:10.4f}"
                              f"{rec.iterations:5d}{rec.per_decade:11.2f}{rec.n0:8d}{rec.wasted:11.4f}"
                              f"{'' if rec.converged else '  NOT converged'}\n")
    finally:
        if g is not None:
            g.close()
    return records


def summary(records) -> dict:
    """Totals of a time loop (``printTimeLoopSummary``, ``src/solver/time_loop.cpp:197-240``): the
    initial setup, the updates per level after it (count and total time), the solves (time,
    iterations average and maximum, converged count), and for correctors that differ from the last
    one of a step (warm start, final tolerances) their iterations and times apart."""
    if not records:
        return {}
    count = {lv: 0 for lv in UpdateLevel}
    t_level = {lv: 0.0 for lv in UpdateLevel}
    for r in records[1:]:  # the first solve's update is the initial setup
        count[r.level] += 1
        t_level[r.level] += r.t_update
    its = [r.iterations for r in records]
    out = {
        "solves": len(records),
        "converged": sum(1 for r in records if r.converged),
        "initial_setup_s": records[0].t_update,
        "updates_s": sum(t_level.values()),
        "reuse": count[UpdateLevel.REUSE],
        "refactorize": count[UpdateLevel.REFACTORIZE],
        "refactorize_mean_s": t_level[UpdateLevel.REFACTORIZE] / max(count[UpdateLevel.REFACTORIZE], 1),
        "rebuild": count[UpdateLevel.REBUILD],
        "rebuild_mean_s": t_level[UpdateLevel.REBUILD] / max(count[UpdateLevel.REBUILD], 1),
        "solves_s": sum(r.t_solve for r in records),
        "iterations_mean": sum(its) / len(its),
        "iterations_max": max(its),
    }
    out["total_s"] = out["initial_setup_s"] + out["updates_s"] + out["solves_s"]
    for key, sel in (("correctors", [r for r in records if not r.final_corrector]),
                     ("last_corrector", [r for r in records if r.final_corrector])):
        out[key] = {"iterations_mean": sum(r.iterations for r in sel) / len(sel) if sel else 0.0,
                    "solves_s": sum(r.t_solve for r in sel)}
    return out


def parse_args(argv=None):
    """(workload, TimeLoopConfig, device) from the reference's sequence flags (``--steps``,
    ``--correctors``, ``--reuse``, ``--rebuild-growth``, ``--rebuild-every``, ``--warm-start``,
    ``--final-rtol``, ``--final-atol``, ``--stop-norm``, ``--atol``, ``--maxit``, ``--local-approx``,
    ``--amg-*``) and a named workload of this package at a chosen size."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m s2l_b200.time_loop",
                                 description="A sequence of solves with setup reuse on the GPU.")
    ap.add_argument("--workload", default="bubbles3d",
                    choices=["poisson2d", "bubbles3d", "convdiff3d", "reference_convdiff2d", "reference_convdiff3d",
                             "reference_coupled2d", "reference_coupled3d"],
                    help="reference_*: the reference's own --generate convdiff/coupled problems")
    ap.add_argument("--nu", type=float, default=1.0, help="reference_*: viscosity")
    ap.add_argument("--ncomp", type=int, default=4, help="reference_coupled*: unknowns per cell")
    ap.add_argument("--pulse", type=float, default=0.0, help="reference_*: amplitude of the convection pulsation")
    ap.add_argument("--pulse-period", type=int, default=20, help="reference_*: period of the pulsation [steps]")
    ap.add_argument("--nx", type=int, default=0, help="grid size (0: the workload's)")
    ap.add_argument("--nsub", type=int, default=0, help="subdomains (0: the workload's)")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--correctors", type=int, default=3)
    ap.add_argument("--reuse", default="auto", choices=["off", "refactor", "auto"])
    ap.add_argument("--rebuild-growth", type=float, default=4.0)
    ap.add_argument("--rebuild-every", type=int, default=0)
    ap.add_argument("--warm-start", action="store_true")
    ap.add_argument("--final-rtol", type=float, default=-1.0, help="< 0: rtol")
    ap.add_argument("--final-atol", type=float, default=-1.0, help="< 0: atol")
    ap.add_argument("--stop-norm", default="l2", choices=["l2", "openfoam"])
    ap.add_argument("--atol", type=float, default=0.0)
    ap.add_argument("--maxit", type=int, default=1000)
    ap.add_argument("--local-approx", default="none", choices=["none", "amg"])
    ap.add_argument("--amg-coarsening", default="sa", choices=["sa", "rs"])
    ap.add_argument("--amg-sweeps", type=int, default=1)
    ap.add_argument("--amg-coarse-enough", type=int, default=500)
    ap.add_argument("--amg-reuse", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.workload.startswith("reference_"):
        w = W.reference_generator(a.workload, nx=a.nx or 32, nsub=a.nsub or 8, nu=a.nu, ncomp=a.ncomp,
                                  pulse=a.pulse, pulse_period=a.pulse_period)
    elif a.workload == "poisson2d":
        w = W.poisson2d(a.nx or 200, a.nsub or 8)
    elif a.workload == "convdiff3d":
        w = W.convdiff3d(a.nx or 128, a.nsub or 128)
    else:
        w = W.bubbles3d(a.nx or 100, a.nsub or 64)
    w.opts.local_approx = a.local_approx
    w.opts.amg_coarsening = a.amg_coarsening
    w.opts.amg_sweeps = a.amg_sweeps
    w.opts.amg_coarse_enough = a.amg_coarse_enough
    w.opts.amg_reuse = bool(a.amg_reuse)
    if a.local_approx == "amg":
        w.opts.local_precision = "double"  # the device AMG is FP64
        w.flexible = False
    cfg = TimeLoopConfig(steps=a.steps, correctors=a.correctors, reuse=a.reuse, rebuild_growth=a.rebuild_growth,
                         rebuild_every=a.rebuild_every, warm_start=a.warm_start,
                         final_rtol=a.final_rtol if a.final_rtol >= 0.0 else None,
                         final_atol=a.final_atol if a.final_atol >= 0.0 else None, stop_norm=a.stop_norm,
                         atol=a.atol, maxit=a.maxit)
    cfg.validate()
    return w, cfg, a.device


def main(argv=None) -> int:
    """Runs the loop on the GPU and prints every solve and the totals, as the reference's
    ``--steps`` run does; exit status 0 when every solve converged, 2 otherwise."""
    import sys
    from . import capi
    w, cfg, device = parse_args(argv)
    ctx = capi.Context(device)
    try:
        sys.stdout.write(f"Time loop: {cfg.steps} steps x {cfg.correctors} correctors, reuse {cfg.reuse}, "
                         f"{w.name} {w.nx}, {w.nsub} subdomains\n"
                         "   step corr  level         update[s]  solve[s]  its  it/decade      n0  wasted[s]\n")
        recs = run_time_loop(w, cfg, ctx=ctx, out=sys.stdout)
    finally:
        ctx.close()
    s = summary(recs)
    sys.stdout.write(f"Time loop summary (reuse {cfg.reuse}, {s['solves']} solves, {s['converged']} converged)\n"
                     f"  initial setup              {s['initial_setup_s']:.3f} s\n"
                     f"  updates                    {s['updates_s']:.3f} s   (reuse {s['reuse']} x, refactorize "
                     f"{s['refactorize']} x {s['refactorize_mean_s']:.3f} s, rebuild {s['rebuild']} x "
                     f"{s['rebuild_mean_s']:.3f} s)\n"
                     f"  solves                     {s['solves_s']:.3f} s   (iterations avg {s['iterations_mean']:.1f}, "
                     f"max {s['iterations_max']})\n"
                     f"  total setup + updates + solves {s['total_s']:.3f} s\n")
    return 0 if s["converged"] == s["solves"] else 2


if __name__ == "__main__":
    raise SystemExit(main())
