#!/usr/bin/env python
"""Benchmark of the B200 solve phase: solves to a true FP64 residual of 1e-8.

Main workload: 3D 7-point variable-coefficient pressure Poisson 100^3 (n = 1.0M), beta = 1/rho with
rho = 1e-3 in 200 seeded spheres of radius 3-8 cells, 64 subdomains (recursive coordinate
bisection), deflated two-level RAS, nev 20, local L L^T, GMRES(50), rtol 1e-8, U[-1,1] right-hand
sides.  Overlap 1 by default: the reference's own overlap, so the reference arm (--impl reference)
runs this very matrix, partition, right-hand side and preconditioner.  Forms timed on it:
  plain_fp64  : FP64 factors, the reference's GMRES, one solve per step (the reference arm's
                configuration exactly: the same-config anchor);
  mixed       : the same factors stored in FP32 + flexible GMRES(50) in FP64, converged only when
                the recomputed FP64 true residual is <= rtol, one solve per step;
  block_mixed : the mixed form for k right-hand sides per step (s2l_gpu_gmres_block);
  serving     : continuous batching (s2l_gpu_serve_batching) of Poisson arrivals of solve requests
                on this matrix (p50/p99 latency, solves/s, error against the FP64 solution);
  amg_local_solves: AMG local solvers (--local-approx amg), plain FP64 GMRES.
Other configurations, as their own forms:
  c2_overlap2 : the same problem at overlap 2 (plain FP64, mixed, 16-right-hand-side block);
  sequence    : 32 matrices of the moving-bubble sequence (bubbles rise half a cell per step) on 64
                uneven subdomains (10k-25k rows), 16 right-hand sides per matrix, the update before
                each matrix (Refactorize on the device, or Rebuild) chosen by the reference's reuse
                policy (--reuse auto);
  c3_convdiff : 3D upwind convection-diffusion 128^3 (n = 2.1M), 128 subdomains, LU factors,
                FGMRES(40) (plain FP64, mixed FP32 factors, 16-right-hand-side block);
  serving_mix : 2000 Poisson arrivals at 50 req/s over 40 seeded cases of the three families;
  parity      : in the CPU-baseline leg, the drop-in check (oracle/_ref/dropin_check) on the main
                workload and at the c1 size: the reference's apply and GMRES against the GPU's on
                the same objects.
Headline (`value`): block_mixed at --head-k right-hand sides per step (default 16), solves/s with b
resident in HBM; `e2e` = the same through the C ABI with pinned host buffers (copies inside the
timed region).  cpu_baseline: the reference itself (oracle/_ref/s2l_ref) on the main workload.

--impl reference times the reference itself (built from its sources into oracle/_ref/ with an
in-process thread-rank MPI) on the host cores, same problem and partition.
With torchrun (N > 1) every rank solves its own replica (the solve phase has no cross-GPU step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "algebraic-multilevel-preconditioner_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "solve time to FP64 residual 1e-8 (mixed/batched vs plain FP64 GPU); p50/p99 latency"
POOL = None  # the run's setup worker processes (setup_phase.worker_pool), on one GPU
_T0 = time.time()


def budgeted(name: str, est_s: float, fn, left_s: float, budget_s: float):
    """fn() when its usual time est_s fits in what is left of the run's budget, else a "skipped"
    record; an exception in fn becomes an "error" record (reported in the line, not fatal to it)."""
    if left_s < est_s:
        log(f"{name} skipped: {left_s:.0f} s of the {budget_s:.0f} s budget left, it takes about {est_s} s")
        return {"skipped": f"time budget: {left_s:.0f} s of {budget_s:.0f} s left, the form takes about {est_s} s"}
    try:
        out = fn()
    except Exception as e:
        out = {"error": f"{type(e).__name__}: {str(e)[-300:]}"}
    log(f"{name} done")
    return out


def release_host_memory() -> None:
    """Give the heap pages freed by a form's host setup back to the system (glibc malloc_trim): the
    many tens-of-MB arrays of a large setup are freed into the heap, not unmapped."""
    try:
        import ctypes
        ctypes.CDLL("libc.so.6").malloc_trim(0)
    except Exception:
        pass


def log(msg: str) -> None:
    """Progress on stderr (the JSON line is the only stdout), with the host memory in use: this
    process (and its setup workers) and what the host has left."""
    mem = ""
    try:
        import psutil
        me = psutil.Process()
        kids = sum(c.memory_info().rss for c in me.children(recursive=True))
        mem = (f" [rss {me.memory_info().rss / 2**30:.1f} GB + workers {kids / 2**30:.1f} GB, "
               f"host free {psutil.virtual_memory().available / 2**30:.0f} GB]")
    except Exception:
        pass
    print(f"[bench {time.time() - _T0:7.1f} s] {msg}{mem}", file=sys.stderr, flush=True)
REF_BIN = os.path.join(REPO, "oracle", "_ref", "s2l_ref")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=100, help="main workload grid size")
    ap.add_argument("--nsub", type=int, default=64, help="main workload subdomains")
    ap.add_argument("--nbubbles", type=int, default=200)
    ap.add_argument("--overlap", type=int, default=1, help="main workload overlap (1: the reference's)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-threads", type=int, default=0, help="reference arm: host threads (0 = all)")
    ap.add_argument("--opt", action="append", default=[], help="device layout option key=value (s2l_gpu_setup_option)")
    ap.add_argument("--block", default="4,8,16", help="block form: right-hand sides per block GMRES (comma list)")
    ap.add_argument("--head-k", type=int, default=16, help="right-hand sides per step of the headline block form")
    ap.add_argument("--serve", type=int, default=400, help="serving form: requests on the main matrix (0 = off)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="serving form: mean arrivals per second")
    ap.add_argument("--overlap2", type=int, default=1, help="c2 at overlap 2 (0 = off)")
    ap.add_argument("--seq", type=int, default=32, help="sequence form: matrices of the moving-bubble sequence (0 = off)")
    ap.add_argument("--seq-reuse", default="auto", choices=["auto", "refactor"])
    ap.add_argument("--c3", type=int, default=128, help="convection-diffusion form: grid size (0 = off)")
    ap.add_argument("--c3-nsub", type=int, default=128)
    ap.add_argument("--amg", type=int, default=1, help="AMG form: AMG local solvers on the main matrix (0 = off)")
    ap.add_argument("--serve-mix", type=int, default=2000,
                    help="serving-mix form: requests over 40 cases, in a child process bounded by the budget (0 = off)")
    ap.add_argument("--serve-mix-rate", type=float, default=50.0)
    ap.add_argument("--serve-mix-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--budget-s", type=float, default=1500.0,
                    help="wall-clock budget of the run: the secondary configurations that no longer fit are skipped")
    ap.add_argument("--autotune", type=int, default=1,
                    help="tune the mixed setup's device layout (s2l_b200.autotune) before the timed forms (0 = off)")
    ap.add_argument("--parity", type=int, default=1,
                    help="the CPU-baseline leg also runs the drop-in parity check on the main workload and c1 (0 = off)")
    return ap.parse_args(argv)


# ------------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampled every 50 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
                power.append(float(p[3]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


def measured_traffic(algorithmic_bytes: float):
    """DRAM bytes of one block local solve from the committed ncu summary (measured on a smaller
    case of the same workload, scaled by its algorithmic bytes), or None."""
    path = os.path.join(REPO, "profiles", "local_solve_block_traffic.txt")
    try:
        vals = {}
        for line in open(path):
            if ":" in line and not line.startswith("#"):
                k, v = line.split(":", 1)
                vals[k.strip()] = v.strip()
        ratio = float(vals["traffic_over_algorithmic_bytes"])
        return ratio * algorithmic_bytes
    except (OSError, KeyError, ValueError):
        return None


def spmv_bytes(st, k: int = 1) -> float:
    """Algorithmic bytes of y = A x for k columns: the CSR once (FP64 values, int32 columns and row
    pointers), x read and y written per column."""
    n = st.n
    return st.A.nnz * 12 + (n + 1) * 4 + k * 16 * n


def gmres_solve_bytes(st, its_cols, restart: int, ls_bytes: float, ls_col_bytes: float) -> float:
    """Algorithmic bytes of one (block) right-preconditioned GMRES(restart) solve whose columns took
    its_cols iterations: per Arnoldi step, the preconditioner (local solve: factors once plus
    ls_col_bytes per column; coarse basis and E once, three vectors per column; the deflated
    form's product with A), the product with A, and CGS2 over the column's basis.  Restarts and
    the Hessenberg work are left out, so this is a lower bound of the traffic."""
    n, n0 = st.n, st.n0
    deflated = n0 > 0 and st.opts.coarse == "deflated"
    basis = sum(s.n_owned * s.V.shape[1] for s in st.subdomains) if n0 else 0
    fixed = (ls_bytes - ls_col_bytes) + spmv_bytes(st, 0) * (2 if deflated else 1)
    if n0:
        fixed += 2 * 8 * basis + 8 * n0 * n0
    total = 0.0
    for i in range(max(its_cols) if len(its_cols) else 0):
        k = sum(1 for t in its_cols if t > i)
        j = i % restart
        col = ls_col_bytes + 16 * n + 3 * 8 * n           # local solve, A x, apply's vector updates
        if n0:
            col += 3 * 8 * n                              # restriction read, prolongation read/write
        if deflated:
            col += 16 * n + 8 * n                         # r - A x0
        col += 2 * (2 * (j + 1) * 8 * n + 16 * n)        # CGS2: dots and update, twice
        total += fixed + k * col
    return total


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


class Replicas:
    """The ranks of a run on N GPUs: independent replicas of the solve phase, no data-path
    collective.  A gloo group carries the barriers around the timed regions and the max over ranks
    of the device-timed totals (RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* from the launcher)."""

    def __init__(self, timeout_s: float = 900.0):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self, sync=None):
        """sync() (the device), then every rank."""
        if sync is not None:
            sync()
        if self.dist is not None:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.dist is None:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def rank0_first(self, make):
        """make() on rank 0, then on the others (rank 0 fills a cache the others read)."""
        out = make() if self.rank == 0 else None
        self.barrier()
        return make() if self.rank != 0 else out

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


# the autotuner's search in the benchmark: a reduced set of candidates (every candidate is a device
# setup of the 100^3 workload), the first value of each option the default
TUNE_SEARCH = (("hop_us", (0.25, 0.1, 0.5)), ("chain_block", (8, 16)), ("sweep_group", (16, 32)),
               ("spmv_tpr", (0, 1)), ("sweep_prefetch", (8, 16, 24)))


def workload_desc(w, overlap) -> str:
    """The main workload, the same words in both arms' lines."""
    return (f"bubbles3d {w.nx}^3 pressure Poisson ({w.nbubbles} bubbles of radius 3-8 cells, density ratio "
            f"{w.rho_ratio:g}), {w.nsub} subdomains, overlap {overlap}, nev {w.opts.nev}, deflated RAS, "
            f"L L^T local factors, GMRES({w.restart}), rtol {w.rtol:g}, U[-1,1] right-hand side")


def main_workload(a):
    from s2l_b200 import workloads as W
    return W.bubbles3d(a.nx, a.nsub, nbubbles=a.nbubbles, overlap=a.overlap)


def rel_err(x, y) -> float:
    import numpy as np
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


# ------------------------------------------------------------------------------------ our arm
class Timer:
    """Device timing of a form: W warm-up steps, then K steps each bracketed by CUDA events on the
    launching stream, a barrier (device sync + every rank) around the timed steps, max over ranks."""

    def __init__(self, a, reps, stream):
        import torch
        self.a, self.reps, self.stream, self.torch = a, reps, stream, torch

    def barrier(self):
        self.reps.barrier(self.torch.cuda.synchronize)

    def run(self, step, steps=None, warmup=None, before=None, after=None):
        """step() -> anything; returns (per-step ms list, total ms max over ranks, last output)."""
        torch = self.torch
        steps = self.a.steps if steps is None else steps
        warmup = self.a.warmup if warmup is None else warmup
        out = None
        for _ in range(warmup):
            out = step()
        if before:
            before()
        self.barrier()
        per = []
        for _ in range(steps):
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(self.stream)
            out = step()
            e_ev.record(self.stream)
            e_ev.synchronize()
            per.append(s_ev.elapsed_time(e_ev))
        self.barrier()
        if after:
            after()
        return per, self.reps.max(sum(per)), out


def single_form(tm, g, b_dev, x_dev, kw, x_ref=None, prof=True):
    """One right-hand side per step (x from zero), with the library's kernel timers."""
    import numpy as np
    res_all = []

    def step():
        x_dev.zero_()
        _, res = g.gmres(b_dev.data_ptr(), device_out=x_dev.data_ptr(), **kw)
        res_all.append(res)
        return res

    g.profile(("local_solve", "spmv") if prof else ())
    per, tot, _ = tm.run(step, before=lambda: res_all.clear())
    ls_ms, ls_n = g.profile_get("local_solve")
    sp_ms, sp_n = g.profile_get("spmv")
    launches = g.launches()
    g.profile(())
    x = x_dev.cpu().numpy()
    out = {"ms_per_solve": tot / len(per), "per_solve_ms": per, "iterations": [r["iterations"] for r in res_all],
           "converged": all(r["converged"] for r in res_all),
           "true_rel_residual": max(r["true_rel_residual"] for r in res_all),
           "p50_ms": float(np.percentile(per, 50)), "p99_ms": float(np.percentile(per, 99)),
           "local_solve_ms_total": ls_ms, "local_solve_launches": ls_n, "spmv_ms_total": sp_ms,
           "spmv_calls": sp_n, "launches": launches, "local_solve_bytes": g.local_solve_bytes(),
           "local_solve_column_bytes": g.stat("local_solve_column_bytes")}
    if x_ref is not None:
        out["rel_error_vs_fp64"] = rel_err(x, x_ref)
    return out, x


def block_form(tm, g, Bk, Xk, k, kw, X_ref=None, prof=False, sampler=None):
    """k right-hand sides per step in one lockstep block GMRES."""
    import numpy as np
    res_k = []

    def step():
        Xk.zero_()
        _, r = g.gmres_block((Bk.data_ptr(), k), device_out=Xk.data_ptr(), **kw)
        res_k[:] = r
        return r

    if prof:
        g.profile(("local_solve", "spmv"))
    per, tot, _ = tm.run(step, before=(sampler.start if sampler else None))
    clocks = sampler.stop() if sampler else None
    prof_out = None
    if prof:
        prof_out = dict(ls=g.profile_get("local_solve"), sp=g.profile_get("spmv"), launches=g.launches())
        g.profile(())
    out = {"rhs": k, "ms_per_block": tot / len(per), "ms_per_solve": tot / len(per) / k,
           "solves_per_s": tm.reps.world * k * len(per) / (tot * 1e-3),
           "iterations": [r["iterations"] for r in res_k], "converged": all(r["converged"] for r in res_k),
           "true_rel_residual": max(r["true_rel_residual"] for r in res_k),
           "p50_block_ms": float(np.percentile(per, 50)), "p99_block_ms": float(np.percentile(per, 99))}
    if X_ref is not None:
        Xh = Xk.cpu().numpy()
        out["rel_error_vs_fp64"] = max(rel_err(Xh[j], X_ref[j]) for j in range(k))
    return out, per, clocks, prof_out


def fp64_solutions(g64, B, kw):
    """The plain FP64 solutions of the rows of B (host), the reference point of every error."""
    import numpy as np
    return np.stack([g64.gmres(B[j], **kw)[0] for j in range(B.shape[0])])


def serve_form(local, st, kw, n_req, rate, bpool, xpool, workers=8, options=None):
    """Poisson arrivals of solve requests on one matrix through the serving engine (continuous
    batching, native workers, the device layout `options`); latency = submitted -> solution ready
    (host clock)."""
    import numpy as np
    from s2l_b200.serving import Engine
    eng = Engine(local, hbm_budget=150 << 30, workers=workers)
    eng.setup("m", lambda: st, options=options)
    t = eng.submit("m", lambda: st, bpool[0], history_cap=0, **kw)  # setup resident, runner warm
    t.wait(600.0)
    t.free()
    rng = np.random.default_rng(2026)
    gaps = rng.exponential(1.0 / rate, n_req)
    tickets = []
    t0 = time.perf_counter()
    t_next = t0
    for i in range(n_req):
        t_next += gaps[i]
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        j = i % len(bpool)
        tickets.append((j, eng.submit("m", lambda: st, bpool[j], history_cap=0, **kw)))
    lat, run, its, err = [], [], [], 0.0
    ok = True
    for j, t in tickets:
        x, r, status = t.wait(600.0)
        ok = ok and status == 0 and r["converged"]
        info = t.info()
        lat.append(info["queue_ms"] + info["run_ms"])
        run.append(info["run_ms"])
        its.append(r["iterations"])
        err = max(err, rel_err(x, xpool[j]))
        t.free()
    t_end = time.perf_counter()
    eng.close()
    return {"requests": n_req, "rate_req_s": rate, "workers": workers, "batching": "continuous (automatic slots)",
            "all_converged": ok, "solves_per_s": n_req / (t_end - t0),
            "ms_per_solve": (t_end - t0) * 1e3 / n_req,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(np.max(lat)), "run_ms_mean": float(np.mean(run)),
            "iterations_mean": float(np.mean(its)), "iterations_max": int(np.max(its)),
            "rel_error_vs_fp64_max": err, "clock": "host (submit to solution ready)"}


def run_ours(a):
    reps = Replicas()
    rank, world, local = reps.rank, reps.world, reps.local
    if world > 1:  # rank 0 sets the main workload up, the other ranks load its pickled copy
        os.environ.setdefault("S2L_CACHE_DIR", os.path.join(REPO, "_cache"))
    import numpy as np
    from s2l_b200 import workloads as W
    from s2l_b200.setup_phase import with_factor_precision, worker_pool

    # one pool of setup worker processes for every host setup of the run (spawned before any CUDA call)
    global POOL
    POOL = worker_pool() if world == 1 else None
    wl = main_workload(a)
    wdesc = workload_desc(wl, a.overlap)
    t0 = time.time()
    st = reps.rank0_first(lambda: W.build(wl)) if world > 1 else W.build(wl, pool=POOL)
    setup_s = time.time() - t0
    log(f"main workload host setup {setup_s:.1f} s (n = {st.n})")
    # ---- device (no CUDA call before the setup's process pool is done)
    import torch
    from s2l_b200 import capi

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = capi.Context(local)
    st32 = with_factor_precision(st, "single")
    layout = {kv.split("=")[0]: float(kv.split("=")[1]) for kv in a.opt}
    tuning = None
    if a.autotune:
        # the mixed setup's layout chosen by timing candidates on the device (4-column blocks, the
        # width of the headline's blocks); the FP64 setup takes the same options
        from s2l_b200 import autotune
        g32, tuning = autotune.tune(ctx, st32, k=4, reps=3, base=layout, search=TUNE_SEARCH)
        layout = dict(layout, **tuning["chosen"])
    else:
        g32 = capi.GpuSetup(ctx, st32, options=layout)
    g64 = capi.GpuSetup(ctx, st, options=layout)
    log(f"device setups ready (layout {layout})")
    stream = torch.cuda.current_stream(dev)
    for g in (g64, g32):
        g.set_stream(stream.cuda_stream)
    tm = Timer(a, reps, stream)
    n = st.n
    kw64 = dict(restart=wl.restart, rtol=wl.rtol, flexible=False, strict=False)
    kw32 = dict(restart=wl.restart, rtol=wl.rtol, flexible=True, strict=True)
    peak, peak_src = measured_peaks()
    b_dev = torch.tensor(st.b, device=dev, dtype=torch.float64)
    x_dev = torch.zeros(n, device=dev, dtype=torch.float64)

    # ---- one right-hand side per step: plain FP64 (the reference arm's configuration) and mixed
    plain, x64 = single_form(tm, g64, b_dev, x_dev, kw64)
    plain["true_rel_residual_host_check"] = float(np.linalg.norm(st.b - st.A @ x64) / np.linalg.norm(st.b))
    mixed, xm = single_form(tm, g32, b_dev, x_dev, kw32, x_ref=x64)
    mixed["true_rel_residual_host_check"] = float(np.linalg.norm(st.b - st.A @ xm) / np.linalg.norm(st.b))

    log(f"plain {plain['ms_per_solve']:.2f} ms, mixed {mixed['ms_per_solve']:.2f} ms per solve")
    # ---- blocks of k right-hand sides (the first is the workload's b), errors against FP64
    kh = a.head_k
    rng = np.random.default_rng(4321)
    B_host = np.stack([st.b] + [rng.uniform(-1.0, 1.0, n) for _ in range(max(kh, 16) - 1)])
    X64 = fp64_solutions(g64, B_host, kw64)
    bw = int(g32.stat("block_width"))
    ks = [int(v) for v in str(a.block).split(",") if v.strip() and int(v) >= 1]
    for extra in (bw, kh):
        if extra not in ks:
            ks = [extra] + ks
    block, head, rf = {}, None, None
    for k in ks:
        Bk = torch.tensor(B_host[:k], device=dev)
        Xk = torch.zeros_like(Bk)
        sampler = ClockSampler(local) if k == kh else None
        out, per, clocks, prof = block_form(tm, g32, Bk, Xk, k, kw32, X_ref=X64[:k], prof=(k == bw), sampler=sampler)
        block[str(k)] = out
        if k == kh:
            head = dict(out, per_block_ms=per, clocks=clocks)
        if k == bw:
            rf = prof
        del Bk, Xk

    log(f"blocks done: head {head['ms_per_block']:.2f} ms per {kh}-column step")
    # ---- end to end through the C ABI with pinned host buffers (headline block form): each step
    # copies its k right-hand sides and initial guesses in and its k solutions out
    b_pin = torch.empty((kh, n), dtype=torch.float64, pin_memory=True)
    b_pin.numpy()[:] = B_host[:kh]
    x_pin = torch.zeros((kh, n), dtype=torch.float64, pin_memory=True)

    def e2e_step():
        x_pin.zero_()
        return g32.gmres_block(b_pin.numpy(), X0=x_pin.numpy(), history_cap=0, **kw32)

    e2e_per, e2e_total, _ = tm.run(e2e_step, warmup=1)
    e2e_err = max(rel_err(x_pin.numpy()[j], X64[j]) for j in range(kh))

    # ---- serving: continuous batching of Poisson arrivals on this matrix (mixed precision)
    serving = None
    if a.serve > 0:
        bpool = B_host[:16]
        serving = serve_form(local, st32, kw32, a.serve, a.serve_rate, bpool, X64[:16], options=layout)
        serving["speedup_vs_plain_fp64_per_solve"] = plain["ms_per_solve"] / serving["ms_per_solve"]

    log(f"serving done: {serving and round(serving['solves_per_s'], 1)} solves/s")
    # ---- AMG local solvers (the reference's --local-approx amg) on the same matrix and basis
    amg_form = amg_local_solves(a, tm, ctx, st, b_dev, x_dev, stream, plain, x64, mixed) if a.amg else None

    # roofline of the headline's dominant kernel group: the block local solve (factors read once,
    # every column's gather and owned write), and of the single-column forms and the SpMV
    head_bytes = g32.local_solve_bytes() + (bw - 1) * g32.stat("local_solve_column_bytes")
    ls_avg_ms = rf["ls"][0] / max(rf["ls"][1], 1)
    traffic = measured_traffic(head_bytes)
    achieved = head_bytes / (ls_avg_ms * 1e-3) / 1e9 if ls_avg_ms > 0 else 0.0

    def rate(nbytes, ms):
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        return {"achieved": gbs, "frac": gbs / peak}

    def ls_rate(f):
        ms = f["local_solve_ms_total"] / max(f["local_solve_launches"], 1)
        return dict(rate(f["local_solve_bytes"], ms), avg_launch_ms=ms, bytes_per_launch=f["local_solve_bytes"])

    spmv = {"single_column_fp32": dict(rate(spmv_bytes(st), mixed["spmv_ms_total"] / max(mixed["spmv_calls"], 1)),
                                       bytes_per_launch=spmv_bytes(st), calls=mixed["spmv_calls"]),
            "single_column_fp64": dict(rate(spmv_bytes(st), plain["spmv_ms_total"] / max(plain["spmv_calls"], 1)),
                                       bytes_per_launch=spmv_bytes(st), calls=plain["spmv_calls"]),
            f"block_{bw}": dict(rate(spmv_bytes(st, bw), rf["sp"][0] / max(rf["sp"][1], 1)),
                                bytes_per_launch=spmv_bytes(st, bw), calls=rf["sp"][1])}
    col32 = mixed["local_solve_column_bytes"]
    hb = gmres_solve_bytes(st, head["iterations"], wl.restart, mixed["local_solve_bytes"], col32)
    mb = gmres_solve_bytes(st, mixed["iterations"][:1], wl.restart, mixed["local_solve_bytes"], col32)
    pb = gmres_solve_bytes(st, plain["iterations"][:1], wl.restart, plain["local_solve_bytes"],
                           plain["local_solve_column_bytes"])
    per_solve = {"headline_block": dict(rate(hb, head["ms_per_block"]), bytes=hb),
                 "mixed": dict(rate(mb, mixed["ms_per_solve"]), bytes=mb),
                 "plain_fp64": dict(rate(pb, plain["ms_per_solve"]), bytes=pb)}
    layout_stats = {"options": layout, "tail_rows": g64.stat("tail_rows"), "sparse_nnz": g64.stat("sparse_nnz"),
                    "coupling_nnz": g64.stat("coupling_nnz"), "dense_entries": g64.stat("dense_entries"),
                    "sweep_group": g64.stat("sweep_group"), "levels_max": g64.stat("levels_max"),
                    "chain_blocks": g64.stat("chain_blocks"), "sweep_tasks": g64.stat("sweep_tasks"),
                    "sweep_padding": g64.stat("sweep_padding"), "kc_max_fp32": g32.stat("kc_max"),
                    "levels_mean": round(g64.stat("levels_mean"), 1), "block_width": bw}
    g64.close()
    g32.close()
    main_info = {"n": st.n, "nnz": int(st.A.nnz), "n0": st.n0, "nnz_factors": st.stats.get("nnz_factors")}
    mixed_ls_gb = mixed["local_solve_bytes"] / 1e9
    # the host copies of the main workload are not needed any more (the other forms hold their own)
    del b_dev, x_dev, st, st32, B_host, X64, b_pin, x_pin

    # ---- the other configurations (each builds, times and frees its own setups)
    # (on one GPU: with replicas the line reports the headline form only)
    log("main workload done")
    one = world == 1
    import gc
    gc.collect()
    torch.cuda.empty_cache()
    release_host_memory()
    # the reference's own run (the line's cpu_baseline and parity) before the other configurations
    cb = parity = None
    if rank == 0 and one and not a.no_cpu_baseline and a.overlap == 1:
        try:
            cb, parity = cpu_baseline_leg(a, wl)
        except Exception as e:  # reported, not fatal to the line
            parity = {"error": str(e)[-300:]}
        log("cpu baseline and parity done")
    # the other configurations, in order of the configurations they stand for, while the run's time
    # budget allows (each form is skipped, not cut, when its usual time no longer fits): 3 warm-up
    # and at most 5 timed steps per form (their setups, not their solves, take the time)
    tm = Timer(argparse.Namespace(**dict(vars(a), steps=min(a.steps, 5), warmup=3)), reps, stream)

    def form(name, on, est_s, fn):
        if not (one and on):
            return None
        out = budgeted(name, est_s, fn, a.budget_s - (time.time() - _T0), a.budget_s)
        gc.collect()
        torch.cuda.empty_cache()
        release_host_memory()
        return out

    c3 = form("c3", a.c3 > 0, 300, lambda: c3_form(a, tm, ctx, stream, dev))
    sequence = form("sequence", a.seq > 0, 330, lambda: sequence_form(a, tm, ctx, stream, dev))
    c2_overlap2 = form("c2 overlap 2", a.overlap2 and a.overlap != 2, 90,
                       lambda: c2_overlap2_form(a, tm, ctx, stream, dev))
    if POOL is not None:
        POOL.shutdown()
    serving_mix = form("serving mix", a.serve_mix > 0, 240, lambda: serve_mix_child(a, local))

    out = {
        "metric": METRIC,
        # whole-job throughput of the headline form: blocks of k right-hand sides, mixed precision
        "value": world * kh * a.steps / (head["ms_per_block"] * a.steps * 1e-3),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": head["ms_per_block"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (FP32 local factors, FP64 Krylov/coarse/true residual)",
        "data": "synthetic (seeded generator, U[-1,1] right-hand sides)",
        "config": {
            "workload": wdesc,
            "form": f"block GMRES, {kh} right-hand sides per step, FP32 local factors, flexible GMRES in FP64, "
                    "converged at FP64 true residual <= rtol",
            "rhs_per_step": kh,
            **main_info,
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU, all subdomains resident",
            "l2": "inputs larger than L2 (local factors %.1f GB per form)" % mixed_ls_gb,
            "setup_s": round(setup_s, 1),
            "layout": layout_stats,
            "autotune": tuning,
        },
        "forms": {
            "block_mixed": block,
            "mixed": {k: mixed[k] for k in ("ms_per_solve", "iterations", "converged", "true_rel_residual",
                                             "true_rel_residual_host_check", "p50_ms", "p99_ms",
                                             "rel_error_vs_fp64")},
            "plain_fp64": dict({k: plain[k] for k in ("ms_per_solve", "iterations", "converged", "true_rel_residual",
                                                      "true_rel_residual_host_check", "p50_ms", "p99_ms")},
                               note="the reference arm's configuration: same matrix, partition, right-hand "
                                    "side, overlap, FP64 L L^T factors, GMRES(50), one right-hand side per solve"),
            "serving": serving,
            "amg_local_solves": amg_form,
            "c2_overlap2": c2_overlap2,
            "sequence": sequence,
            "c3_convdiff": c3,
            "serving_mix": serving_mix,
            "speedup_head_vs_plain_per_solve": plain["ms_per_solve"] / head["ms_per_solve"],
            "speedup_mixed_vs_plain": plain["ms_per_solve"] / mixed["ms_per_solve"],
            "iteration_delta_mixed_vs_plain": mixed["iterations"][0] - plain["iterations"][0],
            "iteration_delta_head_vs_plain": max(head["iterations"]) - plain["iterations"][0],
            "rel_error_head_vs_fp64": head.get("rel_error_vs_fp64"),
        },
        "p50_ms": head["p50_block_ms"],
        "p99_ms": head["p99_block_ms"],
        "e2e": {"value": world * kh * len(e2e_per) / (e2e_total * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": 2 * 8 * n * kh, "d2h_bytes_per_step": 8 * n * kh,
                "ms_per_step": e2e_total / len(e2e_per), "rel_error_vs_fp64": e2e_err},
        "roofline": {"bound": "hbm",
                     "kernel": f"local solve of one {bw}-column block (sweeps, tail coupling, dense tails); the "
                               f"{kh}-column step runs {max(kh // bw, 1)} such blocks at once",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "bytes_per_launch": head_bytes, "avg_launch_ms": ls_avg_ms,
                     "single_column_fp32": ls_rate(mixed), "single_column_fp64": ls_rate(plain),
                     "spmv": spmv, "per_solve": per_solve},
        # kernels launched in the timed region: those of the timed k=bw blocks, times the blocks
        # a k=head step runs at once
        "gpu_launches": int(rf["launches"] * max(kh // bw, 1)),
        "clocks": head["clocks"],
    }
    if cb is not None:
        out["cpu_baseline"] = cb
        out["forms"]["plain_fp64"]["speedup_vs_reference_same_config"] = cb["ms_per_solve"] / plain["ms_per_solve"]
        out["forms"]["speedup_head_vs_reference_per_solve"] = cb["ms_per_solve"] / head["ms_per_solve"]
    if parity is not None and a.parity:
        out["parity"] = parity
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    reps.close()


def amg_local_solves(a, tm, ctx, st, b_dev, x_dev, stream, plain, x64, mixed=None):
    """The same matrix, partition and coarse basis with each A_ii^-1 replaced by one AMG V-cycle:
    FP64 (the hierarchy and the V-cycle in double, the reference's GMRES) and FP32 (the reference's
    --local-precision single: the hierarchy built in float, the V-cycle in float, flexible GMRES in
    FP64 converged at the FP64 true residual)."""
    import copy
    import dataclasses
    import numpy as np
    from s2l_b200 import capi
    from s2l_b200.amg import build_hierarchy_native as build_hierarchy
    out = {}
    for prec in ("double", "single"):
        t0 = time.time()
        subs = [dataclasses.replace(sd, factor=None, amg=build_hierarchy(sd.Aii, single=prec == "single"))
                for sd in st.subdomains]
        st_amg = dataclasses.replace(st, subdomains=subs, opts=copy.copy(st.opts))
        st_amg.opts.local_approx = "amg"
        st_amg.opts.local_precision = prec
        host_s = time.time() - t0
        ga = capi.GpuSetup(ctx, st_amg)
        ga.set_stream(stream.cuda_stream)
        flex = prec == "single"
        kw = dict(restart=50, rtol=1e-8, flexible=flex, strict=flex, maxit=2000)
        f, xa = single_form(tm, ga, b_dev, x_dev, kw, x_ref=x64)
        ga.close()
        levels = sorted({len(sd.amg.levels) + (sd.amg.coarse is not None) for sd in subs})
        out["fp64" if prec == "double" else "fp32"] = {
            "ms_per_solve": f["ms_per_solve"], "iterations": f["iterations"], "converged": f["converged"],
            "true_rel_residual_host_check": float(np.linalg.norm(st.b - st.A @ xa) / np.linalg.norm(st.b)),
            "rel_error_vs_fp64": f["rel_error_vs_fp64"],
            "v_cycle_ms": f["local_solve_ms_total"] / max(f["local_solve_launches"], 1), "levels": levels,
            "operator_entries": int(sum(sd.amg.nnz() for sd in subs)), "host_setup_s": host_s}
    out["vs_exact_factors"] = {"plain_fp64_ms_per_solve": plain["ms_per_solve"], "plain_fp64_iterations": plain["iterations"],
                               "mixed_fp32_ms_per_solve": mixed["ms_per_solve"] if mixed else None}
    return out


def three_forms(tm, ctx, st, w, stream, dev, k=16):
    """Plain FP64, mixed (FP32 factors, flexible FP64 GMRES) and a k-right-hand-side mixed block on a
    host setup; errors against the plain FP64 solutions."""
    import numpy as np
    import torch
    from s2l_b200 import capi
    from s2l_b200.setup_phase import with_factor_precision
    st32 = with_factor_precision(st, "single")
    st64 = with_factor_precision(st, "double")
    g64, g32 = capi.GpuSetup(ctx, st64), capi.GpuSetup(ctx, st32)
    for g in (g64, g32):
        g.set_stream(stream.cuda_stream)
    kw64 = dict(restart=w.restart, rtol=w.rtol, flexible=False, strict=False)
    kw32 = dict(restart=w.restart, rtol=w.rtol, flexible=True, strict=True)
    b_dev = torch.tensor(st.b, device=dev, dtype=torch.float64)
    x_dev = torch.zeros(st.n, device=dev, dtype=torch.float64)
    plain, x64 = single_form(tm, g64, b_dev, x_dev, kw64, prof=False)
    mixed, _ = single_form(tm, g32, b_dev, x_dev, kw32, x_ref=x64, prof=False)
    rng = np.random.default_rng(99)
    B = np.stack([st.b] + [rng.uniform(-1.0, 1.0, st.n) for _ in range(k - 1)])
    X64 = fp64_solutions(g64, B, kw64)
    Bk = torch.tensor(B, device=dev)
    Xk = torch.zeros_like(Bk)
    blk, _, _, _ = block_form(tm, g32, Bk, Xk, k, kw32, X_ref=X64)
    keep = ("ms_per_solve", "iterations", "converged", "true_rel_residual", "p50_ms", "p99_ms")
    out = {"plain_fp64": {q: plain[q] for q in keep},
           "mixed": dict({q: mixed[q] for q in keep}, rel_error_vs_fp64=mixed["rel_error_vs_fp64"]),
           f"block_mixed_{k}": blk,
           "speedup_mixed_vs_plain": plain["ms_per_solve"] / mixed["ms_per_solve"],
           f"speedup_block_{k}_vs_plain_per_solve": plain["ms_per_solve"] / blk["ms_per_solve"],
           "n": st.n, "n0": st.n0, "nnz_factors": st.stats.get("nnz_factors"),
           "local_solve_gb_fp32": g32.local_solve_bytes() / 1e9}
    g64.close()
    g32.close()
    return out


def c2_overlap2_form(a, tm, ctx, stream, dev):
    """The main problem at overlap 2 (the configuration as stated; the reference has overlap 1 only)."""
    from s2l_b200 import workloads as W
    w = W.bubbles3d(a.nx, a.nsub, nbubbles=a.nbubbles, overlap=2)
    t0 = time.time()
    st = W.build(w, pool=POOL)
    setup_s = time.time() - t0
    log(f"c2 overlap 2 host setup {setup_s:.1f} s")
    out = three_forms(tm, ctx, st, w, stream, dev, k=a.head_k)
    out.update(workload=workload_desc(w, 2), setup_s=round(setup_s, 1))
    return out


def c3_form(a, tm, ctx, stream, dev):
    """3D upwind convection-diffusion 128^3 (4-mode divergence-free Fourier field, cell Peclet
    0.1-10), 128 subdomains, overlap 1, nev 24, deflated RAS, LU factors, FGMRES(40)."""
    from s2l_b200 import workloads as W
    w = W.convdiff3d(a.c3, a.c3_nsub, precision="double")
    t0 = time.time()
    st = W.build(w, pool=POOL)
    setup_s = time.time() - t0
    log(f"c3 host setup {setup_s:.1f} s (n = {st.n})")
    out = three_forms(tm, ctx, st, w, stream, dev, k=a.head_k)
    out.update(workload=f"convdiff3d {w.nx}^3 upwind convection-diffusion, {w.nsub} subdomains, overlap 1, nev 24, "
                        f"deflated RAS, LU factors, FGMRES({w.restart}), rtol 1e-8",
               setup_s=round(setup_s, 1))
    return out


def sequence_form(a, tm, ctx, stream, dev):
    """The moving-bubble sequence: a.seq matrices on one pattern (bubbles rise half a cell per step),
    64 uneven subdomains (10k-25k rows), 16 right-hand sides per matrix solved as one block.  Before
    each matrix the reference's reuse policy (time_loop.ReusePolicy, --reuse auto or refactor)
    chooses the update: Refactorize (s2l_gpu_refactor on the device: new local factors on the kept
    patterns, E with the kept basis) or Rebuild (a new host setup, uploaded).  A step is timed from
    the update to the 16 solutions."""
    import dataclasses
    import numpy as np
    import scipy.sparse as sp
    import torch
    from s2l_b200 import capi, workloads as W
    from s2l_b200 import sequence as seqmod
    from s2l_b200.setup_phase import build_setup, with_factor_precision
    from s2l_b200.time_loop import ReusePolicy, UpdateLevel
    w = W.bubbles3d(a.nx, a.nsub, nbubbles=a.nbubbles, overlap=a.overlap, precision="single")
    w.imbalance = 0.15
    prob0 = W.make_problem(w)
    part = W.make_partition(w, prob0)
    sizes = np.bincount(part, minlength=w.nsub)
    k = a.head_k
    kw = dict(restart=w.restart, rtol=w.rtol, flexible=True, strict=True, history_cap=0)
    rng = np.random.default_rng(77)
    B = rng.uniform(-1.0, 1.0, (k, prob0.n))  # original ordering; renumbered per setup
    policy = ReusePolicy(a.seq_reuse)
    g = st = None
    steps = []
    Bq = Xq = None
    try:
        for step in range(a.seq):
            A = prob0.A if step == 0 else W.make_problem(dataclasses.replace(w, time=float(step))).A
            level = UpdateLevel.REBUILD if g is None else policy.decide(True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            host_ms = None
            if level == UpdateLevel.REBUILD:
                st = with_factor_precision(build_setup(A, B[0], part, w.nsub, w.opts, prob0.symmetric, pool=POOL),
                                           "single")
                host_ms = (time.perf_counter() - t0) * 1e3
                st.stats["part"] = part  # the renumbering of later matrices' values (sequence.values_in_setup_order)
                if g is not None:
                    g.close()
                g = capi.GpuSetup(ctx, st, options={"refactor": 1})
                g.set_stream(stream.cuda_stream)
                Bq = torch.tensor(B[:, st.new_to_old], device=dev)
                Xq = torch.zeros_like(Bq)
            else:
                vals, _ = seqmod.values_in_setup_order(A, st)
                g.refactor(vals)
            torch.cuda.synchronize()
            t_update = time.perf_counter() - t0
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            Xq.zero_()
            _, rq = g.gmres_block((Bq.data_ptr(), k), device_out=Xq.data_ptr(), **kw)
            e_ev.record(stream)
            e_ev.synchronize()
            t_solve = s_ev.elapsed_time(e_ev) * 1e-3
            for j, r in enumerate(rq):  # one record per solve, as the reference's loop per corrector
                red = r["true_rel_residual"]
                policy.record(level if j == 0 else UpdateLevel.REUSE, r["iterations"], red, r["converged"],
                              t_update if j == 0 else 0.0, t_solve / k)
            Xh, Bh = Xq.cpu().numpy(), Bq.cpu().numpy()
            At = sp.csr_matrix((st.A.data if level == UpdateLevel.REBUILD else vals, st.A.indices, st.A.indptr),
                               shape=st.A.shape)
            chk = max(float(np.linalg.norm(Bh[j] - At @ Xh[j]) / np.linalg.norm(Bh[j])) for j in range(k))
            log(f"sequence step {step}: {level.name.lower()} {t_update * 1e3:.0f} ms"
                + (f" (host setup {host_ms:.0f} ms)" if host_ms else "") + f", solve {t_solve * 1e3:.0f} ms")
            steps.append({"step": step, "level": level.name.lower(), "update_ms": t_update * 1e3, "host_setup_ms": host_ms,
                          "solve_ms": t_solve * 1e3, "iterations_max": max(r["iterations"] for r in rq),
                          "converged": all(r["converged"] for r in rq), "true_rel_residual_host_check": chk})
    finally:
        if g is not None:
            g.close()
    tot = sum(q["update_ms"] + q["solve_ms"] for q in steps[1:])
    refac = [q["update_ms"] for q in steps if q["level"] == "refactorize"]
    return {"matrices": a.seq, "rhs_per_matrix": k, "reuse": a.seq_reuse,
            "levels": "".join(str(int(UpdateLevel[q["level"].upper()])) for q in steps),
            "subdomain_rows": [int(sizes.min()), int(sizes.max())],
            "rebuilds": sum(q["level"] == "rebuild" for q in steps),
            "refactor_ms_mean": float(np.mean(refac)) if refac else None,
            "solve_ms_mean": float(np.mean([q["solve_ms"] for q in steps])),
            "solves_per_s_after_first": (a.seq - 1) * k / (tot * 1e-3) if tot > 0 else None,
            "all_converged": all(q["converged"] for q in steps), "steps": steps}


def serve_mix_child(a, device: int) -> dict:
    """serve_mix in a child process (its own CUDA context and setup workers), bounded by what is
    left of the run's time budget: a child that fails or runs out of time costs the line this form
    only."""
    left = a.budget_s - (time.time() - _T0) - 30.0
    cmd = [sys.executable, os.path.abspath(__file__), "--serve-mix-only", "--serve-mix", str(a.serve_mix),
           "--serve-mix-rate", str(a.serve_mix_rate)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=max(left, 60.0),
                           env=dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(device))))
    except subprocess.TimeoutExpired as e:
        tail = (e.stderr or b"")[-400:]
        return {"error": f"did not finish within the {left:.0f} s left of the time budget", "stderr_tail":
                tail.decode(errors="replace") if isinstance(tail, bytes) else str(tail)}
    for line in r.stderr.splitlines()[-12:]:
        log("  " + line)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"child exited with {r.returncode}", "stderr_tail": r.stderr[-400:]}
    return json.loads(lines[-1])


def serve_mix(a, device: int) -> dict:
    """Poisson arrivals (a.serve_mix_rate per second) of a.serve_mix solve requests, each on one of
    40 seeded cases of the three workload families at several sizes (2D Poisson with LU factors,
    bubbles3d with L L^T factors, convdiff3d with FP32 LU factors and flexible GMRES), on an engine
    with a 150 GB HBM budget, 4 workers and continuous batching.  Every case is set up and
    resident before the first arrival; latency = request submitted -> solution ready (host clock)."""
    import numpy as np
    from s2l_b200 import workloads as W
    from s2l_b200.serving import Engine
    cases = []
    # 2D Poisson n = 1e4 - 4e6, bubbly pressure n = 1.4e4 - 1e6, convection-diffusion n = 1.4e4 - 1e6
    for nx, nsub in ((100, 8), (150, 8), (200, 8), (300, 8), (400, 16), (500, 16), (700, 16), (850, 32), (1000, 32),
                     (1200, 32), (1500, 64), (2000, 64)):
        cases.append(("poisson2d", W.poisson2d(nx, nsub)))
    for nx, nsub in ((24, 8), (28, 8), (32, 8), (32, 16), (36, 16), (40, 16), (40, 32), (44, 16), (48, 16), (48, 32),
                     (56, 32), (56, 64), (64, 32), (64, 64), (72, 64), (80, 64), (90, 64), (100, 64)):
        w = W.bubbles3d(nx, nsub, nbubbles=max(4, (nx * nx * nx) // 5000), overlap=1)
        cases.append(("bubbles3d", w))
    for nx, nsub in ((24, 8), (32, 8), (40, 16), (48, 16), (56, 32), (64, 32), (72, 64), (80, 64), (90, 64), (100, 128)):
        cases.append(("convdiff3d", W.convdiff3d(nx, nsub)))
    assert len(cases) == 40
    for q, (_, w) in enumerate(cases):
        w.seed = 1000 + q
    eng = Engine(device, hbm_budget=150 << 30, workers=4)
    kws, sizes = [], []
    setup_s = 0.0
    # each case set up on the host, uploaded (made resident by its first solve), then its host setup
    # dropped: only the device setups stay (a setup evicted under the budget would be built again)
    for q, (fam, w) in enumerate(cases):
        flex = w.opts.local_precision == "single"
        kws.append(dict(restart=w.restart, rtol=w.rtol, flexible=flex, strict=flex, history_cap=0))
        t0 = time.time()
        st = W.build(w, pool=POOL)
        setup_s += time.time() - t0
        sizes.append(st.n)
        t = eng.submit(q, (lambda st=st: st), st.b, **kws[q])  # the setup just built, uploaded
        t.wait(600.0)
        t.free()
        del st
        if q % 10 == 9:
            log(f"serving mix: {q + 1} cases set up ({setup_s:.1f} s of host setup)")
    log(f"serving mix: 40 host setups in {setup_s:.1f} s")
    makers = [(lambda w=w: W.build(w, pool=POOL)) for _, w in cases]
    rng = np.random.default_rng(2027)
    gaps = rng.exponential(1.0 / a.serve_mix_rate, a.serve_mix)
    picks = rng.integers(0, len(cases), a.serve_mix)
    pools = {}
    tickets = []
    t_start = time.perf_counter()
    t_next = t_start
    for i in range(a.serve_mix):
        t_next += gaps[i]
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        q = int(picks[i])
        if q not in pools:
            pools[q] = [rng.uniform(-1.0, 1.0, sizes[q]) for _ in range(4)]
        b_i = pools[q][i % 4]
        tickets.append((q, eng.submit(q, makers[q], b_i, **kws[q])))
    lat, fam_lat = [], {}
    ok = True
    for q, t in tickets:
        _, r, status = t.wait(600.0)
        ok = ok and status == 0 and r["converged"]
        info = t.info()
        ms = info["queue_ms"] + info["run_ms"]
        lat.append(ms)
        fam_lat.setdefault(cases[q][0], []).append(ms)
        t.free()
    t_end = time.perf_counter()
    out = {"requests": a.serve_mix, "rate_req_s": a.serve_mix_rate, "cases": len(cases),
           "sizes_n": [int(min(sizes)), int(max(sizes))],
           "hbm_budget_gb": 150, "all_converged": ok, "solves_per_s": a.serve_mix / (t_end - t_start),
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "max_ms": float(np.max(lat)), "setups_built": eng.builds, "evictions": eng.evictions,
           "batching": "continuous (automatic slots)",
           "per_family": {f: {"requests": len(v), "p50_ms": float(np.percentile(v, 50)),
                              "p99_ms": float(np.percentile(v, 99))} for f, v in fam_lat.items()},
           "host_setup_s": setup_s, "clock": "host (submit to solution ready)"}
    eng.close()
    return out


def reference_flags(wl) -> list:
    """The reference's command-line flags for the main workload's preconditioner and solver."""
    return ["--rhs", "random", "--seed", str(wl.seed), "--pou", "boolean", "--one-level", "ras", "--coarse", "deflated",
            "--nev", str(wl.opts.nev), "--local-solver", "sparselu", "--local-factorization", "cholesky",
            "--coarse-solver", "root", "--krylov", "gmres", "--restart", str(wl.restart), "--rtol", str(wl.rtol)]


def reference_case(wl):
    """The main workload's matrix and partition as the reference reads them (oracle.reference_runs)."""
    import numpy as np
    from oracle.reference_runs import MatrixCase
    from s2l_b200 import workloads as W
    prob = W.make_problem(wl)
    part = W.make_partition(wl, prob).astype(np.int32)
    return MatrixCase(prob.A, part, wl.nsub, reference_flags(wl))


def cpu_baseline_leg(a, wl) -> tuple:
    """Rank 0 at N = 1, after every timed region.  The reference itself (oracle/_ref, built from its
    sources) as the baseline and the checker:
      baseline: its bench mode on the main workload (the same matrix, partition, right-hand side and
                preconditioner as plain_fp64), one thread-rank per subdomain on the host's cores,
                2 timed solves after its setup (its own barrier-to-barrier solve timer);
      parity:   the drop-in check (oracle/_ref/dropin_check) on the main workload and at the c1 size:
                the reference's TwoLevelSchwarz::apply and GMRES against the GPU drop-in's on the same
                set-up objects (apply difference, iterations of both, GPU true residual).
    Returns (cpu_baseline dict or None, parity dict or None)."""
    from oracle import reference_runs as R
    if not os.path.exists(R.REF_BIN):
        return None, None
    threads = a.ref_threads or os.cpu_count() or 1
    case = reference_case(wl)
    try:
        rec = case.bench(steps=2, warmup=0)
        cb = None
        if rec is not None:
            ms = 1e3 * sum(rec["solve_s"]) / len(rec["solve_s"])
            cb = {"value": 1e3 / ms, "unit": "solves/s", "cores": threads, "kind": "reference", "ms_per_solve": ms,
                  "iterations": rec.get("iterations"), "setup_s": rec.get("setup_s"),
                  "sample": f"{len(rec['solve_s'])} full solves after the setup, {wl.nsub} thread-ranks on {threads} "
                            f"host threads ({wl.nsub / threads:.1f} thread-ranks per thread), same matrix, partition, "
                            f"right-hand side and preconditioner as plain_fp64"}
        parity = {}
        if os.path.exists(R.DROPIN_BIN):
            runs = [(f"main_{wl.nx}cube_{wl.nsub}sub_overlap1", case.dropin)]
            np1, args1 = R.FULL_SIZE["c1_laplace2d_200_8sub"]
            runs.append(("c1_laplace2d_200_8sub", lambda: R.dropin(np1, args1)))
            for name, fn in runs:
                t0 = time.time()
                try:
                    r = fn()
                    parity[name] = {"apply_rel": r["apply_rel_diff"], "its_ref": r["ref_iterations"],
                                    "its_gpu": r["gpu_iterations"], "gpu_true_rel_residual": r["gpu_true_rel_residual"],
                                    "x_rel_diff": r["x_rel_diff"], "ok": bool(r["ok"]),
                                    "wall_s": round(time.time() - t0, 1)}
                except Exception as e:  # reported in the line, not fatal to it
                    parity[name] = {"error": str(e)[-300:]}
        return cb, parity or None
    finally:
        case.close()


def run_reference(a):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/s2l_ref was not built "
                                                             "(the reference compiles only where its sources are)"}))
        return
    import numpy as np
    wl = main_workload(a)
    if a.overlap != 1:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's overlap is one layer"}))
        return
    threads = a.ref_threads or os.cpu_count() or 1
    case = reference_case(wl)
    try:
        rec = case.bench(a.steps, a.warmup)
    finally:
        case.close()
    if rec is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference run failed"}))
        return
    per = rec["solve_s"]
    ms = 1e3 * sum(per) / len(per)
    value = 1e3 / ms
    out = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "solves/s", "n_gpus": a.gpus,
        "steps": len(per), "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, U[-1,1] right-hand sides)",
        "config": {"workload": workload_desc(wl, 1),
                   "form": f"the reference's GMRES with its TwoLevelSchwarz (Eigen L L^T factors in FP64, root "
                           f"coarse solver), one right-hand side per solve, {wl.nsub} thread-ranks on {threads} host "
                           f"threads",
                   "n": int(wl.nx ** 3), "iterations": rec.get("iterations"), "setup_s": rec.get("setup_s"),
                   "true_rel_residual": rec.get("true_rel_residual")},
        "p50_ms": float(np.percentile(np.array(per) * 1e3, 50)), "p99_ms": float(np.percentile(np.array(per) * 1e3, 99)),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(per)} full solves, {wl.nsub} thread-ranks on {threads} host threads"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    args = parse()
    if args.serve_mix_only:  # the serving-mix form alone (run as a child of the bench)
        from s2l_b200.setup_phase import worker_pool
        POOL = worker_pool()
        print(json.dumps(serve_mix(args, 0)), flush=True)
        POOL.shutdown()
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
