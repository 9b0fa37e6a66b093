#!/usr/bin/env python
"""Benchmark of the B200 solve phase: solves to a true FP64 residual of 1e-8.

Workload (default): 3D 7-point variable-coefficient pressure Poisson 100^3 (n = 1.0M),
beta = 1/rho with rho = 1e-3 in 200 seeded spheres of radius 3-8 cells, 64 subdomains (recursive
coordinate bisection), overlap 2, nev 20, deflated two-level RAS, local L L^T, GMRES(50),
rtol 1e-8, U[-1,1] right-hand sides.  Forms timed:
  plain_fp64  : FP64 factors, the reference's GMRES (true-residual restart rule), one solve per step;
  mixed       : the same factors stored in FP32 + flexible GMRES(50) in FP64, converged only when
                the recomputed FP64 true residual is <= rtol, one solve per step;
  block_mixed : the mixed form for k right-hand sides per step (s2l_gpu_gmres_block);
  batched / block_mixed_threads: several solves or blocks from host threads at once;
  serving     : Poisson arrivals over three resident matrices on the worker threads (p50/p99);
  sequence_refactor: the next matrices of the moving-bubble sequence, each refactorized on the
                device (s2l_gpu_refactor) and solved for --head-k right-hand sides;
  amg_local_solves: the same matrix with AMG local solvers (--local-approx amg), plain FP64 GMRES.
Headline (`value`): block_mixed at --head-k right-hand sides per step (default 16, the batching
configuration's right-hand sides per matrix), solves/s with b resident in HBM; `e2e` = the same
through the C ABI with pinned host buffers (copies inside the timed region).

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


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bubbles3d", choices=["bubbles3d", "convdiff3d"],
                    help="bubbles3d: the headline configuration; convdiff3d: 128^3 convection-diffusion, "
                         "128 subdomains, LU factors, FGMRES(40)")
    ap.add_argument("--nx", type=int, default=0, help="grid size (0: the workload's)")
    ap.add_argument("--nsub", type=int, default=0, help="subdomains (0: the workload's)")
    ap.add_argument("--nbubbles", type=int, default=200)
    ap.add_argument("--overlap", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-threads", type=int, default=0, help="reference arm: host threads (0 = all)")
    ap.add_argument("--opt", action="append", default=[], help="device layout option key=value (s2l_gpu_setup_option)")
    ap.add_argument("--batch", default="2,4,8", help="batched form: right-hand sides solved at once (comma list)")
    ap.add_argument("--block", default="4,8,16", help="block form: right-hand sides per block GMRES (comma list)")
    ap.add_argument("--head-k", type=int, default=16, help="right-hand sides per step of the headline block form")
    ap.add_argument("--serve", type=int, default=120, help="serving form: requests (0 = off)")
    ap.add_argument("--seq", type=int, default=8, help="sequence form: matrices of the moving-bubble sequence (0 = off)")
    ap.add_argument("--serve-rate", type=float, default=50.0, help="serving form: mean arrivals per second")
    ap.add_argument("--amg", type=int, default=1,
                    help="AMG form: the same matrix with AMG local solvers (--local-approx amg), 0 = off")
    ap.add_argument("--serve-mix", type=int, default=0,
                    help="serving-mix form: requests over 40 seeded cases of the three families (0 = off)")
    ap.add_argument("--block-threads", default="2,4", help="block form with k=4 blocks from several host threads")
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


# ------------------------------------------------------------------------------------ our arm
def run_ours(a):
    reps = Replicas()
    rank, world, local = reps.rank, reps.world, reps.local
    os.environ.setdefault("S2L_CACHE_DIR", os.path.join(REPO, "_cache"))
    from s2l_b200 import workloads as W
    from s2l_b200.setup_phase import with_factor_precision

    if a.workload == "convdiff3d":
        wl = W.convdiff3d(a.nx or 128, a.nsub or 128, precision="double")
        a.seq = 0  # the moving-bubble sequence belongs to the bubbles workload
        wdesc = (f"convdiff3d {wl.nx}^3 upwind convection-diffusion (4-mode divergence-free Fourier field), "
                 f"{wl.nsub} subdomains, overlap 1, nev 24, deflated RAS, LU factors, FGMRES({wl.restart}), rtol 1e-8")
    else:
        wl = W.bubbles3d(a.nx or 100, a.nsub or 64, nbubbles=a.nbubbles, overlap=a.overlap)
        wdesc = (f"bubbles3d {wl.nx}^3 pressure Poisson, {wl.nsub} subdomains, overlap {a.overlap}, nev 20, "
                 f"deflated RAS, LL^T factors, GMRES({wl.restart}), rtol 1e-8")
    if world > 1:
        # rank 0 fills the setup cache first; the replicas then load it (setup is outside the timing)
        st = reps.rank0_first(lambda: W.build(wl))
    else:
        t0 = time.time()
        st = W.build(wl)
        setup_s = time.time() - t0
    # ---- device (no CUDA call before the setup's process pool is done)
    import numpy as np
    import torch
    from s2l_b200 import capi

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = capi.Context(local)
    st32 = with_factor_precision(st, "single")
    layout = {kv.split("=")[0]: float(kv.split("=")[1]) for kv in a.opt}
    g64 = capi.GpuSetup(ctx, st, options=layout)
    # the mixed setup keeps its factor patterns on the device for the sequence form's refactorizations
    g32 = capi.GpuSetup(ctx, st32, options=dict(layout, refactor=1) if a.seq > 0 else layout)
    stream = torch.cuda.current_stream(dev)
    for g in (g64, g32):
        g.set_stream(stream.cuda_stream)
    n = st.n
    b_dev = torch.tensor(st.b, device=dev, dtype=torch.float64)
    x_dev = torch.zeros(n, device=dev, dtype=torch.float64)
    forms = {
        "plain_fp64": (g64, dict(restart=wl.restart, rtol=wl.rtol, flexible=False, strict=False)),
        "mixed": (g32, dict(restart=wl.restart, rtol=wl.rtol, flexible=True, strict=True)),
    }

    def barrier():
        reps.barrier(torch.cuda.synchronize)

    max_over_ranks = reps.max

    results = {}
    peak, peak_src = measured_peaks()
    sampler = None
    for name, (g, kw) in forms.items():
        for _ in range(a.warmup):
            x_dev.zero_()
            g.gmres(b_dev.data_ptr(), device_out=x_dev.data_ptr(), **kw)
        headline = False
        g.profile(("local_solve", "spmv"))
        barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        its = []
        conv = []
        true_res = []
        for k in range(a.steps):
            ev[k][0].record(stream)
            x_dev.zero_()
            _, res = g.gmres(b_dev.data_ptr(), device_out=x_dev.data_ptr(), **kw)
            ev[k][1].record(stream)
            its.append(res["iterations"])
            conv.append(res["converged"])
            true_res.append(res["true_rel_residual"])
        barrier()
        per = [s.elapsed_time(e) for s, e in ev]
        total_ms = max_over_ranks(sum(per))
        clocks = sampler.stop() if headline else None
        ls_ms, ls_n = g.profile_get("local_solve")
        sp_ms, sp_n = g.profile_get("spmv")
        launches = g.launches()
        g.profile(())
        # independent FP64 check of the last solution
        x = x_dev.cpu().numpy()
        true_chk = float(np.linalg.norm(st.b - st.A @ x) / np.linalg.norm(st.b))
        results[name] = {
            "ms_per_solve": total_ms / a.steps, "per_solve_ms": per, "iterations": its, "converged": all(conv),
            "true_rel_residual": max(true_res), "true_rel_residual_host_check": true_chk,
            "local_solve_ms_total": ls_ms, "local_solve_launches": ls_n, "launches": launches,
            "local_solve_bytes": g.local_solve_bytes(), "clocks": clocks,
            "local_solve_column_bytes": g.stat("local_solve_column_bytes"),
            "spmv_ms_total": sp_ms, "spmv_calls": sp_n,
            "p50_ms": float(np.percentile(per, 50)), "p99_ms": float(np.percentile(per, 99)),
        }
    # ---- batched form: k right-hand sides solved at once on one setup (k host threads, each call on
    # its own workspace and stream); a step is one batch, timed from the first call to the last return
    import threading
    g, kw = forms["mixed"]
    batched = {}
    for k in [int(v) for v in str(a.batch).split(",") if v.strip() and int(v) > 1]:
        rng = np.random.default_rng(4321)
        bs = [b_dev] + [torch.tensor(rng.uniform(-1.0, 1.0, n), device=dev) for _ in range(k - 1)]
        xs = [torch.zeros(n, device=dev, dtype=torch.float64) for _ in range(k)]
        its_k = [None] * k
        conv_k = [None] * k

        def one_batch():
            errs = []

            def body(j):
                try:
                    _, r = g.gmres(bs[j].data_ptr(), device_out=xs[j].data_ptr(), **kw)
                    its_k[j] = r["iterations"]
                    conv_k[j] = r["converged"] and r["true_rel_residual"] <= wl.rtol
                except Exception as e:  # re-raised below
                    errs.append(e)

            for x in xs:
                x.zero_()
            torch.cuda.synchronize()
            ts = [threading.Thread(target=body, args=(j,)) for j in range(k)]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            if errs:
                raise errs[0]

        for _ in range(a.warmup):
            one_batch()
        barrier()
        per_b = []
        for _ in range(a.steps):
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            one_batch()
            e_ev.record(stream)  # every call of the batch has returned with its work complete
            e_ev.synchronize()
            per_b.append(s_ev.elapsed_time(e_ev))
        barrier()
        tot = max_over_ranks(sum(per_b))
        batched[str(k)] = {"rhs": k, "ms_per_batch": tot / a.steps, "solves_per_s": world * k * a.steps / (tot * 1e-3),
                           "iterations": list(its_k), "converged": all(conv_k),
                           "p50_batch_ms": float(np.percentile(per_b, 50)),
                           "p99_batch_ms": float(np.percentile(per_b, 99))}
        del bs, xs
    # ---- block form: k right-hand sides in one lockstep block GMRES (s2l_gpu_gmres_block): the
    # preconditioner, A and the orthogonalization run once per step for all k columns
    block = {}
    head = None
    bw = int(g.stat("block_width"))  # one block of this width is the unit wider steps run concurrently
    ks = [int(v) for v in str(a.block).split(",") if v.strip() and int(v) >= 1]
    for extra in (bw, a.head_k):
        if extra not in ks:
            ks = [extra] + ks
    for k in ks:
        is_head = k == a.head_k
        is_rf = k == bw
        rng = np.random.default_rng(4321)
        Bk = torch.stack([b_dev] + [torch.tensor(rng.uniform(-1.0, 1.0, n), device=dev) for _ in range(k - 1)])
        Xk = torch.zeros_like(Bk)
        res_k = None
        for _ in range(a.warmup):
            Xk.zero_()
            _, res_k = g.gmres_block((Bk.data_ptr(), k), device_out=Xk.data_ptr(), **kw)
        if is_rf:
            g.profile(("local_solve", "spmv"))
        if is_head:
            sampler = ClockSampler(local)
            sampler.start()
        barrier()
        per_k = []
        for _ in range(a.steps):
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            Xk.zero_()
            _, res_k = g.gmres_block((Bk.data_ptr(), k), device_out=Xk.data_ptr(), **kw)
            e_ev.record(stream)
            e_ev.synchronize()
            per_k.append(s_ev.elapsed_time(e_ev))
        barrier()
        tot = max_over_ranks(sum(per_k))
        if is_head:
            head_clocks = sampler.stop()
        if is_rf:
            rf_ls = g.profile_get("local_solve")
            rf_sp = g.profile_get("spmv")
            rf_launches = g.launches()
            g.profile(())
        Xh = Xk.cpu().numpy()
        chk = max(float(np.linalg.norm(Bk[j].cpu().numpy() - st.A @ Xh[j]) / np.linalg.norm(Bk[j].cpu().numpy()))
                  for j in range(k))
        block[str(k)] = {"rhs": k, "ms_per_block": tot / a.steps, "ms_per_solve": tot / a.steps / k,
                         "solves_per_s": world * k * a.steps / (tot * 1e-3),
                         "iterations": [r["iterations"] for r in res_k],
                         "converged": all(r["converged"] for r in res_k), "true_rel_residual_host_check": chk,
                         "p50_block_ms": float(np.percentile(per_k, 50)),
                         "p99_block_ms": float(np.percentile(per_k, 99))}
        if is_head:
            head = dict(block[str(k)], per_block_ms=per_k, clocks=head_clocks)
        if is_rf:
            rf = dict(ls=rf_ls, sp=rf_sp, launches=rf_launches, steps=a.steps)
        del Bk, Xk
    # ---- several k=4 blocks at once from host threads (each on its own workspace and stream)
    block_thr = {}
    for nt in [int(v) for v in str(a.block_threads).split(",") if v.strip() and int(v) > 1]:
        rng = np.random.default_rng(99)
        Bs = [torch.tensor(rng.uniform(-1.0, 1.0, (4, n)), device=dev) for _ in range(nt)]
        Xs = [torch.zeros_like(B_) for B_ in Bs]
        conv_t = [True] * nt

        def one_round():
            errs = []

            def body(j):
                try:
                    _, rr = g.gmres_block((Bs[j].data_ptr(), 4), device_out=Xs[j].data_ptr(), **kw)
                    conv_t[j] = all(r["converged"] for r in rr)
                except Exception as e:  # re-raised below
                    errs.append(e)

            for X_ in Xs:
                X_.zero_()
            torch.cuda.synchronize()
            ts = [threading.Thread(target=body, args=(j,)) for j in range(nt)]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            if errs:
                raise errs[0]

        for _ in range(a.warmup):
            one_round()
        barrier()
        per_t = []
        for _ in range(a.steps):
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            one_round()
            e_ev.record(stream)
            e_ev.synchronize()
            per_t.append(s_ev.elapsed_time(e_ev))
        barrier()
        tot = max_over_ranks(sum(per_t))
        block_thr[str(nt)] = {"threads": nt, "rhs_per_block": 4, "solves_per_s": world * 4 * nt * a.steps / (tot * 1e-3),
                              "converged": all(conv_t)}
        del Bs, Xs
    # ---- serving: Poisson arrivals of solve requests over three resident matrices (this workload in
    # mixed precision, the 2D Poisson case, a convection-diffusion case with FP32 LU factors) on the
    # engine's worker threads; latency = request submitted -> solution ready (host clock)
    serving = None
    if a.serve > 0:
        from s2l_b200.serving import Engine
        cases = {"bubbles3d": (lambda: st32, dict(restart=wl.restart, rtol=wl.rtol, flexible=True, strict=True))}
        wp = W.poisson2d()
        st_p = W.build(wp)
        cases["poisson2d"] = (lambda: st_p, dict(restart=wp.restart, rtol=wp.rtol))
        wc = W.convdiff3d(32, 8)
        st_c = W.build(wc)
        cases["convdiff3d"] = (lambda: st_c, dict(restart=wc.restart, rtol=wc.rtol, flexible=True, strict=True))
        eng = Engine(local, hbm_budget=150 << 30, workers=4)
        for key, (mk, kwk) in cases.items():  # warm: setups built and resident before the arrivals
            t = eng.submit(key, mk, mk().b, **kwk)
            t.wait(600.0)
            t.free()
        rng = np.random.default_rng(2026)
        keys = list(cases)
        mix = [0.5, 0.25, 0.25]
        gaps = rng.exponential(1.0 / a.serve_rate, a.serve)
        picks = rng.choice(len(keys), a.serve, p=mix)
        tickets = []
        t0 = time.perf_counter()
        t_next = t0
        for i in range(a.serve):
            t_next += gaps[i]
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            key = keys[picks[i]]
            mk, kwk = cases[key]
            b_i = rng.uniform(-1.0, 1.0, mk().n)
            tickets.append((key, eng.submit(key, mk, b_i, history_cap=0, **kwk)))
        lat = []
        per_key = {k: {"lat": [], "run": [], "its": []} for k in keys}
        ok = True
        for key, t in tickets:
            _, r, status = t.wait(600.0)
            ok = ok and status == 0 and r["converged"]
            info = t.info()
            lat.append(info["queue_ms"] + info["run_ms"])
            per_key[key]["lat"].append(info["queue_ms"] + info["run_ms"])
            per_key[key]["run"].append(info["run_ms"])
            per_key[key]["its"].append(r["iterations"])
            t.free()
        t_end = time.perf_counter()
        serving = {"requests": a.serve, "rate_req_s": a.serve_rate, "mix": dict(zip(keys, mix)),
                   "all_converged": ok, "solves_per_s": a.serve / (t_end - t0),
                   "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                   "max_ms": float(np.max(lat)), "workers": 4, "setups_built": eng.builds,
                   "per_case": {k: {"requests": len(v["lat"]),
                                    "p50_ms": float(np.percentile(v["lat"], 50)) if v["lat"] else None,
                                    "p99_ms": float(np.percentile(v["lat"], 99)) if v["lat"] else None,
                                    "run_ms_mean": float(np.mean(v["run"])) if v["run"] else None,
                                    "iterations_mean": float(np.mean(v["its"])) if v["its"] else None}
                                for k, v in per_key.items()},
                   "clock": "host (submit to solution ready)"}
        eng.close()

    serving_mix = serve_mix(a, local) if a.serve_mix > 0 else None

    # ---- AMG local solvers (the reference's --local-approx amg): the same matrix, partition and
    # coarse basis, each subdomain's A_ii^-1 replaced by one AMG V-cycle; plain FP64 GMRES
    amg_form = None
    if a.amg and a.workload == "bubbles3d":
        import dataclasses
        from s2l_b200.amg import build_hierarchy_native as build_hierarchy
        t0a = time.time()
        subs_amg = [dataclasses.replace(sd, factor=None, amg=build_hierarchy(sd.Aii)) for sd in st.subdomains]
        st_amg = dataclasses.replace(st, subdomains=subs_amg)
        amg_setup_s = time.time() - t0a
        ga = capi.GpuSetup(ctx, st_amg)
        ga.set_stream(stream.cuda_stream)
        kwa = dict(restart=wl.restart, rtol=wl.rtol, flexible=False, strict=False, maxit=2000)
        for _ in range(a.warmup):
            x_dev.zero_()
            ga.gmres(b_dev.data_ptr(), device_out=x_dev.data_ptr(), **kwa)
        ga.profile(("local_solve",))
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        its_a = []
        for k in range(a.steps):
            evs[k][0].record(stream)
            x_dev.zero_()
            _, ra = ga.gmres(b_dev.data_ptr(), device_out=x_dev.data_ptr(), **kwa)
            evs[k][1].record(stream)
            its_a.append(ra["iterations"])
        barrier()
        per_a = [s_.elapsed_time(e_) for s_, e_ in evs]
        vc_ms, vc_n = ga.profile_get("local_solve")
        ga.profile(())
        xa = x_dev.cpu().numpy()
        levels = sorted({len(sd.amg.levels) + (sd.amg.coarse is not None) for sd in subs_amg})
        amg_form = {"ms_per_solve": max_over_ranks(sum(per_a)) / a.steps, "iterations": its_a,
                    "converged": bool(ra["converged"]),
                    "true_rel_residual_host_check": float(np.linalg.norm(st.b - st.A @ xa) / np.linalg.norm(st.b)),
                    "v_cycle_ms": vc_ms / max(vc_n, 1), "levels": levels,
                    "operator_entries": int(sum(sd.amg.nnz() for sd in subs_amg)),
                    "host_setup_s": amg_setup_s,
                    "vs_plain_fp64_exact": {"ms_per_solve": results["plain_fp64"]["ms_per_solve"],
                                            "iterations": results["plain_fp64"]["iterations"]}}
        ga.close()

    # ---- end to end through the C ABI with pinned host buffers (headline block form): each step
    # copies its k right-hand sides and initial guesses in and its k solutions out
    g, kw = forms["mixed"]
    kh = a.head_k
    rng = np.random.default_rng(4321)
    b_pin = torch.empty((kh, n), dtype=torch.float64, pin_memory=True)
    b_pin.numpy()[0] = st.b
    for j in range(1, kh):
        b_pin.numpy()[j] = rng.uniform(-1.0, 1.0, n)
    x_pin = torch.zeros((kh, n), dtype=torch.float64, pin_memory=True)
    barrier()
    e2e = []
    for _ in range(a.steps):
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x_pin.zero_()
        s_ev.record(stream)
        g.gmres_block(b_pin.numpy(), X0=x_pin.numpy(), history_cap=0, **kw)
        e_ev.record(stream)
        e_ev.synchronize()
        e2e.append(s_ev.elapsed_time(e_ev))
    barrier()
    e2e_total = max_over_ranks(sum(e2e))

    # ---- sequence: the next matrices of the moving-bubble sequence (bubble centres rise half a cell
    # per step, same pattern), each refactorized on the device (s2l_gpu_refactor: new local factors
    # on the kept patterns, E with the kept basis; the reference's refactorize level) and solved for
    # head_k right-hand sides; a step is timed from the upload of the new values to the solutions
    sequence = None
    if a.seq > 0:
        import dataclasses
        import scipy.sparse as sp
        from s2l_b200 import sequence as seqmod
        g, kw = forms["mixed"]
        rng = np.random.default_rng(77)
        Bq = torch.tensor(rng.uniform(-1.0, 1.0, (kh, n)), device=dev)
        Xq = torch.zeros_like(Bq)
        steps_q = []
        for step in range(1, a.seq + 1):
            prob = W.make_problem(dataclasses.replace(wl, time=float(step)))
            vals, _ = seqmod.values_in_setup_order(prob.A, st)
            At = sp.csr_matrix((vals, st.A.indices, st.A.indptr), shape=st.A.shape)
            barrier()
            s_ev, m_ev, e_ev = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            s_ev.record(stream)
            g.refactor(vals)
            m_ev.record(stream)
            Xq.zero_()
            _, rq = g.gmres_block((Bq.data_ptr(), kh), device_out=Xq.data_ptr(), **kw)
            e_ev.record(stream)
            e_ev.synchronize()
            Xh = Xq.cpu().numpy()
            Bh = Bq.cpu().numpy()
            chk = max(float(np.linalg.norm(Bh[j] - At @ Xh[j]) / np.linalg.norm(Bh[j])) for j in range(kh))
            steps_q.append({"step": step, "refactor_ms": s_ev.elapsed_time(m_ev), "solve_ms": m_ev.elapsed_time(e_ev),
                            "refactor_phases_ms": {k: round(g.stat("refactor_ms_" + k), 2)
                                                   for k in ("coarse", "coarse_inverse", "sparse", "tail", "dense",
                                                             "commit")},
                            "iterations_max": max(r["iterations"] for r in rq),
                            "converged": all(r["converged"] for r in rq), "true_rel_residual_host_check": chk})
        g.refactor(st32.A.data)  # back to the setup's own matrix
        tot_ms = sum(q["refactor_ms"] + q["solve_ms"] for q in steps_q)
        sequence = {"matrices": a.seq, "rhs_per_matrix": kh, "update": "refactorize", "steps": steps_q,
                    "refactor_ms_mean": float(np.mean([q["refactor_ms"] for q in steps_q])),
                    "refactor_plan_gb": g.stat("refactor_bytes") / 1e9,
                    "solves_per_s": a.seq * kh / (tot_ms * 1e-3)}
        del Bq, Xq

    mixed = results["mixed"]
    plain = results["plain_fp64"]
    # roofline of the headline's dominant kernel group: the block local solve (factors read once,
    # every column's gather and owned write)
    head_bytes = g32.local_solve_bytes() + (bw - 1) * g32.stat("local_solve_column_bytes")
    ls_avg_ms = rf["ls"][0] / max(rf["ls"][1], 1)
    traffic = measured_traffic(head_bytes)
    achieved = head_bytes / (ls_avg_ms * 1e-3) / 1e9 if ls_avg_ms > 0 else 0.0
    ls_avg_ms32 = mixed["local_solve_ms_total"] / max(mixed["local_solve_launches"], 1)
    achieved32 = mixed["local_solve_bytes"] / (ls_avg_ms32 * 1e-3) / 1e9 if ls_avg_ms32 > 0 else 0.0
    ls_avg_ms64 = plain["local_solve_ms_total"] / max(plain["local_solve_launches"], 1)
    achieved64 = plain["local_solve_bytes"] / (ls_avg_ms64 * 1e-3) / 1e9 if ls_avg_ms64 > 0 else 0.0

    def rate(nbytes, ms):
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        return {"achieved": gbs, "frac": gbs / peak}

    # SpMV (y = A x and the residual forms, averaged over every call; bytes of y = A x, so a lower bound)
    spmv = {"single_column_fp32": dict(rate(spmv_bytes(st), mixed["spmv_ms_total"] / max(mixed["spmv_calls"], 1)),
                                       bytes_per_launch=spmv_bytes(st), calls=mixed["spmv_calls"]),
            "single_column_fp64": dict(rate(spmv_bytes(st), plain["spmv_ms_total"] / max(plain["spmv_calls"], 1)),
                                       bytes_per_launch=spmv_bytes(st), calls=plain["spmv_calls"]),
            f"block_{bw}": dict(rate(spmv_bytes(st, bw), rf["sp"][0] / max(rf["sp"][1], 1)),
                                bytes_per_launch=spmv_bytes(st, bw), calls=rf["sp"][1])}
    # whole solves: algorithmic bytes of every Arnoldi step over the solve's wall time
    col32 = mixed["local_solve_column_bytes"]
    per_solve = {
        "headline_block": dict(rate(gmres_solve_bytes(st, head["iterations"], wl.restart, mixed["local_solve_bytes"],
                                                      col32), head["ms_per_block"]),
                               bytes=gmres_solve_bytes(st, head["iterations"], wl.restart,
                                                       mixed["local_solve_bytes"], col32)),
        "mixed": dict(rate(gmres_solve_bytes(st, mixed["iterations"][:1], wl.restart, mixed["local_solve_bytes"],
                                             col32), mixed["ms_per_solve"]),
                      bytes=gmres_solve_bytes(st, mixed["iterations"][:1], wl.restart, mixed["local_solve_bytes"],
                                              col32)),
        "plain_fp64": dict(rate(gmres_solve_bytes(st, plain["iterations"][:1], wl.restart, plain["local_solve_bytes"],
                                                  plain["local_solve_column_bytes"]), plain["ms_per_solve"]),
                           bytes=gmres_solve_bytes(st, plain["iterations"][:1], wl.restart,
                                                   plain["local_solve_bytes"], plain["local_solve_column_bytes"])),
    }
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
            "n": st.n, "nnz": int(st.A.nnz), "n0": st.n0, "nnz_factors": st.stats.get("nnz_factors"),
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU, all subdomains resident",
            "l2": "inputs larger than L2 (local factors %.1f GB per form)" % (mixed["local_solve_bytes"] / 1e9),
            "setup_s": round(setup_s, 1) if world == 1 else None,
            "layout": {"options": layout, "tail_rows": g64.stat("tail_rows"), "sparse_nnz": g64.stat("sparse_nnz"),
                       "coupling_nnz": g64.stat("coupling_nnz"), "dense_entries": g64.stat("dense_entries"),
                       "sweep_group": g64.stat("sweep_group"), "levels_max": g64.stat("levels_max"),
                       "chain_blocks": g64.stat("chain_blocks"), "sweep_tasks": g64.stat("sweep_tasks"),
                       "sweep_padding": g64.stat("sweep_padding"), "kc_max_fp32": g32.stat("kc_max"),
                       "levels_mean": round(g64.stat("levels_mean"), 1)},
        },
        "forms": {
            "block_mixed": block,
            "mixed": {k: mixed[k] for k in ("ms_per_solve", "iterations", "converged", "true_rel_residual",
                                             "true_rel_residual_host_check", "p50_ms", "p99_ms")},
            "plain_fp64": {k: plain[k] for k in ("ms_per_solve", "iterations", "converged", "true_rel_residual",
                                                  "true_rel_residual_host_check", "p50_ms", "p99_ms")},
            "batched_mixed": batched,
            "block_mixed_threads": block_thr,
            "serving": serving,
            "serving_mix": serving_mix,
            "amg_local_solves": amg_form,
            "sequence_refactor": sequence,
            "speedup_head_vs_plain_per_solve": plain["ms_per_solve"] / head["ms_per_solve"],
            "speedup_mixed_vs_plain": plain["ms_per_solve"] / mixed["ms_per_solve"],
            "iteration_delta_mixed_vs_plain": mixed["iterations"][0] - plain["iterations"][0],
            "iteration_delta_head_vs_plain": max(head["iterations"]) - plain["iterations"][0],
        },
        "p50_ms": head["p50_block_ms"],
        "p99_ms": head["p99_block_ms"],
        "e2e": {"value": world * kh * a.steps / (e2e_total * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": 2 * 8 * n * kh, "d2h_bytes_per_step": 8 * n * kh,
                "ms_per_step": e2e_total / a.steps},
        "roofline": {"bound": "hbm",
                     "kernel": f"local solve of one {bw}-column block (sweeps, tail coupling, dense tails); the "
                               f"{kh}-column step runs {max(kh // bw, 1)} such blocks at once",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "bytes_per_launch": head_bytes, "avg_launch_ms": ls_avg_ms,
                     "single_column_fp32": {"achieved": achieved32, "frac": achieved32 / peak,
                                            "avg_launch_ms": ls_avg_ms32, "bytes_per_launch": mixed["local_solve_bytes"]},
                     "single_column_fp64": {"achieved": achieved64, "frac": achieved64 / peak,
                                            "avg_launch_ms": ls_avg_ms64, "bytes_per_launch": plain["local_solve_bytes"]},
                     "spmv": spmv, "per_solve": per_solve},
        # kernels launched in the timed region: those of the timed k=bw blocks, times the blocks
        # a k=head step runs at once
        "gpu_launches": int(rf["launches"] * max(kh // bw, 1)),
        "clocks": head["clocks"],
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(st, plain["iterations"][0], wl.restart)
    if rank == 0:
        print(json.dumps(out), flush=True)
    g64.close()
    g32.close()
    ctx.close()
    reps.close()


def serve_mix(a, device: int) -> dict:
    """Poisson arrivals (a.serve_rate per second) of a.serve_mix solve requests, each on one of 40
    seeded cases of the three workload families at several sizes (2D Poisson with LU factors,
    bubbles3d with L L^T factors, convdiff3d with FP32 LU factors and flexible GMRES), on an engine
    with a 150 GB HBM budget and 4 workers.  Every case is set up and resident before the first
    arrival; latency = request submitted -> solution ready (host clock)."""
    import numpy as np
    from s2l_b200 import workloads as W
    from s2l_b200.serving import Engine
    cases = []
    for nx in (100, 120, 140, 160, 180, 200):
        for nsub in (4, 8):
            cases.append(("poisson2d", W.poisson2d(nx, nsub)))
    for nx, nsub in ((24, 8), (24, 16), (28, 8), (28, 16), (32, 8), (32, 16), (32, 32), (36, 8), (36, 16), (36, 32),
                     (40, 8), (40, 16), (40, 32), (44, 16), (44, 32), (48, 16), (48, 32), (48, 64)):
        w = W.bubbles3d(nx, nsub, nbubbles=max(4, (nx * nx * nx) // 5000), overlap=2)
        cases.append(("bubbles3d", w))
    for nx in (24, 28, 32, 40, 48):
        for nsub in (8, 16):
            cases.append(("convdiff3d", W.convdiff3d(nx, nsub)))
    assert len(cases) == 40
    for q, (_, w) in enumerate(cases):
        w.seed = 1000 + q
    t0 = time.time()
    built = [W.build(w) for _, w in cases]
    setup_s = time.time() - t0
    eng = Engine(device, hbm_budget=150 << 30, workers=4)
    kws = []
    for (fam, w), st in zip(cases, built):
        flex = w.opts.local_precision == "single"
        kws.append(dict(restart=w.restart, rtol=w.rtol, flexible=flex, strict=flex, history_cap=0))
    for q, st in enumerate(built):  # setups resident before the arrivals (first solve of each)
        t = eng.submit(q, (lambda st=st: st), st.b, **kws[q])
        t.wait(600.0)
        t.free()
    rng = np.random.default_rng(2027)
    gaps = rng.exponential(1.0 / a.serve_rate, a.serve_mix)
    picks = rng.integers(0, len(cases), a.serve_mix)
    tickets = []
    t_start = time.perf_counter()
    t_next = t_start
    for i in range(a.serve_mix):
        t_next += gaps[i]
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        q = int(picks[i])
        st = built[q]
        b_i = rng.uniform(-1.0, 1.0, st.n)
        tickets.append((q, eng.submit(q, (lambda st=st: st), b_i, **kws[q])))
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
    out = {"requests": a.serve_mix, "rate_req_s": a.serve_rate, "cases": len(cases),
           "sizes_n": [int(min(st.n for st in built)), int(max(st.n for st in built))],
           "hbm_budget_gb": 150, "all_converged": ok, "solves_per_s": a.serve_mix / (t_end - t_start),
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "max_ms": float(np.max(lat)), "setups_built": eng.builds, "evictions": eng.evictions,
           "per_family": {f: {"requests": len(v), "p50_ms": float(np.percentile(v, 50)),
                              "p99_ms": float(np.percentile(v, 99))} for f, v in fam_lat.items()},
           "host_setup_s": setup_s, "clock": "host (submit to solution ready)"}
    eng.close()
    return out


def cpu_baseline(st, iterations: int, restart: int) -> dict:
    """The oracle (sequential C restatement) on a bounded sample: 3 GMRES iterations of the same solve."""
    from oracle.oracle import OracleSetup
    o = OracleSetup(st)
    t0 = time.perf_counter()
    _, res = o.gmres(st.b, restart=restart, rtol=1e-8, maxit=3)
    dt = time.perf_counter() - t0
    o.close()
    per_it = dt / max(res["iterations"], 1)
    est = per_it * iterations
    return {"value": 1.0 / est, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": f"{res['iterations']} GMRES iterations of the same FP64 solve ({dt:.1f} s, "
                      f"{per_it * 1e3:.0f} ms/iteration), scaled to the GPU's {iterations} iterations"}


# ------------------------------------------------------------------------------------ reference arm
def reference_workload(a):
    """The headline workload at the sizes of the arguments (0: the workload's own, 100^3 and 64
    subdomains): the reference runs one thread-rank per subdomain on the same partition."""
    from s2l_b200 import workloads as W
    return W.bubbles3d(a.nx or 100, a.nsub or 64, nbubbles=a.nbubbles, overlap=a.overlap)


def run_reference(a):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    binary = os.path.join(REPO, "oracle", "_ref", "s2l_ref")
    if not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/s2l_ref was not built "
                                                             "(the reference compiles only where its sources are)"}))
        return
    import numpy as np
    from s2l_b200 import workloads as W
    from s2l_b200.rng import random_rhs  # noqa: F401  (the reference draws the same rhs itself)

    wl = reference_workload(a)
    prob = W.make_problem(wl)
    part = W.make_partition(wl, prob).astype(np.int32)
    threads = a.ref_threads or os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        mtx = os.path.join(td, "A.mtx")
        write_mtx(mtx, prob.A)
        pf = os.path.join(td, "part.bin")
        part.tofile(pf)
        env = dict(os.environ, S2L_NP=str(wl.nsub), S2L_PART_FILE=pf, OMP_NUM_THREADS="1",
                   S2L_REF_THREADS=str(threads))
        cmd = [binary, "--matrix", mtx, "--rhs", "random", "--seed", str(wl.seed), "--pou", "boolean",
               "--one-level", "ras", "--coarse", "deflated", "--nev", "20", "--local-solver", "sparselu",
               "--local-factorization", "cholesky", "--coarse-solver", "root", "--krylov", "gmres",
               "--restart", str(wl.restart), "--rtol", str(wl.rtol), "--verbose", "0",
               "--bench-steps", str(a.steps), "--bench-warmup", str(a.warmup)]
        r = subprocess.run(cmd, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed ({r.returncode}): "
                                                              f"{r.stderr.strip().splitlines()[-1:]}"}))
        return
    rec = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    per = rec["solve_s"]
    ms = 1e3 * sum(per) / len(per)
    value = 1e3 / ms
    out = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "solves/s", "n_gpus": a.gpus,
        "steps": len(per), "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (same generator, partition and rhs)",
        "config": {"workload": f"bubbles3d {wl.nx}^3 pressure Poisson, {wl.nsub} subdomains, overlap 1 (the "
                               f"reference has no overlap 2), nev 20, deflated RAS, Eigen LL^T, root coarse "
                               f"solver, GMRES(50), rtol 1e-8",
                   "n": int(prob.n), "iterations": rec.get("iterations"), "setup_s": rec.get("setup_s"),
                   "true_rel_residual": rec.get("true_rel_residual")},
        "p50_ms": float(np.percentile(np.array(per) * 1e3, 50)), "p99_ms": float(np.percentile(np.array(per) * 1e3, 99)),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(per)} full solves, {wl.nsub} thread-ranks on {threads} host threads"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def write_mtx(path, A):
    """Matrix Market coordinate file (1-based), full precision."""
    import numpy as np
    A = A.tocoo()
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{A.shape[0]} {A.shape[1]} {A.nnz}\n")
        data = np.column_stack([A.row + 1, A.col + 1, A.data])
        np.savetxt(f, data, fmt=["%d", "%d", "%.17g"])


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
