"""Autotuner of the device layout of one setup (no counterpart in the reference).

The layout options of ``s2l_gpu_setup_option`` choose how the same factors and matrix are laid out
on the device: where each factor is split between the sparse sweeps and the dense tail (the cost
model's ``hop_us``), how long the chain blocks are (``chain_block``), how many lanes a sparse-sweep
row may take (``sweep_group``), how the product with A is spread (``spmv_tpr``) and how far ahead a
sweep warp hints its entries into L2 (``sweep_prefetch``, set on an uploaded setup).  Their best
values depend on the matrix, the partition and the precision.  ``tune`` builds device setups of the
same host setup with candidate values, times each with CUDA events on the device (the library's
kernel timers around the local solve and the SpMV of ``s2l_gpu_apply_block`` / ``s2l_gpu_spmv``),
and keeps the fastest: a coordinate search, one option at a time, starting from the defaults.

The objective is the time of one Arnoldi step's layout-dependent kernels for a block of ``k``
right-hand sides: one block local solve plus ``spmv_per_step`` products with A.
"""
from __future__ import annotations

import time

import numpy as np

from . import capi

# candidate values per option, searched in this order (the first value of each is the default)
SEARCH = (
    ("hop_us", (0.25, 0.1, 0.5, 1.0)),
    ("chain_block", (8, 4, 16)),
    ("sweep_group", (16, 32, 8)),
    ("spmv_tpr", (0, 1, 2, 4)),
    ("sweep_prefetch", (8, 16, 24)),
)
# options a device setup takes after its upload: tried on the current best setup, not on a new one
RUNTIME = ("sweep_prefetch", "spin_sleep_ns")


def measure(g: capi.GpuSetup, k: int, reps: int, rng) -> dict:
    """Average device time [ms] of one block local solve of k columns and of one product with A."""
    R = rng.uniform(-1.0, 1.0, (k, g.n))
    x = rng.uniform(-1.0, 1.0, g.n)
    g.apply_block(R)  # warm-up (and the block buffers)
    g.spmv(x)
    g.profile(("local_solve", "spmv"))
    for _ in range(reps):
        g.apply_block(R)
        g.spmv(x)
    ls_ms, ls_n = g.profile_get("local_solve")
    sp_ms, sp_n = g.profile_get("spmv")
    g.profile(())
    # the deflated apply runs a product with A of its own: keep only the spmv calls' own share
    return {"local_solve_ms": ls_ms / max(ls_n, 1), "spmv_ms": sp_ms / max(sp_n, 1)}


def tune(ctx: capi.Context, st, k: int = 4, reps: int = 5, spmv_per_step: int = 2, base=None, search=SEARCH,
         seed: int = 0):
    """Coordinate search over `search`; returns (the fastest GpuSetup, report).  `base`: options
    every candidate keeps (e.g. {"refactor": 1})."""
    rng = np.random.default_rng(seed)
    base = dict(base or {})
    current = {}
    best_g, best_t, best_m = None, None, None
    report = {"k": k, "reps": reps, "candidates": []}
    t0 = time.perf_counter()

    def objective(m):
        return m["local_solve_ms"] + spmv_per_step * m["spmv_ms"]

    def trial(opts):
        nonlocal best_g, best_t, best_m
        g = capi.GpuSetup(ctx, st, options=dict(base, **opts))
        m = measure(g, k, reps, rng)
        t = objective(m)
        report["candidates"].append(dict(options=dict(opts), ms=t, **m))
        if best_t is None or t < best_t:
            if best_g is not None:
                best_g.close()
            best_g, best_t, best_m = g, t, m
            return True
        g.close()
        return False

    def runtime_trial(opts, name, v):
        nonlocal best_t, best_m
        best_g.set_option(name, v)
        m = measure(best_g, k, reps, rng)
        t = objective(m)
        report["candidates"].append(dict(options=dict(opts), ms=t, **m))
        if t < best_t:
            best_t, best_m = t, m
            return True
        return False

    trial({})
    default_t = best_t
    for name, values in search:
        chosen = current.get(name)
        for v in values[1:]:
            opts = dict(current, **{name: v})
            if name in RUNTIME:
                if runtime_trial(opts, name, v):
                    chosen = v
                else:  # back to the value the best setup had
                    best_g.set_option(name, chosen if chosen is not None else values[0])
            elif trial(opts):
                chosen = v
        if chosen is not None:
            current[name] = chosen
    report.update(chosen=current, ms=best_t, default_ms=default_t, gain=default_t / best_t if best_t else None,
                  tune_s=time.perf_counter() - t0, **{"chosen_" + q: v for q, v in best_m.items()})
    return best_g, report
