"""Runs of the reference itself, built from its sources into oracle/_ref/.  TEST INFRASTRUCTURE ONLY:
the GPU parity tests and the benchmark's CPU-baseline leg use them as the checker and the baseline;
the product path never does.

* ``s2l_ref``: the reference's decomposition, TwoLevelSchwarz and Krylov solver on thread-ranks (an
  in-process MPI stand-in); bench mode prints one JSON record (setup time, per-solve times,
  iterations, true residual).
* ``dropin_check``: on the same thread-ranks and set-up objects, the reference's preconditioner and
  Krylov solver against the GPU drop-in (host/s2l_dropin.*): Preconditioner::apply of seeded
  vectors (relative difference), and GMRES iterations, true residual and solution difference.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "s2l_ref")
DROPIN_BIN = os.path.join(HERE, "_ref", "dropin_check")
COMMON = ["--local-solver", "sparselu", "--coarse-solver", "root", "--verbose", "0", "--rhs", "random"]

# The benchmark configurations at their full sizes on the reference's own generators:
#  c1: 2D Poisson 200 x 200 (n = 40,000), 8 subdomains, RAS + additive coarse term, nev 20, exact LU,
#      GMRES(30), rtol 1e-8 (the configuration the reference itself runs, src/main.cpp:160-170);
#  c2 at overlap 1: bubbly pressure 100^3 (n = 1.0M), 200 bubbles, density ratio 1000, 64 subdomains,
#      deflated RAS, nev 20, L L^T, GMRES(50), rtol 1e-8 (the reference's generator has one radius for
#      every bubble: 0.055 = 5.5 cells, the middle of the configuration's 3-8 cells; the reference's
#      overlap is one layer)
FULL_SIZE = {
    "c1_laplace2d_200_8sub": (8, ["--generate", "laplace2d", "--nx", "200", "--nev", "20", "--coarse", "additive",
                                  "--one-level", "ras", "--local-factorization", "lu", "--restart", "30",
                                  "--rtol", "1e-8", "--seed", "12345"]),
    "c2_bubbles3d_100_64sub_overlap1": (64, ["--generate", "bubbles3d", "--nx", "100", "--nbubbles", "200",
                                             "--radius", "0.055", "--rho-ratio", "1000", "--nev", "20", "--coarse",
                                             "deflated", "--one-level", "ras", "--local-factorization", "cholesky",
                                             "--restart", "50", "--rtol", "1e-8", "--seed", "12345"]),
}


def dropin(np_: int, args: list, env_extra: dict | None = None, timeout: float = 1200.0) -> dict:
    """dropin_check on np_ thread-ranks with the reference's flags `args`: apply_rel_diff,
    ref_iterations, gpu_iterations, gpu_true_rel_residual, x_rel_diff, ok (and rc)."""
    env = dict(os.environ, S2L_NP=str(np_), OMP_NUM_THREADS="1", **(env_extra or {}))
    r = subprocess.run([DROPIN_BIN, *COMMON, *args], env=env, capture_output=True, text=True, timeout=timeout)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if not lines:
        raise RuntimeError(f"dropin_check: no result (rc={r.returncode}): {r.stderr[-2000:]}")
    return dict(json.loads(lines[-1]), rc=r.returncode)


def write_mtx(path: str, A) -> None:
    """Matrix Market coordinate file (1-based), full precision (%.17g round-trips FP64)."""
    A = A.tocoo()
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{A.shape[0]} {A.shape[1]} {A.nnz}\n")
        rows, cols, vals = A.row + 1, A.col + 1, A.data
        step = 1 << 18
        for s in range(0, A.nnz, step):
            e = min(A.nnz, s + step)
            f.write("".join(f"{r} {c} {v:.17g}\n"
                            for r, c, v in zip(rows[s:e].tolist(), cols[s:e].tolist(), vals[s:e].tolist())))


class MatrixCase:
    """A matrix, its partition and the reference's flags for it (Matrix Market file and partition
    file in a temporary directory, read by the reference's --matrix and the METIS stand-in)."""

    def __init__(self, A, part, nsub: int, flags: list):
        import numpy as np
        self.td = tempfile.TemporaryDirectory()
        self.mtx = os.path.join(self.td.name, "A.mtx")
        write_mtx(self.mtx, A)
        self.part = os.path.join(self.td.name, "part.bin")
        np.asarray(part, dtype=np.int32).tofile(self.part)
        self.nsub = nsub
        self.flags = ["--matrix", self.mtx, *flags]

    def env(self) -> dict:
        return {"S2L_PART_FILE": self.part}

    def bench(self, steps: int, warmup: int) -> dict | None:
        """The reference's bench mode: setup, `warmup` untimed and `steps` timed solves."""
        env = dict(os.environ, S2L_NP=str(self.nsub), OMP_NUM_THREADS="1", **self.env())
        r = subprocess.run([REF_BIN, *self.flags, "--verbose", "0", "--bench-steps", str(steps), "--bench-warmup",
                            str(warmup)], env=env, capture_output=True, text=True)
        if r.returncode != 0:
            return None
        return json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])

    def dropin(self) -> dict:
        return dropin(self.nsub, self.flags, self.env())

    def close(self):
        self.td.cleanup()
