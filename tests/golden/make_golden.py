#!/usr/bin/env python
"""Generates the golden fixtures of tests/golden/ by running the reference itself.

The reference (fraBuffoli/Algebraic-Multilevel-Preconditioner) is built from its own sources with
oracle/ref/Makefile into oracle/_ref/s2l_ref (thread-rank MPI stand-in, METIS stand-in).  For every
case below it runs in dump mode and the outputs are packed into <case>.npz:

  global_*    renumbered matrix A (CSR), right-hand side b, partition, ownership, coarse offsets
  subI_*      per subdomain: meta [begin, n_owned, n_ghost, m], ghosts, D, V (column-major), the
              exact local factors (Eigen SparseLU / SimplicialLLT / LDLT; perm_in/perm_out), A_ii,
              and one local solve of the reference's LocalSolver (ls_b -> ls_x)
  applyK_*    seeded r (mt19937_64(1000+K), U[-1,1], renumbered ordering) and the reference's
              DistributedMatrix::apply, OneLevelSchwarz::apply, CoarseSpace::apply and
              Preconditioner::apply of it
  krylov_*    the reference's Krylov solve of A x = b from x0 = 0: x, residual history, and
              [iterations, converged, rel_residual, true_rel_residual, restarts, breakdown,
               initial_residual_of, final_residual_of] (the last two for --stop-norm openfoam)

Run here (where the reference sources are): python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(REPO, "oracle", "_ref", "s2l_ref")

COMMON = ["--rhs", "random", "--seed", "12345", "--local-solver", "sparselu", "--coarse-solver", "root",
          "--verbose", "0", "--rtol", "1e-8"]

CASES = {
    # the 2D Poisson family (RAS + additive coarse term, exact LU), small
    "laplace2d_ras_additive_lu": (4, ["--generate", "laplace2d", "--nx", "24", "--pou", "boolean", "--one-level",
                                      "ras", "--coarse", "additive", "--nev", "8", "--local-factorization", "lu",
                                      "--restart", "30"]),
    # multiplicity partition of unity, ASM, deflated, Cholesky chain
    "laplace2d_asm_deflated_mult": (3, ["--generate", "laplace2d", "--nx", "20", "--pou", "multiplicity",
                                        "--one-level", "asm", "--coarse", "deflated", "--nev", "6",
                                        "--local-factorization", "cholesky", "--restart", "30"]),
    # the bubbly-pressure family (deflated RAS, L L^T), small
    "bubbles3d_ras_deflated_llt": (4, ["--generate", "bubbles3d", "--nx", "12", "--nbubbles", "6", "--radius",
                                       "0.15", "--rho-ratio", "1000", "--pou", "boolean", "--one-level", "ras",
                                       "--coarse", "deflated", "--nev", "10", "--local-factorization", "cholesky",
                                       "--restart", "50"]),
    # nonsymmetric convection-diffusion, LU factors in single precision
    "convdiff3d_ras_deflated_lu_single": (4, ["--generate", "convdiff3d", "--nx", "10", "--pou", "boolean",
                                              "--one-level", "ras", "--coarse", "deflated", "--nev", "8",
                                              "--local-factorization", "lu", "--local-precision", "single",
                                              "--restart", "40"]),
    # BiCGStab with the 2D Poisson problem, one-level RAS only
    "laplace2d_bicgstab_onelevel": (4, ["--generate", "laplace2d", "--nx", "20", "--pou", "boolean",
                                        "--one-level", "ras", "--coarse", "none", "--local-factorization", "lu",
                                        "--krylov", "bicgstab"]),
    # LDL^T factors (the second link of the reference's Cholesky -> LDL^T -> LU chain)
    "laplace2d_ras_deflated_ldlt": (2, ["--generate", "laplace2d", "--nx", "16", "--pou", "boolean",
                                        "--one-level", "ras", "--coarse", "deflated", "--nev", "6",
                                        "--local-factorization", "ldlt", "--restart", "30"]),
    # OpenFOAM stopping norm (relTol semantics), GMRES on the bubbly-pressure family
    "bubbles3d_gmres_openfoam": (4, ["--generate", "bubbles3d", "--nx", "12", "--nbubbles", "6", "--radius", "0.15",
                                     "--rho-ratio", "1000", "--pou", "boolean", "--one-level", "ras", "--coarse",
                                     "deflated", "--nev", "10", "--local-factorization", "cholesky", "--restart",
                                     "20", "--stop-norm", "openfoam", "--rtol", "1e-6"]),
    # OpenFOAM norm with an absolute tolerance only (relTol 0), BiCGStab, two-level additive
    "laplace2d_bicgstab_openfoam_atol": (3, ["--generate", "laplace2d", "--nx", "20", "--pou", "boolean",
                                             "--one-level", "ras", "--coarse", "additive", "--nev", "6",
                                             "--local-factorization", "lu", "--krylov", "bicgstab", "--stop-norm",
                                             "openfoam", "--rtol", "0", "--atol", "1e-9"]),
}


def load_dump(d: str) -> dict:
    out = {}
    dt = {"f64": np.float64, "f32": np.float32, "i64": np.int64, "i32": np.int32}
    for f in sorted(os.listdir(d)):
        if not f.startswith("manifest_rank"):
            continue
        for line in open(os.path.join(d, f)):
            name, t, cnt = line.split()
            out[name] = np.fromfile(os.path.join(d, name + ".bin"), dtype=dt[t], count=int(cnt))
    return out


def run_case(name: str, np_: int, args: list, dest: str) -> dict:
    with tempfile.TemporaryDirectory() as td:
        env = dict(os.environ, S2L_NP=str(np_), OMP_NUM_THREADS="1")
        cmd = [BIN, *COMMON, *args, "--dump-dir", td, "--napply", "2"]
        r = subprocess.run(cmd, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: reference run failed\n{r.stdout}\n{r.stderr}")
        data = load_dump(td)
    data["command"] = np.array(" ".join(["S2L_NP=" + str(np_), "s2l_ref", *COMMON, *args]))
    np.savez_compressed(dest, **data)
    return data


def main(names=None):
    if not os.path.exists(BIN):
        sys.exit(f"{BIN} missing: build it with `make -C oracle/ref` (needs the reference sources)")
    for name, (np_, args) in CASES.items():
        if names and name not in names:
            continue
        dest = os.path.join(HERE, name + ".npz")
        d = run_case(name, np_, args, dest)
        km = d["krylov_meta"]
        print(f"{name}: n={int(d['global_meta'][0])} nsub={np_} n0={int(d['global_meta'][3])} "
              f"iterations={int(km[0])} converged={bool(km[1])} true_res={km[3]:.2e} "
              f"({os.path.getsize(dest) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main(sys.argv[1:])
