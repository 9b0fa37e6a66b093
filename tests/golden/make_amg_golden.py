"""Golden vectors of the reference's AMG local solver (``--local-approx amg``).

Runs the reference itself (oracle/_ref/amg_dump, built from the reference's sources by
oracle/ref/Makefile) on local matrices A_ii of the three workload families and stores A_ii, seeded
vectors and the reference's solve() of each (one AMGCL V-cycle from x = 0, smoothed aggregation or
Ruge-Stuben coarsening, Gauss-Seidel) in tests/golden/amg_<case>.npz; and, for the reference's refactorize() along the
moving-bubble sequence (a new hierarchy, or --amg-reuse), in tests/golden/amg_refactor_<case>.npz.
Test infrastructure; run it where the reference
sources are:  python tests/golden/make_amg_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "algebraic-multilevel-preconditioner_b200"))
DUMP = os.path.join(REPO, "oracle", "_ref", "amg_dump")

CASES = {  # name: (family, setup keywords, subdomain, coarse_enough, sweeps[, coarsening])
    "bubbles3d_3lev": ("bubbles3d", {}, 0, 50, 1),
    "bubbles3d_2lev_sweeps2": ("bubbles3d", {}, 1, 200, 2),
    "poisson2d_3lev": ("poisson2d", {}, 0, 50, 1),
    "convdiff3d_3lev": ("convdiff3d", {}, 0, 50, 1),
    "convdiff3d_direct": ("convdiff3d", {}, 2, 500, 1),
    # Ruge-Stuben coarsening (--amg-coarsening rs)
    "rs_bubbles3d": ("bubbles3d", {}, 0, 50, 1, "rs"),
    "rs_bubbles3d_sweeps2": ("bubbles3d", {}, 5, 100, 2, "rs"),
    "rs_poisson2d": ("poisson2d", {}, 1, 30, 1, "rs"),
    "rs_convdiff3d": ("convdiff3d", {}, 0, 50, 1, "rs"),
}


# single precision (--local-precision single: AMGCL's builtin<float>, setup and V-cycle in float)
SINGLE_CASES = {  # name: (family, setup keywords, subdomain, coarse_enough, sweeps, coarsening)
    "single_bubbles3d_3lev": ("bubbles3d", {}, 0, 50, 1, "sa"),
    "single_poisson2d_3lev": ("poisson2d", {}, 0, 50, 1, "sa"),
    "single_rs_convdiff3d": ("convdiff3d", {}, 0, 50, 1, "rs"),
    "single_rs_bubbles3d_sweeps2": ("bubbles3d", {}, 5, 100, 2, "rs"),
}


# refactorization: the reference's solver set up on A_ii of the bubble sequence at time 0, then
# refactorize()d with A_ii at a later time (bubbles moved), with and without --amg-reuse
REFACTOR_CASES = {  # name: (subdomain, coarse_enough, sweeps, time of the new matrix, reuse)
    "bubbles3d_reuse": (0, 50, 1, 4.0, 1),
    "bubbles3d_new": (0, 50, 1, 4.0, 0),
    "bubbles3d_reuse_2lev": (3, 200, 2, 6.0, 1),
}


def write_matrix(path, A, vecs=()):
    with open(path, "wb") as f:
        np.array([A.shape[0], A.nnz, len(vecs)], dtype=np.int64).tofile(f)
        A.indptr.astype(np.int64).tofile(f)
        A.indices.astype(np.int64).tofile(f)
        A.data.astype(np.float64).tofile(f)
        if len(vecs):
            np.asarray(vecs, dtype=np.float64).tofile(f)


def reference_apply(A, vecs, coarse_enough, sweeps, A_next=None, reuse=0, coarsening="sa", single=False):
    A = sp.csr_matrix(A)
    A.sort_indices()
    with tempfile.TemporaryDirectory() as d:
        fin, fout, fnext = os.path.join(d, "in.bin"), os.path.join(d, "out.bin"), os.path.join(d, "next.bin")
        write_matrix(fin, A, vecs)
        cmd = [DUMP, fin, fout, str(coarse_enough), str(sweeps), coarsening]
        if A_next is not None:
            A_next = sp.csr_matrix(A_next)
            A_next.sort_indices()
            write_matrix(fnext, A_next)
            cmd += [fnext, str(int(reuse))]
        env = dict(os.environ, S2L_AMG_SINGLE="1" if single else "0")
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode:
            raise RuntimeError(r.stderr)
        return np.fromfile(fout).reshape(len(vecs), -1), r.stderr.strip()


def main():
    from conftest import small_setup
    for name, case in CASES.items():
        fam, kw, i, ce, sweeps = case[:5]
        coarsening = case[5] if len(case) > 5 else "sa"
        _, st = small_setup(fam, **kw)
        s = st.subdomains[i]
        idx = s.l2g()
        A = sp.csr_matrix(st.A[idx][:, idx])
        A.sort_indices()
        vecs = np.random.default_rng(700 + i).uniform(-1.0, 1.0, (2, A.shape[0]))
        out, info = reference_apply(A, vecs, ce, sweeps, coarsening=coarsening)
        extra = {"coarsening": coarsening} if coarsening != "sa" else {}
        np.savez_compressed(os.path.join(HERE, f"amg_{name}.npz"), indptr=A.indptr, indices=A.indices, data=A.data,
                            vecs=vecs, out=out, coarse_enough=ce, sweeps=sweeps, info=info, **extra)
        print(name, A.shape[0], info)
    for name, (fam, kw, i, ce, sweeps, coarsening) in SINGLE_CASES.items():
        _, st = small_setup(fam, **kw)
        s = st.subdomains[i]
        idx = s.l2g()
        A = sp.csr_matrix(st.A[idx][:, idx])
        A.sort_indices()
        vecs = np.random.default_rng(900 + i).uniform(-1.0, 1.0, (2, A.shape[0]))
        out, info = reference_apply(A, vecs, ce, sweeps, coarsening=coarsening, single=True)
        np.savez_compressed(os.path.join(HERE, f"amg_{name}.npz"), indptr=A.indptr, indices=A.indices, data=A.data,
                            vecs=vecs, out=out, coarse_enough=ce, sweeps=sweeps, info=info, coarsening=coarsening,
                            precision="single")
        print(name, A.shape[0], info)
    import dataclasses
    from s2l_b200 import sequence as seqmod
    from s2l_b200 import workloads as W
    w, st = small_setup("bubbles3d")
    for name, (i, ce, sweeps, t, reuse) in REFACTOR_CASES.items():
        s = st.subdomains[i]
        idx = s.l2g()
        A0 = sp.csr_matrix(st.A[idx][:, idx])
        A0.sort_indices()
        vals, _ = seqmod.values_in_setup_order(W.make_problem(dataclasses.replace(w, time=t)).A, st)
        A1g = sp.csr_matrix((vals, st.A.indices, st.A.indptr), shape=st.A.shape)
        A1 = sp.csr_matrix(A1g[idx][:, idx])
        A1.sort_indices()
        vecs = np.random.default_rng(800 + i).uniform(-1.0, 1.0, (2, A0.shape[0]))
        out, info = reference_apply(A0, vecs, ce, sweeps, A_next=A1, reuse=reuse)
        np.savez_compressed(os.path.join(HERE, f"amg_refactor_{name}.npz"), indptr=A0.indptr, indices=A0.indices,
                            data=A0.data, data_next=A1.data, vecs=vecs, out=out, coarse_enough=ce, sweeps=sweeps,
                            reuse=reuse, info=info)
        print("refactor", name, A0.shape[0], info)


if __name__ == "__main__":
    main()
