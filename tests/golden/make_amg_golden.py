"""Golden vectors of the reference's AMG local solver (``--local-approx amg``).

Runs the reference itself (oracle/_ref/amg_dump, built from the reference's sources by
oracle/ref/Makefile) on local matrices A_ii of the three workload families and stores A_ii, seeded
vectors and the reference's solve() of each (one AMGCL V-cycle from x = 0, smoothed aggregation,
Gauss-Seidel) in tests/golden/amg_<case>.npz.  Test infrastructure; run it where the reference
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

CASES = {  # name: (family, setup keywords, subdomain, coarse_enough, sweeps)
    "bubbles3d_3lev": ("bubbles3d", {}, 0, 50, 1),
    "bubbles3d_2lev_sweeps2": ("bubbles3d", {}, 1, 200, 2),
    "poisson2d_3lev": ("poisson2d", {}, 0, 50, 1),
    "convdiff3d_3lev": ("convdiff3d", {}, 0, 50, 1),
    "convdiff3d_direct": ("convdiff3d", {}, 2, 500, 1),
}


def reference_apply(A, vecs, coarse_enough, sweeps):
    A = sp.csr_matrix(A)
    A.sort_indices()
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            np.array([A.shape[0], A.nnz, len(vecs)], dtype=np.int64).tofile(f)
            A.indptr.astype(np.int64).tofile(f)
            A.indices.astype(np.int64).tofile(f)
            A.data.astype(np.float64).tofile(f)
            np.asarray(vecs, dtype=np.float64).tofile(f)
        r = subprocess.run([DUMP, fin, fout, str(coarse_enough), str(sweeps), "sa"], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stderr)
        return np.fromfile(fout).reshape(len(vecs), -1), r.stderr.strip()


def main():
    from conftest import small_setup
    for name, (fam, kw, i, ce, sweeps) in CASES.items():
        _, st = small_setup(fam, **kw)
        s = st.subdomains[i]
        idx = s.l2g()
        A = sp.csr_matrix(st.A[idx][:, idx])
        A.sort_indices()
        vecs = np.random.default_rng(700 + i).uniform(-1.0, 1.0, (2, A.shape[0]))
        out, info = reference_apply(A, vecs, ce, sweeps)
        np.savez_compressed(os.path.join(HERE, f"amg_{name}.npz"), indptr=A.indptr, indices=A.indices, data=A.data,
                            vecs=vecs, out=out, coarse_enough=ce, sweeps=sweeps, info=info)
        print(name, A.shape[0], info)


if __name__ == "__main__":
    main()
