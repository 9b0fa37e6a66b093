#!/usr/bin/env python
"""Writes tests/golden/bubbles3d_24_generator.npz from the reference's own 24^3 bubbles fixture
(test/gamg/run_gamg_23038420/check_s2l.mtx and check_s2l_rhs.mtx, written by the reference's
matrix generator: bubbles3d 24^3, nb=150, R=0.04, rho_ratio=1000, cfl=0.5, t=3, seed=2024, the
alpha source; the reference's own check found them equal to OpenFOAM's assembly).  Stored: the
CSR pattern's SHA-256, the values in CSR order and the generated right-hand side.

Run where the reference sources are: python tests/golden/make_bubbles_fixture.py
"""
import hashlib
import os

import numpy as np
import scipy.io
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(os.environ.get("S2L_REFERENCE_DIR", "/root/reference"), "test/gamg/run_gamg_23038420")


def pattern_hash(A: sp.csr_matrix) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(A.indptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(A.indices, dtype=np.int64).tobytes())
    return h.hexdigest()


def main():
    A = sp.csr_matrix(scipy.io.mmread(os.path.join(SRC, "check_s2l.mtx")))
    A.sort_indices()
    b = np.asarray(scipy.io.mmread(os.path.join(SRC, "check_s2l_rhs.mtx")), dtype=np.float64).ravel()
    np.savez_compressed(os.path.join(HERE, "bubbles3d_24_generator.npz"), pattern_sha256=pattern_hash(A),
                        n=A.shape[0], data=A.data, rhs=b)


if __name__ == "__main__":
    main()
