"""Matrix sequences: the next matrix of a sequence into an existing setup's numbering.

The reference reads step k of a sequence (``--matrix p_%04d.mtx``, ``--rhs ...``) and refills only
the values and the right-hand side of the decomposed system, after checking that the size, the
symmetry and the sparsity pattern did not change (``DomainDecomposer::updateValues``,
``src/partition/domain_decomposer.cpp:335-388``).  Here the same check is made against a setup,
and the values come out in the order of the setup's renumbered CSR, ready for
``GpuSetup.update_matrix`` (``s2l_gpu_update_matrix``) or ``Engine.update``.
"""
from __future__ import annotations

import numpy as np
import scipy.io
import scipy.sparse as sp

from . import partition as partmod


class PatternChanged(ValueError):
    pass


def read_mtx(path: str) -> sp.csr_matrix:
    """A Matrix Market file as CSR (sorted columns, explicit zeros kept)."""
    A = sp.csr_matrix(scipy.io.mmread(path))
    A.sort_indices()
    return A


def new_to_old(st) -> np.ndarray:
    """The setup's renumbering (new row i is original row new_to_old[i])."""
    _, n2o, _ = partmod.renumber(st.stats["part"], st.nsub)
    return n2o


def values_in_setup_order(A_next: sp.spmatrix, st, b_next: np.ndarray | None = None):
    """(values, b) of the next matrix (original numbering) in the order of st.A's CSR.

    Raises PatternChanged when the size or the sparsity pattern differs from the setup's matrix.
    """
    A_next = sp.csr_matrix(A_next)
    if A_next.shape != st.A.shape:
        raise PatternChanged(f"size changed: {A_next.shape} != {st.A.shape}")
    n2o = new_to_old(st)
    Ap = partmod.permute(A_next, n2o)
    Ap.sort_indices()
    if not (np.array_equal(Ap.indptr, st.A.indptr) and np.array_equal(Ap.indices, st.A.indices)):
        raise PatternChanged("the sparsity pattern changed")
    b = None if b_next is None else np.ascontiguousarray(np.asarray(b_next, dtype=np.float64)[n2o])
    return np.ascontiguousarray(Ap.data, dtype=np.float64), b


def load_step(pattern: str, step: int, st, rhs_pattern: str | None = None):
    """Step `step` of a sequence of Matrix Market files (``pattern % step``), in setup order."""
    A = read_mtx(pattern % step)
    b = None
    if rhs_pattern:
        b = np.asarray(scipy.io.mmread(rhs_pattern % step)).ravel()
    return values_in_setup_order(A, st, b)
