"""A sequence of matrices with one preconditioner (the reference's UpdateLevel::Reuse).

s2l_gpu_update_matrix gives A new values with the same pattern and keeps the factors, the coarse
basis and E.  The GPU must then match the oracle built from the new A with the old local
factors, basis and E: the two-level apply to 1e-12 (the deflated apply multiplies by A) and GMRES
to +-1 iteration with the FP64 true residual of the new A <= rtol.
"""
import dataclasses

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import small_setup
from oracle.oracle import OracleSetup

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _rescaled(st, seed):
    """D A D (D diagonal, within 10% of 1): same pattern and CSR order, still SPD."""
    rng = np.random.default_rng(seed)
    d = 1.0 + 0.1 * rng.uniform(-1.0, 1.0, st.n)
    A = st.A.tocsr()
    rows = np.repeat(np.arange(st.n), np.diff(A.indptr))
    A2 = sp.csr_matrix((A.data * d[rows] * d[A.indices], A.indices.copy(), A.indptr.copy()), shape=A.shape)
    return A2


def test_update_matrix_keeps_the_preconditioner():
    from s2l_b200 import capi
    ctx = capi.Context(0)
    w, st = small_setup("bubbles3d")
    g = capi.GpuSetup(ctx, st)
    rng = np.random.default_rng(41)
    for step in range(2):  # two matrices of the sequence, one setup
        A2 = _rescaled(st, 100 + step)
        st2 = dataclasses.replace(st, A=A2)  # new operator, old factors / basis / E
        o2 = OracleSetup(st2)
        g.update_matrix(A2.data)
        x = rng.standard_normal(st.n)
        assert rel(g.spmv(x), A2 @ x) <= 1e-14
        r = rng.standard_normal(st.n)
        assert rel(g.apply(r), o2.apply(r)) <= 1e-12
        xg, rg = g.gmres(st.b, restart=w.restart, rtol=1e-8)
        xo, ro = o2.gmres(st.b, restart=w.restart, rtol=1e-8)
        assert rg["converged"] and ro["converged"] and abs(rg["iterations"] - ro["iterations"]) <= 1
        assert np.linalg.norm(st.b - A2 @ xg) <= 1.1e-8 * np.linalg.norm(st.b)
        o2.close()
    g.close()
    ctx.close()


def test_update_matrix_refused_while_a_solve_runs():
    from s2l_b200 import capi
    ctx = capi.Context(0)
    ctx.serve_start(1)
    w, st = small_setup("bubbles3d")
    g = capi.GpuSetup(ctx, st)
    t = g.submit(st.b, restart=w.restart, rtol=0.0, maxit=10**7, history_cap=0)  # runs until canceled
    with pytest.raises(capi.S2LError) as e:
        g.update_matrix(st.A.data)
    assert e.value.code == 7
    t.cancel()
    t.wait(60.0)
    t.free()
    g.update_matrix(st.A.data)  # fine once nothing runs
    g.close()
    ctx.close()
