"""A new preconditioner for new matrix values, on the device (the reference's UpdateLevel::Refactorize).

s2l_gpu_refactor refactorizes every local factor on its kept pattern and permutations and
recomputes E = W^T A W with the kept coarse basis.  The oracle does the same on the CPU
(oracle.refactor_setup: its refactorization reproduces SuperLU's factors to rounding, and the
coarse matrix comes from the host setup code).  The GPU must then match the oracle built from the
refactorized setup: the two-level apply to 1e-12 with FP64 factors (1e-5 with FP32 factors),
GMRES to +-1 iteration with the FP64 true residual <= rtol.  A failed refactorization
(non-positive pivot, non-finite value) must leave the setup as it was.
"""
import dataclasses

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import small_setup
from oracle.oracle import OracleSetup, refactor_setup

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def ctx():
    from s2l_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def _new_values(st, seed, symmetric):
    """Same pattern, new values: D A D (D within 10% of 1) and, for a nonsymmetric matrix, 5%
    independent noise on every entry."""
    rng = np.random.default_rng(seed)
    d = 1.0 + 0.1 * rng.uniform(-1.0, 1.0, st.n)
    A = st.A.tocsr()
    rows = np.repeat(np.arange(st.n), np.diff(A.indptr))
    v = A.data * d[rows] * d[A.indices]
    if not symmetric:
        v = v * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, v.size))
    return sp.csr_matrix((v, A.indices.copy(), A.indptr.copy()), shape=A.shape)


CASES = [
    ("bubbles3d", {}, {}),
    ("bubbles3d", {"precision": "single"}, {}),
    ("bubbles3d", {}, {"chain_block": 1, "tail_max": 0}),
    ("convdiff3d", {}, {}),
    ("convdiff3d", {"precision": "single"}, {"tail_rows": 40}),
    ("poisson2d", {"nx": 24, "nsub": 4, "pou": "multiplicity", "one_level": "asm", "coarse": "additive"}, {}),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_refactor_matches_oracle(ctx, case):
    from s2l_b200.capi import GpuSetup
    name, kw, layout = CASES[case]
    w, st = small_setup(name, **kw)
    g = GpuSetup(ctx, st, options=dict(layout, refactor=1))
    assert g.stat("refactor_bytes") > 0
    rng = np.random.default_rng(31 + case)
    tol = 1e-5 if kw.get("precision") == "single" else 1e-12
    for step in range(2):  # two matrices of a sequence on one setup
        A2 = _new_values(st, 200 + 10 * case + step, st.symmetric)
        st2 = refactor_setup(st, A2)
        o2 = OracleSetup(st2)
        g.refactor(A2.data)
        x = rng.standard_normal(st.n)
        assert rel(g.spmv(x), A2 @ x) <= 1e-14
        for _ in range(2):
            r = rng.standard_normal(st.n)
            assert rel(g.apply(r), o2.apply(r)) <= tol, rel(g.apply(r), o2.apply(r))
            if st.n0:
                assert rel(g.coarse_apply(r), o2.coarse_apply(r)) <= 1e-11
        flexible = kw.get("precision") == "single"
        xg, rg = g.gmres(st.b, restart=w.restart, rtol=1e-8, flexible=flexible, strict=flexible)
        xo, ro = o2.gmres(st.b, restart=w.restart, rtol=1e-8, flexible=flexible, strict=flexible)
        assert rg["converged"] and ro["converged"]
        assert abs(rg["iterations"] - ro["iterations"]) <= 1
        assert np.linalg.norm(st.b - A2 @ xg) <= 1.1e-8 * np.linalg.norm(st.b)
        o2.close()
    g.close()


def test_refactor_same_values_keeps_the_preconditioner(ctx):
    """Refactorizing the setup's own matrix gives back the setup's preconditioner."""
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st, options={"refactor": 1})
    r = np.random.default_rng(3).standard_normal(st.n)
    z0 = g.apply(r)
    g.refactor(st.A.data)
    assert rel(g.apply(r), z0) <= 1e-12
    g.close()


def test_refactor_moving_bubbles_converges_like_a_new_setup(ctx):
    """The next matrices of the moving-bubble sequence: refactorized, GMRES converges in about the
    iterations of the oracle on the refactorized setup."""
    from s2l_b200 import workloads as W
    from s2l_b200 import sequence as seqmod
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st, options={"refactor": 1})
    for step in (1, 2):
        prob = W.make_problem(dataclasses.replace(w, time=float(step)))
        vals, _ = seqmod.values_in_setup_order(prob.A, st)
        A2 = sp.csr_matrix((vals, st.A.indices, st.A.indptr), shape=st.A.shape)
        g.refactor(vals)
        o2 = OracleSetup(refactor_setup(st, A2))
        xg, rg = g.gmres(st.b, restart=w.restart, rtol=1e-8)
        _, ro = o2.gmres(st.b, restart=w.restart, rtol=1e-8)
        assert rg["converged"] and abs(rg["iterations"] - ro["iterations"]) <= 1
        assert np.linalg.norm(st.b - A2 @ xg) <= 1.1e-8 * np.linalg.norm(st.b)
        o2.close()
    g.close()


def test_refactor_failure_leaves_the_setup_unchanged(ctx):
    from s2l_b200.capi import GpuSetup, S2LError
    _, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st, options={"refactor": 1})
    r = np.random.default_rng(4).standard_normal(st.n)
    z0 = g.apply(r)
    with pytest.raises(S2LError) as e:
        g.refactor(-st.A.data)  # negative definite: L L^T fails at the first pivot
    assert e.value.code == 4
    bad = st.A.data.copy()
    bad[7] = np.nan
    with pytest.raises(S2LError) as e:
        g.refactor(bad)
    assert e.value.code == 4
    assert rel(g.apply(r), z0) <= 1e-15
    assert rel(g.spmv(r), st.A @ r) <= 1e-14
    g.close()


def test_refactor_needs_the_option(ctx):
    from s2l_b200.capi import GpuSetup, S2LError
    _, st = small_setup("poisson2d")
    g = GpuSetup(ctx, st)
    with pytest.raises(S2LError) as e:
        g.refactor(st.A.data)
    assert e.value.code == 7
    g.close()


def test_refactor_makes_the_coarse_correction_consistent_with_the_new_matrix(ctx):
    """The reference's check of update(Refactorize) (test/test_reuse.cpp:16-19): with Q = W E^-1 W^T,
    W^T (r - A Q r) = 0 for the new A once E is recomputed, and not while the preconditioner is kept
    (Reuse: the operator has the new values, E the old ones)."""
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st, options={"refactor": 1})
    rows, cols, vals = [], [], []
    for i, s in enumerate(st.subdomains):
        l2g = s.l2g()
        for a in range(s.V.shape[1]):
            rows.append(l2g)
            cols.append(np.full(l2g.size, st.offsets[i] + a))
            vals.append(s.V[:, a])
    W = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(st.n, st.n0))
    A2 = _new_values(st, 77, True)
    r = np.random.default_rng(8).standard_normal(st.n)
    scale = np.linalg.norm(W.T @ r)
    g.update_matrix(A2.data)
    stale = np.linalg.norm(W.T @ (r - A2 @ g.coarse_apply(r))) / scale
    g.refactor(A2.data)
    fresh = np.linalg.norm(W.T @ (r - A2 @ g.coarse_apply(r))) / scale
    assert fresh <= 1e-10 and stale > 1e-4, (fresh, stale)
    g.close()


def _permuted(st, sub: int):
    """P_in A_ii Q of subdomain `sub` in the kept pivot order, with the global CSR position of each
    of its entries."""
    s = st.subdomains[sub]
    f = s.factor
    l2g = s.l2g()
    rows, cols = l2g[f.perm_in], l2g[np.argsort(f.perm_out)]
    A = st.A.tocsr()
    pos = sp.csr_matrix((np.arange(A.nnz, dtype=np.float64) + 1.0, A.indices, A.indptr), shape=A.shape)
    P = pos[rows][:, cols].toarray().astype(np.int64) - 1  # -1: not in the pattern
    return P


def _shrink_pivot(st, sub: int, k: int, factor: float):
    """Matrix values with entry (k, k) of P_in A_ii Q of subdomain `sub` multiplied by `factor`."""
    P = _permuted(st, sub)
    assert P[k, k] >= 0
    v = st.A.data.copy()
    v[P[k, k]] *= factor
    return v


@pytest.mark.parametrize("where", ["sparse", "tail"])
def test_refactor_reports_a_small_relative_pivot(ctx, where):
    """LU refactorization keeps the setup's pivot order (the reference's SparseLU pivots again).  A
    pivot that became small against the entries it divides is reported, and the setup is left
    unchanged; with the check off (pivot_tol 0) the same values refactorize.
    sparse: no tail (tail_max 0), the first pivot (column 0 has no updates, its multipliers are
    A(i, 0) / A(0, 0));  tail: one sparse row (tail_rows >= every subdomain), the tail's first pivot
    is entry (1, 1) when A(0, 1) = 0 (no update from column 0), its multipliers are its row."""
    from s2l_b200.capi import GpuSetup, S2LError
    _, st = small_setup("convdiff3d")
    assert st.subdomains[0].factor.kind == "lu"
    if where == "sparse":
        layout, v = {"tail_max": 0}, _shrink_pivot(st, 0, 0, 1e-9)
    else:
        sub = next(i for i in range(st.nsub) if _permuted(st, i)[0, 1] < 0)
        layout, v = {"tail_rows": 4096}, _shrink_pivot(st, sub, 1, 1e-9)
    g = GpuSetup(ctx, st, options=dict(layout, refactor=1))
    r = np.random.default_rng(5).standard_normal(st.n)
    z0 = g.apply(r)
    with pytest.raises(S2LError) as e:
        g.refactor(v)
    assert e.value.code == 4 and "pivot_tol" in str(e.value)
    assert rel(g.apply(r), z0) <= 1e-15
    g.close()
    g = GpuSetup(ctx, st, options=dict(layout, refactor=1, pivot_tol=0.0))
    g.refactor(v)
    g.close()
