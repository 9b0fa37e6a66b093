"""The library's host AMG setup (s2l_amg_build / s2l_amg_rebuild, C++) against the Python
restatement (s2l_b200.amg) and the reference's fixtures.  Host code only: runs without a GPU.

Both restate the reference's AMGCL setup with the same arithmetic in the same order, so every
level must agree bit for bit (patterns and values), for smoothed aggregation and Ruge-Stuben, for
a new hierarchy and for a rebuild with kept transfer operators; the oracle's V-cycle on the native
hierarchy must reproduce the reference's own solve() (tests/golden/amg_*.npz).
"""
import dataclasses
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import small_setup
from s2l_b200 import capi
from s2l_b200.amg import build_hierarchy, rebuild_hierarchy

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def same_hierarchy(H1, H2):
    assert len(H1.levels) == len(H2.levels)
    for a, b in zip(H1.levels, H2.levels):
        for m1, m2 in ((a.A, b.A), (a.P, b.P), (a.R, b.R)):
            assert (m1 is None) == (m2 is None)
            if m1 is None:
                continue
            assert m1.shape == m2.shape
            assert np.array_equal(m1.indptr, m2.indptr) and np.array_equal(m1.indices, m2.indices)
            assert np.array_equal(m1.data, m2.data)
    assert (H1.coarse is None) == (H2.coarse is None)
    if H1.coarse is not None:
        assert np.array_equal(H1.coarse, H2.coarse)


def local_matrices():
    out = []
    for name, i in (("bubbles3d", 0), ("bubbles3d", 5), ("convdiff3d", 1), ("poisson2d", 2)):
        _, st = small_setup(name)
        s = st.subdomains[i]
        idx = s.l2g()
        A = sp.csr_matrix(st.A[idx][:, idx])
        A.sort_indices()
        out.append((f"{name}[{i}]", A))
    return out


@pytest.mark.parametrize("coarsening", ["sa", "rs"])
@pytest.mark.parametrize("coarse_enough", [30, 100, 5000])
def test_native_equals_python(coarsening, coarse_enough):
    for label, A in local_matrices():
        N = capi.NativeAmg.build(A, coarse_enough, coarsening)
        same_hierarchy(N.hierarchy(), build_hierarchy(A, coarse_enough=coarse_enough, coarsening=coarsening))
        N.close()


@pytest.mark.parametrize("coarsening", ["sa", "rs"])
def test_native_rebuild_equals_python(coarsening):
    from s2l_b200 import sequence as seqmod
    from s2l_b200 import workloads as W
    w, st = small_setup("bubbles3d")
    vals, _ = seqmod.values_in_setup_order(W.make_problem(dataclasses.replace(w, time=4.0)).A, st)
    A1g = sp.csr_matrix((vals, st.A.indices, st.A.indptr), shape=st.A.shape)
    for i in (0, 3):
        idx = st.subdomains[i].l2g()
        A0 = sp.csr_matrix(st.A[idx][:, idx])
        A1 = sp.csr_matrix(A1g[idx][:, idx])
        N0 = capi.NativeAmg.build(A0, 50, coarsening)
        N1 = N0.rebuild(A1)
        H0 = build_hierarchy(A0, coarse_enough=50, coarsening=coarsening)
        same_hierarchy(N1.hierarchy(), rebuild_hierarchy(H0, A1))
        with pytest.raises(capi.S2LError):
            N0.rebuild(A1[:-1, :-1])
        N0.close()
        N1.close()


@pytest.mark.parametrize("fixture", sorted(f for f in os.listdir(GOLDEN) if f.startswith("amg_")
                                           and not f.startswith(("amg_refactor_", "amg_single_"))))
def test_native_hierarchy_reproduces_the_reference(fixture):
    from oracle.oracle import amg_apply
    g = np.load(os.path.join(GOLDEN, fixture))
    n = g["indptr"].size - 1
    A = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    coarsening = str(g["coarsening"]) if "coarsening" in g.files else "sa"
    N = capi.NativeAmg.build(A, int(g["coarse_enough"]), coarsening)
    H = N.hierarchy(sweeps=int(g["sweeps"]))
    for v, ref in zip(g["vecs"], g["out"]):
        assert np.linalg.norm(amg_apply(H, v) - ref) <= 1e-12 * np.linalg.norm(ref)
    N.close()


def test_native_refuses_bad_input():
    A = sp.csr_matrix(np.array([[2.0, -1.0], [-1.0, 2.0]]))
    dup = sp.csr_matrix((np.array([1.0, 1.0, -1.0, -1.0, 2.0]), np.array([0, 0, 1, 0, 1]),
                         np.array([0, 3, 5])), shape=(2, 2))  # column 0 twice in row 0
    with pytest.raises(capi.S2LError):
        capi.NativeAmg.build(dup, 1, "sa")
    nan = A.copy()
    nan.data[1] = np.nan
    with pytest.raises(capi.S2LError):
        capi.NativeAmg.build(nan, 1, "rs")
    with pytest.raises(capi.S2LError):
        capi.NativeAmg.build(A, 0, "sa")
    with pytest.raises(KeyError):
        capi.NativeAmg.build(A, 1, "xx")
