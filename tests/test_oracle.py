"""The CPU oracle against dense sequential references of the same operators.

Mirrors the reference's own test pattern (test/test_preconditioner.cpp:104-192): the two-level
apply on the same partition is compared with a dense matrix assembled from the global matrix, the
subdomain index sets, D_i and V_i, at 1e-9 there; the oracle must do far better (1e-12).
"""
import os

import numpy as np
import pytest

from conftest import small_setup
from oracle.oracle import OracleSetup

VARIANTS = [(ol, co, pou) for ol in ("ras", "asm") for co in ("additive", "deflated", "none")
            for pou in ("boolean", "multiplicity")]


def dense_apply_operator(st, one_level, coarse):
    n = st.n
    Ad = st.A.toarray()
    M1 = np.zeros((n, n))
    R0 = np.zeros((st.n0, n))
    for i, s in enumerate(st.subdomains):
        l2g = s.l2g()
        inv = np.linalg.inv(Ad[np.ix_(l2g, l2g)])
        M1[np.ix_(l2g, l2g)] += (np.diag(s.D) @ inv) if one_level == "ras" else inv
        if st.n0:
            R0[st.offsets[i]:st.offsets[i + 1], l2g] = s.V.T
    if coarse == "none" or st.n0 == 0:
        return M1
    Q = R0.T @ np.linalg.solve(R0 @ Ad @ R0.T, R0)
    if coarse == "additive":
        return Q + M1
    return Q + M1 @ (np.eye(n) - Ad @ Q)


@pytest.mark.parametrize("one_level,coarse,pou", VARIANTS)
def test_apply_matches_dense_reference(one_level, coarse, pou, rng):
    _, st = small_setup("poisson2d", nx=24, nsub=4, pou=pou, one_level=one_level, coarse=coarse)
    o = OracleSetup(st)
    M = dense_apply_operator(st, one_level, coarse)
    for _ in range(2):
        r = rng.standard_normal(st.n)
        z = o.apply(r)
        zr = M @ r
        assert np.linalg.norm(z - zr) <= 1e-12 * np.linalg.norm(zr)


@pytest.mark.parametrize("name", ["bubbles3d", "convdiff3d"])
def test_apply_3d_matches_dense(name, rng):
    _, st = small_setup(name, nx=10, nsub=4, nbubbles=3) if name == "bubbles3d" else small_setup(name, nx=10, nsub=4)
    o = OracleSetup(st)
    M = dense_apply_operator(st, st.opts.one_level, st.opts.coarse)
    r = rng.standard_normal(st.n)
    zr = M @ r
    assert np.linalg.norm(o.apply(r) - zr) <= 1e-12 * np.linalg.norm(zr)


def test_local_solve_and_spmv(rng):
    _, st = small_setup("bubbles3d", nx=12, nsub=4, nbubbles=4)
    o = OracleSetup(st)
    x = rng.standard_normal(st.n)
    assert np.array_equal(o.spmv(x), st.A @ x) or np.allclose(o.spmv(x), st.A @ x, rtol=1e-15, atol=1e-15)
    for i, s in enumerate(st.subdomains):
        b = rng.standard_normal(s.n_local)
        y = o.local_solve(i, b)
        assert np.linalg.norm(s.Aii @ y - b) <= 1e-12 * np.linalg.norm(b)


@pytest.mark.parametrize("name", ["poisson2d", "bubbles3d", "convdiff3d"])
def test_krylov_converges(name):
    w, st = small_setup(name)
    o = OracleSetup(st)
    x, res = o.gmres(st.b, restart=w.restart, rtol=1e-8)
    assert res["converged"]
    assert np.linalg.norm(st.b - st.A @ x) <= 1.1e-8 * np.linalg.norm(st.b)
    assert res["history"].size == res["iterations"] + 1 + 0 * res["restarts"] or res["restarts"] > 0
    x2, res2 = o.bicgstab(st.b, rtol=1e-8)
    assert res2["converged"]
    assert np.linalg.norm(st.b - st.A @ x2) <= 1.1e-8 * np.linalg.norm(st.b)


def test_gmres_zero_rhs():
    _, st = small_setup("poisson2d")
    o = OracleSetup(st)
    x, res = o.gmres(np.zeros(st.n))
    assert res["converged"] and res["iterations"] == 0 and not np.any(x)


def test_single_precision_factors_flexible_gmres():
    w, st = small_setup("convdiff3d", precision="single")
    o = OracleSetup(st)
    x, res = o.gmres(st.b, restart=w.restart, rtol=1e-8, flexible=True, strict=True)
    assert res["converged"]
    assert np.linalg.norm(st.b - st.A @ x) <= 1e-8 * np.linalg.norm(st.b)


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
def test_openfoam_norm_warm_start(method):
    """OpenFOAM test from x0 != 0: the oracle's normalisation factor is the mean-shifted one of
    src/solver/krylov.cpp:48-58 (the golden fixtures cover x0 = 0), and the final normalised residual
    meets sum|b - A x| <= rtol sum|b - A x0| (include/solver/krylov.hpp:24-34)."""
    w, st = small_setup("bubbles3d")
    o = OracleSetup(st)
    x0 = np.random.default_rng(3).uniform(0.0, 0.2, st.n)
    rs = st.A @ np.ones(st.n)
    xm = x0.mean()
    F = np.abs(st.A @ x0 - xm * rs).sum() + np.abs(st.b - xm * rs).sum() + 1e-20
    kw = dict(rtol=1e-6, stop_norm="openfoam")
    x, res = o.gmres(st.b, x0=x0, restart=w.restart, **kw) if method == "gmres" else o.bicgstab(st.b, x0=x0, **kw)
    r0 = np.abs(st.b - st.A @ x0).sum()
    assert abs(res["initial_residual_of"] - r0 / F) <= 1e-12 * r0 / F
    r1 = np.abs(st.b - st.A @ x).sum()
    assert res["converged"] and r1 <= 1.1e-6 * r0
    assert abs(res["final_residual_of"] - r1 / F) <= 1e-9 * r1 / F


def test_sequence_values_in_setup_order(tmp_path):
    """A Matrix Market sequence step lands in the setup's renumbered CSR order (the reference's
    DomainDecomposer::updateValues), and a changed pattern is refused."""
    import dataclasses
    import scipy.io
    import scipy.sparse as sp
    from s2l_b200 import sequence, workloads as W
    w = W.bubbles3d(10, 4, nbubbles=4)
    st = W.build(w, workers=1, use_cache=False)
    prob = W.make_problem(dataclasses.replace(w, time=2.0))
    scipy.io.mmwrite(str(tmp_path / "p_0002.mtx"), prob.A)
    vals, b = sequence.load_step(str(tmp_path / "p_%04d.mtx"), 2, st)
    n2o = sequence.new_to_old(st)
    expect = prob.A.tocsr()[n2o][:, n2o].tocsr()
    expect.sort_indices()
    assert np.array_equal(vals, expect.data) and b is None
    x = np.random.default_rng(1).standard_normal(st.n)
    A2 = sp.csr_matrix((vals, st.A.indices, st.A.indptr), shape=st.A.shape)
    assert np.allclose(A2 @ x, (prob.A @ x[np.argsort(n2o)])[n2o], rtol=1e-13, atol=1e-12)
    bad = prob.A.tolil()
    bad[0, st.n - 1] = 1.0
    with pytest.raises(sequence.PatternChanged):
        sequence.values_in_setup_order(bad.tocsr(), st)


@pytest.mark.parametrize("name", ["bubbles3d", "convdiff3d", "poisson2d"])
def test_oracle_refactorization_pinned_on_superlu(name):
    """The oracle's refactorization on a kept pattern (LocalSolver::refactorize) reproduces the
    setup's SuperLU factors of the same matrix to rounding, and factorizes a matrix with new
    values of the same pattern exactly (P_in A_ii Q = L U)."""
    import scipy.sparse as sp
    from oracle.oracle import refactor_factor
    _, st = small_setup(name)
    for s in st.subdomains[:3]:
        f = s.factor
        idx = s.l2g()
        Aii = st.A[idx][:, idx]
        g = refactor_factor(f, Aii)
        assert abs(g.L - f.L).max() <= 1e-12 * abs(f.L).max()
        if f.kind == "lu":
            assert abs(g.U - f.U).max() <= 1e-12 * abs(f.U).max()
        d = 1.0 + 0.1 * np.random.default_rng(3).uniform(-1.0, 1.0, Aii.shape[0])
        A2 = (sp.diags(d) @ Aii @ sp.diags(d)).tocsr()
        g2 = refactor_factor(f, A2)
        Ah = A2[f.perm_in][:, np.argsort(f.perm_out)]
        LU = g2.L @ (g2.U if f.kind == "lu" else g2.L.T)
        assert abs(LU - Ah).max() <= 1e-13 * abs(Ah).max()


def test_oracle_refactorization_reports_bad_pivots():
    from oracle.oracle import refactor_factor
    _, st = small_setup("bubbles3d")
    s = st.subdomains[0]
    idx = s.l2g()
    with pytest.raises(ValueError):
        refactor_factor(s.factor, -st.A[idx][:, idx])


AMG_GOLDEN = sorted(f for f in os.listdir(os.path.join(os.path.dirname(__file__), "golden"))
                    if f.startswith("amg_") and not f.startswith(("amg_refactor_", "amg_single_")))
AMG_SINGLE_GOLDEN = sorted(f for f in os.listdir(os.path.join(os.path.dirname(__file__), "golden"))
                           if f.startswith("amg_single_"))
AMG_REFACTOR_GOLDEN = sorted(f for f in os.listdir(os.path.join(os.path.dirname(__file__), "golden"))
                             if f.startswith("amg_refactor_"))


@pytest.mark.parametrize("fixture", AMG_GOLDEN)
def test_amg_hierarchy_and_cycle_pinned_on_the_reference(fixture):
    """The AMG local solver (--local-approx amg): the setup restatement (s2l_b200.amg) plus the
    oracle's V-cycle reproduce the reference's own solve() (AMGCL, run by
    tests/golden/make_amg_golden.py) to rounding, on 1 to 4 levels, 1 or 2 sweeps, smoothed
    aggregation or Ruge-Stuben coarsening (amg_rs_*)."""
    import scipy.sparse as sp
    from oracle.oracle import amg_apply
    from s2l_b200.amg import build_hierarchy
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", fixture))
    n = g["indptr"].size - 1
    A = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    coarsening = str(g["coarsening"]) if "coarsening" in g.files else "sa"
    H = build_hierarchy(A, coarse_enough=int(g["coarse_enough"]), sweeps=int(g["sweeps"]), coarsening=coarsening)
    levels = str(g["info"]).split("[")[1].split(" levels")[0]
    assert len(H.levels) + (H.coarse is not None) == int(levels)
    for v, ref in zip(g["vecs"], g["out"]):
        x = amg_apply(H, v)
        assert np.linalg.norm(x - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("fixture", AMG_SINGLE_GOLDEN)
def test_single_precision_amg_pinned_on_the_reference(fixture):
    """--local-precision single with --local-approx amg: the library's host setup in float
    (s2l_amg_build with S2L_AMG_SINGLE, AMGCL's builtin<float> restated) builds the reference's
    hierarchy (same levels); the oracle's V-cycle on it (FP64 arithmetic on the float values)
    reproduces the reference's float solve() to 1e-5, the tolerance of the FP32 paths."""
    import scipy.sparse as sp
    from oracle.oracle import amg_apply
    from s2l_b200 import capi
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", fixture))
    n = g["indptr"].size - 1
    A = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    N = capi.NativeAmg.build(A, int(g["coarse_enough"]), str(g["coarsening"]), single=True)
    H = N.hierarchy(sweeps=int(g["sweeps"]))
    N.close()
    levels = str(g["info"]).split("[")[1].split(" levels")[0]
    assert len(H.levels) + (H.coarse is not None) == int(levels)
    for lv in H.levels:  # every stored value is a float
        for M in (lv.A, lv.P, lv.R):
            if M is not None:
                assert np.array_equal(M.data, M.data.astype(np.float32).astype(np.float64))
    for v, ref in zip(g["vecs"], g["out"]):
        x = amg_apply(H, v)
        assert np.linalg.norm(x - ref) <= 1e-5 * np.linalg.norm(ref), np.linalg.norm(x - ref) / np.linalg.norm(ref)


@pytest.mark.parametrize("fixture", AMG_REFACTOR_GOLDEN)
def test_amg_refactorization_pinned_on_the_reference(fixture):
    """The reference's refactorize() of its AMG local solver along the moving-bubble sequence: a new
    hierarchy on the new A_ii (build_hierarchy), or with --amg-reuse the kept transfer operators and
    new Galerkin products (rebuild_hierarchy); the oracle's V-cycle on either reproduces the
    reference's solve() after refactorize() to rounding."""
    import scipy.sparse as sp
    from oracle.oracle import amg_apply
    from s2l_b200.amg import build_hierarchy, rebuild_hierarchy
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", fixture))
    n = g["indptr"].size - 1
    A0 = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    A1 = sp.csr_matrix((g["data_next"], g["indices"], g["indptr"]), shape=(n, n))
    ce, sweeps = int(g["coarse_enough"]), int(g["sweeps"])
    H0 = build_hierarchy(A0, coarse_enough=ce, sweeps=sweeps)
    H1 = rebuild_hierarchy(H0, A1) if int(g["reuse"]) else build_hierarchy(A1, coarse_enough=ce, sweeps=sweeps)
    if int(g["reuse"]):
        assert all(a.P is b.P and a.R is b.R for a, b in zip(H0.levels, H1.levels))
    for v, ref in zip(g["vecs"], g["out"]):
        x = amg_apply(H1, v)
        assert np.linalg.norm(x - ref) <= 1e-12 * np.linalg.norm(ref)
    # the other choice gives another operator: the fixture tells them apart
    H2 = build_hierarchy(A1, coarse_enough=ce, sweeps=sweeps) if int(g["reuse"]) else rebuild_hierarchy(H0, A1)
    assert np.linalg.norm(amg_apply(H2, g["vecs"][0]) - g["out"][0]) > 1e-8 * np.linalg.norm(g["out"][0])


def test_amg_rebuild_with_the_same_values_is_the_same_hierarchy():
    import scipy.sparse as sp
    from s2l_b200.amg import build_hierarchy, rebuild_hierarchy
    _, st = small_setup("bubbles3d")
    s = st.subdomains[0]
    idx = s.l2g()
    A = sp.csr_matrix(st.A[idx][:, idx])
    H = build_hierarchy(A, coarse_enough=50)
    H2 = rebuild_hierarchy(H, A)
    assert len(H2.levels) == len(H.levels)
    for a, b in zip(H.levels, H2.levels):
        assert (a.A != b.A).nnz == 0
    assert np.array_equal(H.coarse, H2.coarse)
    with pytest.raises(ValueError):
        rebuild_hierarchy(H, A[:-1, :-1])


@pytest.mark.parametrize("name,kw", [("bubbles3d", {"amg_coarse_enough": 100}),
                                     ("convdiff3d", {"amg_coarse_enough": 50, "amg_sweeps": 2}),
                                     ("poisson2d", {"amg_coarse_enough": 100, "pou": "multiplicity",
                                                    "one_level": "asm", "coarse": "additive"}),
                                     ("bubbles3d", {"amg_coarse_enough": 100, "amg_coarsening": "rs"})])
def test_oracle_two_level_with_amg_local_solves(name, kw):
    """Setups with --local-approx amg: the oracle's local solves are the hierarchy's V-cycle, and
    its GMRES converges with the two-level preconditioner built on them."""
    from oracle.oracle import amg_apply
    w, st = small_setup(name, local_approx="amg", **kw)
    assert all(s.factor is None and s.amg is not None for s in st.subdomains)
    o = OracleSetup(st)
    rng = np.random.default_rng(5)
    for i in (0, st.nsub - 1):
        b = rng.standard_normal(st.subdomains[i].n_local)
        assert np.array_equal(o.local_solve(i, b), amg_apply(st.subdomains[i].amg, b))
    x, r = o.gmres(st.b, restart=w.restart, rtol=1e-8, maxit=2000)
    assert r["converged"]
    assert np.linalg.norm(st.b - st.A @ x) <= 1.1e-8 * np.linalg.norm(st.b)
    o.close()


def test_amg_local_solvers_keep_the_coarse_space():
    """As in the reference (test/test_inexact.cpp:15-18): with --local-approx amg only the local
    solves change; the coarse basis and E are those of the exact-factor setup."""
    _, st = small_setup("bubbles3d")
    _, sa = small_setup("bubbles3d", local_approx="amg", amg_coarse_enough=100)
    assert np.array_equal(st.offsets, sa.offsets)
    for a, b in zip(st.subdomains, sa.subdomains):
        assert np.array_equal(a.V, b.V) and a.factor is not None and b.factor is None and b.amg is not None
    assert np.array_equal(st.E, sa.E)


def test_bubbles_generator_reproduces_the_reference_fixture():
    """The bubbles3d generator (s2l_b200.problems.bubbles, single radius) against the reference's
    own 24^3 fixture (test/gamg/run_gamg_23038420/check_s2l*.mtx: nb=150, R=0.04, rho_ratio=1000,
    cfl=0.5, t=3, seed=2024; tests/golden/make_bubbles_fixture.py): the same pattern, values and
    generated right-hand side to rounding."""
    import hashlib
    from s2l_b200 import problems
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "bubbles3d_24_generator.npz"))
    p = problems.bubbles(3, 24, nbubbles=150, radius=0.04, rho_ratio=1000.0, cfl=0.5, time=3.0, seed=2024)
    A = p.A.tocsr()
    A.sort_indices()
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(A.indptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(A.indices, dtype=np.int64).tobytes())
    assert h.hexdigest() == str(g["pattern_sha256"])
    assert np.abs(A.data - g["data"]).max() <= 1e-13 * np.abs(g["data"]).max()
    assert np.abs(p.rhs_generated - g["rhs"]).max() <= 1e-13 * np.abs(g["rhs"]).max()


@pytest.mark.parametrize("fixture,make", [
    ("laplace2d_ras_additive_lu", lambda P: P.laplace(2, 24)),
    ("laplace2d_asm_deflated_mult", lambda P: P.laplace(2, 20)),
    ("bubbles3d_ras_deflated_llt", lambda P: P.bubbles(3, 12, nbubbles=6, radius=0.15, rho_ratio=1000.0)),
    ("convdiff3d_ras_deflated_lu_single", lambda P: P.convdiff(3, 10)),
])
def test_generators_reproduce_the_reference_golden_matrices(fixture, make):
    """The laplace2d, bubbles3d and convdiff3d generators against the matrices the reference's own generator
    produced for the golden fixtures (tests/golden/make_golden.py), in the fixture's numbering."""
    import scipy.sparse as sp
    from s2l_b200 import problems
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", fixture + ".npz"))
    n = g["global_A_rp"].size - 1
    R = sp.csr_matrix((g["global_A_v"], g["global_A_ci"], g["global_A_rp"]), shape=(n, n))
    n2o = g["global_new_to_old"]
    A = make(problems).A.tocsr()[n2o][:, n2o].tocsr()
    A.sort_indices()
    R.sort_indices()
    assert np.array_equal(A.indptr, R.indptr) and np.array_equal(A.indices, R.indices)
    assert abs(A - R).max() <= 1e-13 * abs(R).max()


def test_coupled_generator_structure():
    """coupled2d (the reference's --generate coupled2d): ncomp unknowns per cell; component c is the
    convection-diffusion operator with viscosity nu (1 + c) plus gamma on the diagonal, coupled to
    component c + 1 (cyclically) by -gamma; with one component it is convdiff2d."""
    import scipy.sparse as sp
    from s2l_b200 import problems
    cpl = problems.convdiff(2, 12, ncomp=3, coupled=True)
    n = 144
    assert cpl.A.shape == (3 * n, 3 * n) and not cpl.symmetric
    A = cpl.A.tocsr()
    gamma = 1.0 * (1.0 / 12) / (1.0 / 12)
    for comp in range(3):
        idx = np.arange(n) * 3 + comp
        block = A[idx][:, idx]
        want = problems.convdiff(2, 12, nu=1.0 + comp).A + gamma * sp.identity(n)
        assert abs(block - want).max() <= 1e-14 * abs(want).max()
        nxt = np.arange(n) * 3 + (comp + 1) % 3
        assert np.allclose(A[idx][:, nxt].toarray(), -gamma * np.eye(n))
    assert abs(problems.convdiff(2, 12, ncomp=1, coupled=True).A - problems.convdiff(2, 12).A).max() == 0.0


def test_convdiff_description_as_the_reference_prints_it():
    """The description line of the reference's generator (src/utils/matrix_generators.cpp:184-191):
    the pulse and the time appear only for a pulsating convection, before (n=..., nnz=...)."""
    from s2l_b200 import problems
    p = problems.convdiff(2, 12, pulse=0.5, time=3.0, pulse_period=10)
    assert p.description.startswith("convdiff2d 12x12 nu=1 pulse=0.5 t=3 (n=144, nnz="), p.description
    q = problems.convdiff(3, 6, ncomp=2, coupled=True)
    assert q.description.startswith("coupled3d 6x6x6 nu=1 ncomp=2 (n=432, nnz="), q.description
    assert "pulse" not in q.description


@pytest.mark.parametrize("kind,extra", [("reference_convdiff2d", {"pulse": 0.5, "pulse_period": 10}),
                                        ("reference_coupled2d", {"ncomp": 2})])
def test_reference_generator_workloads_solve(kind, extra):
    """Workloads on the reference's own generators (nonsymmetric convdiff with a pulsating
    convection, coupled with two unknowns per cell): the setup builds, the unknowns of a cell stay
    in one subdomain, and the oracle's two-level GMRES converges."""
    from s2l_b200 import workloads as W
    w = W.reference_generator(kind, nx=20, nsub=4, **extra)
    st = W.build(w, workers=1, use_cache=False)
    part = st.stats["part"]
    if kind.endswith("coupled2d"):
        assert st.n == 2 * 400 and np.array_equal(part[0::2], part[1::2])
    o = OracleSetup(st)
    x, res = o.gmres(st.b, restart=w.restart, rtol=1e-8)
    assert res["converged"] and np.linalg.norm(st.b - st.A @ x) <= 1.1e-8 * np.linalg.norm(st.b)
    o.close()


def test_setup_with_a_shared_worker_pool_is_the_same_setup():
    """build_setup(pool=...) (one pool of spawned workers for several setups, largest subdomains
    first) gives the setup of the serial path, entry for entry."""
    from s2l_b200 import workloads as W
    from s2l_b200.setup_phase import worker_pool
    w = W.bubbles3d(14, 4, nbubbles=3, overlap=1)
    serial = W.build(w, workers=1, use_cache=False)
    pool = worker_pool(2)
    try:
        pooled = [W.build(w, use_cache=False, pool=pool) for _ in range(2)]
    finally:
        pool.shutdown()
    for st in pooled:
        assert np.array_equal(st.E, serial.E)
        for a, b in zip(st.subdomains, serial.subdomains):
            assert np.array_equal(a.V, b.V)
            assert (a.factor.L != b.factor.L).nnz == 0
            assert np.array_equal(a.factor.perm_in, b.factor.perm_in)
