"""AMG local solves on the GPU (the reference's --local-approx amg).

Setups whose subdomains carry an AMG hierarchy (s2l_b200.amg, pinned on the reference's AMGCL by
tests/test_oracle.py) instead of factors: the GPU's local solves, one-level and two-level applies
must equal the oracle's (one V-cycle from x = 0 per subdomain, Gauss-Seidel in the serial order)
to 1e-12, GMRES must take the oracle's iterations +-1 and reach the FP64 true residual rtol.
"""
import numpy as np
import pytest

from conftest import small_setup
from oracle.oracle import OracleSetup

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def ctx():
    from s2l_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


CASES = [
    ("bubbles3d", {"amg_coarse_enough": 100}),
    ("bubbles3d", {"amg_coarse_enough": 5000}),  # one coarsest level: the local matrix itself
    ("convdiff3d", {"amg_coarse_enough": 50, "amg_sweeps": 2}),
    ("poisson2d", {"amg_coarse_enough": 100, "pou": "multiplicity", "one_level": "asm", "coarse": "additive"}),
    ("poisson2d", {"amg_coarse_enough": 30, "coarse": "none"}),
    ("bubbles3d", {"amg_coarse_enough": 100, "amg_coarsening": "rs"}),   # Ruge-Stuben levels
    ("convdiff3d", {"amg_coarse_enough": 50, "amg_coarsening": "rs"}),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_amg_local_solves_and_applies_match_oracle(ctx, case):
    from s2l_b200.capi import GpuSetup
    name, kw = CASES[case]
    w, st = small_setup(name, local_approx="amg", **kw)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    rng = np.random.default_rng(60 + case)
    for i in range(st.nsub):
        b = rng.standard_normal(st.subdomains[i].n_local)
        assert rel(g.local_solve(i, b), o.local_solve(i, b)) <= 1e-12, i
    for _ in range(2):  # two calls in a row: the work vectors start clean every time
        r = rng.standard_normal(st.n)
        assert rel(g.one_level_apply(r), o.one_level_apply(r)) <= 1e-12
        assert rel(g.apply(r), o.apply(r)) <= 1e-12
    xg, rg = g.gmres(st.b, restart=w.restart, rtol=1e-8, maxit=2000)
    xo, ro = o.gmres(st.b, restart=w.restart, rtol=1e-8, maxit=2000)
    assert rg["converged"] and ro["converged"]
    assert abs(rg["iterations"] - ro["iterations"]) <= 1
    assert np.linalg.norm(st.b - st.A @ xg) <= 1.1e-8 * np.linalg.norm(st.b)
    o.close()
    g.close()


def test_amg_bicgstab_matches_oracle(ctx):
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d", local_approx="amg", amg_coarse_enough=100)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    xg, rg = g.bicgstab(st.b, rtol=1e-8, maxit=2000)
    _, ro = o.bicgstab(st.b, rtol=1e-8, maxit=2000)
    assert rg["converged"] and abs(rg["iterations"] - ro["iterations"]) <= 1
    assert np.linalg.norm(st.b - st.A @ xg) <= 1.1e-8 * np.linalg.norm(st.b)
    o.close()
    g.close()


def test_amg_setups_refuse_block_calls_and_refactor(ctx):
    from s2l_b200.capi import GpuSetup, S2LError
    _, st = small_setup("bubbles3d", local_approx="amg", amg_coarse_enough=100)
    g = GpuSetup(ctx, st)
    with pytest.raises(S2LError) as e:
        g.apply_block(np.ones((2, st.n)))
    assert e.value.code == 1
    g.close()
    with pytest.raises(S2LError) as e:
        GpuSetup(ctx, st, options={"refactor": 1})
    assert e.value.code == 1


@pytest.mark.parametrize("coarsening", ["sa", "rs"])
def test_amg_local_solve_is_a_fixed_linear_operator(ctx, coarsening):
    """As the reference requires of its AMG local solver (test/test_inexact.cpp:6-9, for plain
    GMRES): B(b1 + 2 b2) = B b1 + 2 B b2 to rounding, and the same right-hand side twice gives
    bitwise-identical results, for the local solves and the two-level apply."""
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("bubbles3d", local_approx="amg", amg_coarse_enough=100, amg_coarsening=coarsening)
    g = GpuSetup(ctx, st)
    rng = np.random.default_rng(77)
    for i in (0, st.nsub - 1):
        n = st.subdomains[i].n_local
        b1, b2 = rng.standard_normal(n), rng.standard_normal(n)
        y1, y2, y12 = g.local_solve(i, b1), g.local_solve(i, b2), g.local_solve(i, b1 + 2.0 * b2)
        assert rel(y12, y1 + 2.0 * y2) <= 1e-13
        assert np.array_equal(g.local_solve(i, b1), y1)
    r = rng.standard_normal(st.n)
    assert np.array_equal(g.apply(r), g.apply(r))
    g.close()


SINGLE_CASES = [
    ("bubbles3d", {"amg_coarse_enough": 100}),
    ("convdiff3d", {"amg_coarse_enough": 50, "amg_coarsening": "rs"}),
    ("poisson2d", {"amg_coarse_enough": 30, "amg_sweeps": 2}),
]


@pytest.mark.parametrize("case", range(len(SINGLE_CASES)))
def test_single_precision_amg_matches_oracle(ctx, case):
    """--local-approx amg with --local-precision single: the hierarchy built in float by the host
    setup (pinned on the reference's AMGCL<float> in tests/test_oracle.py), the V-cycle on the
    device in float.  Local solves and the two-level apply against the oracle's FP64 V-cycle on the
    same float hierarchy at 1e-5 (the FP32 tolerance); flexible GMRES in FP64 reaches the FP64 true
    residual rtol, converged only at the recomputed residual, within +-3 iterations of the oracle."""
    from s2l_b200.capi import GpuSetup
    name, kw = SINGLE_CASES[case]
    w, st = small_setup(name, local_approx="amg", precision="single", **kw)
    assert st.opts.local_precision == "single"
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    rng = np.random.default_rng(90 + case)
    for i in range(st.nsub):
        b = rng.standard_normal(st.subdomains[i].n_local)
        assert rel(g.local_solve(i, b), o.local_solve(i, b)) <= 1e-5, i
    r = rng.standard_normal(st.n)
    assert rel(g.apply(r), o.apply(r)) <= 1e-5
    xg, rg = g.gmres(st.b, restart=w.restart, rtol=1e-8, maxit=2000, flexible=True, strict=True)
    _, ro = o.gmres(st.b, restart=w.restart, rtol=1e-8, maxit=2000, flexible=True, strict=True)
    assert rg["converged"] and abs(rg["iterations"] - ro["iterations"]) <= 3
    assert np.linalg.norm(st.b - st.A @ xg) <= 1e-8 * np.linalg.norm(st.b)
    o.close()
    g.close()
