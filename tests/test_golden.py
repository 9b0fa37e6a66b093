"""The oracle against the reference's own outputs (golden fixtures from tests/golden/make_golden.py).

With the reference's exact partition, ghost lists, partition of unity, coarse basis and local
factors, the oracle must reproduce: DistributedMatrix::apply (1e-14), LocalSolver::solve (1e-12;
float factors 1e-5), OneLevelSchwarz/CoarseSpace/TwoLevelSchwarz::apply (1e-12; float 1e-5), and
the Krylov solve: identical iteration count (float factors +-1), history and solution.
"""
import numpy as np
import pytest

import golden_fixture as G
from oracle.oracle import OracleSetup

CASES = G.cases()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_fixtures_present():
    assert len(CASES) >= 6


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_reference(case):
    st, applies, kr, local = G.load(case)
    single = st.opts.local_precision == "single"
    tol = 1e-5 if single else 1e-12
    o = OracleSetup(st)
    for i, (b, x) in enumerate(local):
        assert rel(o.local_solve(i, b), x) <= tol
    for a in applies:
        assert rel(o.spmv(a["r"]), a["spmv"]) <= 1e-14
        assert rel(o.one_level_apply(a["r"]), a["one_level"]) <= tol
        if "coarse" in a:
            assert rel(o.coarse_apply(a["r"]), a["coarse"]) <= 1e-12
        assert rel(o.apply(a["r"]), a["z"]) <= tol
    stop = dict(stop_norm=kr["stop_norm"], atol=kr["atol"])
    if kr["method"] == "gmres":
        x, res = o.gmres(st.b, restart=kr["restart"], rtol=kr["rtol"], **stop)
    else:
        x, res = o.bicgstab(st.b, rtol=kr["rtol"], **stop)
    assert res["converged"] == kr["converged"]
    assert abs(res["iterations"] - kr["iterations"]) <= (1 if single else 0)
    if not single:
        n = min(res["history"].size, kr["history"].size)
        assert np.allclose(res["history"][:n], kr["history"][:n], rtol=1e-9, atol=0)
        assert rel(x, kr["x"]) <= 1e-10
    if kr["stop_norm"] == "openfoam":
        # normalised residuals sum|b - A x| / F of x0 and x (include/solver/krylov.hpp:51-52)
        assert abs(res["initial_residual_of"] - kr["initial_residual_of"]) <= 1e-10 * kr["initial_residual_of"]
        assert abs(res["final_residual_of"] - kr["final_residual_of"]) <= 1e-3 * kr["final_residual_of"]
        assert res["final_residual_of"] <= 1.1 * max(kr["rtol"] * res["initial_residual_of"], kr["atol"])
    else:
        assert res["true_rel_residual"] <= 1.1 * kr["rtol"]
