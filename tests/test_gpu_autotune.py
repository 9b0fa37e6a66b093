"""The layout autotuner (s2l_b200.autotune): candidate device layouts of one host setup, timed on the
device, the fastest kept.  Whatever it chooses, the tuned setup must give the reference's results:
the two-level apply against the oracle at 1e-12 (FP64 factors) / 1e-5 (FP32 factors), GMRES to
the FP64 true residual.  Tuned on a uniform and on an uneven partition (sizes within a factor of
about 2.5, like the batching configuration's 10k-25k rows)."""
import numpy as np
import pytest

from conftest import small_setup
from oracle.oracle import OracleSetup

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("case", ["uniform_fp32", "uneven_fp64"])
def test_tuned_layout_keeps_parity(case):
    from s2l_b200 import autotune, capi, workloads as W
    if case == "uniform_fp32":
        w, st = small_setup("bubbles3d", precision="single")
        tol = 1e-5
    else:
        w = W.bubbles3d(18, 8, nbubbles=6, overlap=1)
        w.imbalance = 0.15
        st = W.build(w, workers=1, use_cache=False)
        sizes = np.bincount(st.stats["part"], minlength=w.nsub)
        assert sizes.max() > 1.3 * sizes.min()
        tol = 1e-12
    ctx = capi.Context(0)
    g, rep = autotune.tune(ctx, st, k=4, reps=3)
    assert rep["ms"] <= rep["default_ms"] and rep["gain"] >= 1.0
    assert len(rep["candidates"]) >= 1 + sum(len(v) - 1 for _, v in autotune.SEARCH)
    for name, v in rep["chosen"].items():
        assert name in dict(autotune.SEARCH) and v in dict(autotune.SEARCH)[name]
    o = OracleSetup(st)
    rng = np.random.default_rng(8)
    for _ in range(2):
        r = rng.standard_normal(st.n)
        assert rel(g.apply(r), o.apply(r)) <= tol
    R = rng.uniform(-1.0, 1.0, (4, st.n))
    Z = g.apply_block(R)
    for j in range(4):
        assert rel(Z[j], o.apply(R[j])) <= tol
    flexible = tol > 1e-12
    x, res = g.gmres(st.b, restart=w.restart, rtol=1e-8, flexible=flexible, strict=flexible)
    assert res["converged"] and np.linalg.norm(st.b - st.A @ x) <= 1.1e-8 * np.linalg.norm(st.b)
    o.close()
    g.close()
    ctx.close()
