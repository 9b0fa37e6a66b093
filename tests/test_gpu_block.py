"""Block solves: k right-hand sides through one preconditioner / product / orthogonalization per step.

s2l_gpu_apply_block must give, column by column, the single-vector s2l_gpu_apply (1e-12 with FP64
factors; 1e-5 with FP32 factors, as against the oracle), for every k from 1 to 16 and several
layouts.  s2l_gpu_gmres_block runs each column's own GMRES recurrence: iteration counts within +-1
of the single solves and the recomputed FP64 true residual <= rtol (1.1 rtol for the reference's
restart rule).
"""
import numpy as np
import pytest

from conftest import small_setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from s2l_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


CASES = [
    ("bubbles3d", {}, {}),
    ("bubbles3d", {}, {"tail_max": 0}),
    ("bubbles3d", {}, {"tail_rows": 30, "sweep_group": 8}),
    ("poisson2d", {"nx": 24, "nsub": 4, "pou": "multiplicity", "one_level": "asm", "coarse": "additive"}, {}),
    ("poisson2d", {"nx": 24, "nsub": 4, "pou": "multiplicity", "one_level": "ras", "coarse": "deflated"}, {}),
    ("convdiff3d", {}, {"chain_block": 1}),
    ("convdiff3d", {"precision": "single"}, {}),
]


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 16])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_apply_block_matches_single(ctx, case, k):
    from s2l_b200.capi import GpuSetup
    name, kw, layout = CASES[case]
    _, st = small_setup(name, **kw)
    g = GpuSetup(ctx, st, options=layout)
    R = np.random.default_rng(10 + k).standard_normal((k, st.n))
    Z = g.apply_block(R)
    tol = 1e-5 if kw.get("precision") == "single" else 1e-12
    for j in range(k):
        assert rel(Z[j], g.apply(R[j])) <= tol, (j, rel(Z[j], g.apply(R[j])))
    g.close()


@pytest.mark.parametrize("name,k", [("bubbles3d", 4), ("poisson2d", 3), ("convdiff3d", 8)])
def test_gmres_block_matches_single_solves(ctx, name, k):
    from s2l_b200.capi import GpuSetup
    w, st = small_setup(name)
    g = GpuSetup(ctx, st)
    B = np.random.default_rng(21).uniform(-1.0, 1.0, (k, st.n))
    X, res = g.gmres_block(B, restart=w.restart, rtol=1e-8)
    for j in range(k):
        xs, rs = g.gmres(B[j], restart=w.restart, rtol=1e-8)
        assert res[j]["converged"] and rs["converged"]
        assert abs(res[j]["iterations"] - rs["iterations"]) <= 1
        true = np.linalg.norm(B[j] - st.A @ X[j]) / np.linalg.norm(B[j])
        assert true <= 1.1e-8 and abs(true - res[j]["true_rel_residual"]) <= 1e-10
        assert rel(X[j], xs) <= 1e-6
        n = min(res[j]["history"].size, rs["history"].size)
        assert np.allclose(res[j]["history"][:n], rs["history"][:n], rtol=1e-6, atol=1e-13)
    g.close()


def test_gmres_block_mixed_precision_flexible(ctx):
    """FP32 factors, flexible GMRES, converged only at the FP64 true residual <= rtol."""
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("convdiff3d", precision="single")
    g = GpuSetup(ctx, st)
    B = np.random.default_rng(5).uniform(-1.0, 1.0, (5, st.n))
    X, res = g.gmres_block(B, restart=w.restart, rtol=1e-8, flexible=True, strict=True)
    for j in range(5):
        _, rs = g.gmres(B[j], restart=w.restart, rtol=1e-8, flexible=True, strict=True)
        assert res[j]["converged"] and abs(res[j]["iterations"] - rs["iterations"]) <= 2
        assert np.linalg.norm(B[j] - st.A @ X[j]) <= 1e-8 * np.linalg.norm(B[j])
    g.close()


def test_gmres_block_device_pointers_zero_column_and_warm_start(ctx):
    import torch
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st)
    B = np.random.default_rng(6).uniform(-1.0, 1.0, (4, st.n))
    B[2] = 0.0  # a zero right-hand side: x = 0, converged, no iteration
    bd = torch.tensor(B, device="cuda", dtype=torch.float64)
    xd = torch.full_like(bd, 3.0)
    _, res = g.gmres_block((bd.data_ptr(), 4), device_out=xd.data_ptr(), restart=w.restart, rtol=1e-8)
    torch.cuda.synchronize()
    X = xd.cpu().numpy()
    assert res[2]["converged"] and res[2]["iterations"] == 0 and not np.any(X[2])
    for j in (0, 1, 3):
        assert res[j]["converged"]
        assert np.linalg.norm(B[j] - st.A @ X[j]) <= 1.1e-8 * np.linalg.norm(B[j])
    # warm start from the solution: converged at once
    X2, res2 = g.gmres_block(B, X0=X, restart=w.restart, rtol=1e-6)
    assert all(r["converged"] and r["iterations"] == 0 for r in res2)
    g.close()


def test_gmres_block_rejects_bad_arguments(ctx):
    from s2l_b200.capi import GpuSetup, S2LError
    w, st = small_setup("poisson2d")
    g = GpuSetup(ctx, st)
    with pytest.raises(S2LError):
        g.gmres_block(np.ones((17, st.n)))  # more than 16 right-hand sides
    with pytest.raises(S2LError):
        g.gmres_block(np.ones((16, st.n)), restart=100)  # (restart + 1) x 16 coefficients too many
    g.close()


def test_gmres_block_split_into_concurrent_sub_blocks(ctx):
    """k above the block width runs as several blocks at once (here forced to width 2): each
    column still matches its single solve."""
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st, options={"block_width": 2})
    assert g.stat("block_width") == 2
    B = np.random.default_rng(8).uniform(-1.0, 1.0, (7, st.n))
    X, res = g.gmres_block(B, restart=w.restart, rtol=1e-8)
    for j in range(7):
        xs, rs = g.gmres(B[j], restart=w.restart, rtol=1e-8)
        assert res[j]["converged"] and abs(res[j]["iterations"] - rs["iterations"]) <= 1
        assert np.linalg.norm(B[j] - st.A @ X[j]) <= 1.1e-8 * np.linalg.norm(B[j])
        assert rel(X[j], xs) <= 1e-6
    g.close()
