"""GPU solve phase against the CPU oracle, through the C ABI (libs2l_gpu.so).

Tolerances (FP64 path): SpMV 1e-14 relative (same products, different summation grouping);
local solves, coarse correction, one-level and two-level apply 1e-12 relative; Krylov iteration
counts within +-1 of the oracle and the recomputed FP64 true residual <= rtol (1.1 rtol for the
reference's slack rule).  FP32-factor path: within 1e-5 of the oracle's float solve.
"""
import numpy as np
import pytest

from conftest import small_setup
from oracle.oracle import OracleSetup

pytestmark = pytest.mark.gpu

VARIANTS = [(ol, co, pou) for ol in ("ras", "asm") for co in ("additive", "deflated", "none")
            for pou in ("boolean", "multiplicity")]


@pytest.fixture(scope="module")
def ctx():
    from s2l_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_spmv_matches(ctx, rng):
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st)
    x = rng.standard_normal(st.n)
    assert rel(g.spmv(x), st.A @ x) <= 1e-14
    g.close()


@pytest.mark.parametrize("name", ["poisson2d", "bubbles3d", "convdiff3d"])
def test_local_solves_match(ctx, rng, name):
    from s2l_b200.capi import GpuSetup
    _, st = small_setup(name)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    for i, s in enumerate(st.subdomains):
        b = rng.standard_normal(s.n_local)
        assert rel(g.local_solve(i, b), o.local_solve(i, b)) <= 1e-12
    g.close()


@pytest.mark.parametrize("one_level,coarse,pou", VARIANTS)
def test_apply_matches_oracle(ctx, rng, one_level, coarse, pou):
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("poisson2d", nx=24, nsub=4, pou=pou, one_level=one_level, coarse=coarse)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    for _ in range(2):
        r = rng.standard_normal(st.n)
        assert rel(g.one_level_apply(r), o.one_level_apply(r)) <= 1e-12
        if coarse != "none":
            assert rel(g.coarse_apply(r), o.coarse_apply(r)) <= 1e-12
        assert rel(g.apply(r), o.apply(r)) <= 1e-12
    g.close()


@pytest.mark.parametrize("name", ["bubbles3d", "convdiff3d"])
def test_apply_3d_matches_oracle(ctx, rng, name):
    from s2l_b200.capi import GpuSetup
    _, st = small_setup(name)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    r = rng.standard_normal(st.n)
    assert rel(g.apply(r), o.apply(r)) <= 1e-12
    # the same input twice gives bitwise-identical output (fixed-order kernels)
    assert np.array_equal(g.apply(r), g.apply(r))
    g.close()


@pytest.mark.parametrize("name", ["poisson2d", "bubbles3d", "convdiff3d"])
def test_gmres_matches_oracle(ctx, name):
    from s2l_b200.capi import GpuSetup
    w, st = small_setup(name)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    x, res = g.gmres(st.b, restart=w.restart, rtol=1e-8)
    xo, reso = o.gmres(st.b, restart=w.restart, rtol=1e-8)
    assert res["converged"] and reso["converged"]
    assert abs(res["iterations"] - reso["iterations"]) <= 1
    true = np.linalg.norm(st.b - st.A @ x) / np.linalg.norm(st.b)
    assert true <= 1.1e-8 and abs(true - res["true_rel_residual"]) <= 1e-10
    n = min(res["history"].size, reso["history"].size)
    assert np.allclose(res["history"][:n], reso["history"][:n], rtol=1e-6, atol=1e-13)
    g.close()


@pytest.mark.parametrize("name", ["poisson2d", "bubbles3d"])
def test_bicgstab_matches_oracle(ctx, name):
    from s2l_b200.capi import GpuSetup
    w, st = small_setup(name)
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    x, res = g.bicgstab(st.b, rtol=1e-8)
    xo, reso = o.bicgstab(st.b, rtol=1e-8)
    assert res["converged"] and reso["converged"]
    assert abs(res["iterations"] - reso["iterations"]) <= 2
    assert np.linalg.norm(st.b - st.A @ x) <= 1.1e-8 * np.linalg.norm(st.b)
    g.close()


def _of_residual(st, x, F):
    """OpenFOAM normalised residual sum|b - A x| / F (include/solver/krylov.hpp:24-34)."""
    return np.abs(st.b - st.A @ x).sum() / F


def _of_factor(st, x0):
    """OpenFOAM normalisation factor of x0 (src/solver/krylov.cpp:48-58), in numpy."""
    xm = x0.mean()
    Ax0 = st.A @ x0
    if xm == 0.0:
        return np.abs(Ax0).sum() + np.abs(st.b).sum() + 1e-20
    rs = st.A @ np.ones(st.n)
    return np.abs(Ax0 - xm * rs).sum() + np.abs(st.b - xm * rs).sum() + 1e-20


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
@pytest.mark.parametrize("warm", [False, True])
@pytest.mark.parametrize("rtol,atol", [(1e-6, 0.0), (0.0, 1e-9), (1e-3, 1e-7)])
def test_openfoam_stopping_norm_matches_oracle(ctx, method, warm, rtol, atol):
    """The OpenFOAM test sum|b - A x| <= max(rtol sum|b - A x0|, atol F): GPU and oracle take the
    same number of iterations and report the same normalised residuals; a warm start x0 != 0
    exercises the mean-shifted factor F."""
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    x0 = np.random.default_rng(3).uniform(0.0, 0.2, st.n) if warm else np.zeros(st.n)
    kw = dict(rtol=rtol, stop_norm="openfoam", atol=atol)
    if method == "gmres":
        x, res = g.gmres(st.b, x0=x0.copy(), restart=w.restart, **kw)
        xo, reso = o.gmres(st.b, x0=x0.copy(), restart=w.restart, **kw)
    else:
        x, res = g.bicgstab(st.b, x0=x0.copy(), **kw)
        xo, reso = o.bicgstab(st.b, x0=x0.copy(), **kw)
    assert res["converged"] and reso["converged"]
    assert res["iterations"] == reso["iterations"]
    F = _of_factor(st, x0)
    assert abs(res["initial_residual_of"] - _of_residual(st, x0, F)) <= 1e-10 * res["initial_residual_of"]
    assert abs(res["initial_residual_of"] - reso["initial_residual_of"]) <= 1e-12 * reso["initial_residual_of"]
    fin = _of_residual(st, x, F)
    # the residual sums of the GPU and of numpy differ by rounding (~1e-16 of sum|A x| / F)
    assert abs(res["final_residual_of"] - fin) <= 1e-6 * fin + 1e-14
    assert fin <= 1.1 * max(rtol * res["initial_residual_of"], atol)
    assert rel(x, xo) <= 1e-8
    g.close()


def test_openfoam_x0_already_converged(ctx):
    """No iteration when x0 already satisfies the OpenFOAM test (src/solver/gmres.cpp:52)."""
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st)
    x1, r1 = g.gmres(st.b, restart=w.restart, rtol=1e-10)
    x2, r2 = g.gmres(st.b, x0=x1.copy(), restart=w.restart, rtol=0.0, stop_norm="openfoam", atol=1e-6)
    assert r2["converged"] and r2["iterations"] == 0
    assert np.array_equal(x1, x2)
    g.close()


def test_stop_norm_option_errors(ctx):
    from s2l_b200.capi import GpuSetup, S2LError
    w, st = small_setup("poisson2d")
    g = GpuSetup(ctx, st)
    with pytest.raises(S2LError) as e:
        g.gmres(st.b, atol=1e-6)  # an absolute tolerance needs the OpenFOAM norm
    assert e.value.code == 1 and "OpenFOAM" in str(e.value)
    g.close()


def test_single_precision_factors(ctx, rng):
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("convdiff3d", precision="single")
    g = GpuSetup(ctx, st)
    o = OracleSetup(st)
    for i, s in enumerate(st.subdomains[:3]):
        b = rng.standard_normal(s.n_local)
        assert rel(g.local_solve(i, b), o.local_solve(i, b)) <= 1e-5
    x, res = g.gmres(st.b, restart=w.restart, rtol=1e-8, flexible=True, strict=True)
    xo, reso = o.gmres(st.b, restart=w.restart, rtol=1e-8, flexible=True, strict=True)
    assert res["converged"]
    assert abs(res["iterations"] - reso["iterations"]) <= 2
    assert np.linalg.norm(st.b - st.A @ x) <= 1e-8 * np.linalg.norm(st.b)
    g.close()


def test_device_pointers(ctx, rng):
    import torch
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("bubbles3d")
    g = GpuSetup(ctx, st)
    r = rng.standard_normal(st.n)
    rd = torch.tensor(r, device="cuda", dtype=torch.float64)
    zd = torch.empty_like(rd)
    torch.cuda.synchronize()
    g.apply(rd.data_ptr(), out=zd.data_ptr())
    assert rel(zd.cpu().numpy(), g.apply(r)) == 0.0
    bd = torch.tensor(st.b, device="cuda", dtype=torch.float64)
    xd = torch.zeros_like(bd)
    _, res = g.gmres(bd.data_ptr(), restart=w.restart, device_out=xd.data_ptr())
    x = xd.cpu().numpy()
    assert res["converged"] and np.linalg.norm(st.b - st.A @ x) <= 1.1e-8 * np.linalg.norm(st.b)
    g.close()


def test_bad_arguments_fail_loudly(ctx):
    from s2l_b200 import capi
    _, st = small_setup("poisson2d")
    g = capi.GpuSetup(ctx, st)
    with pytest.raises(ValueError):
        g.apply(np.zeros(st.n + 1))
    with pytest.raises(capi.S2LError):
        g.local_solve(st.nsub + 3, np.zeros(4))
    g.close()


def test_malformed_csr_is_refused_before_it_is_read(ctx):
    """A row pointer that runs past the entries and then back is refused (S2L_ERR_BADARG) before
    any entry is copied, for the matrix and for a factor."""
    import dataclasses
    import types
    from s2l_b200 import capi
    _, st = small_setup("poisson2d")
    rp = st.A.indptr.astype(np.int64).copy()
    rp[1] = rp[-1] + 1000
    bad = types.SimpleNamespace(indptr=rp, indices=st.A.indices, data=st.A.data, shape=st.A.shape)
    with pytest.raises(capi.S2LError) as e:
        capi.GpuSetup(ctx, dataclasses.replace(st, A=bad))
    assert e.value.code == 1 and "monotone" in str(e.value)
    f = st.subdomains[0].factor
    Lrp = f.L.indptr.astype(np.int64).copy()
    Lrp[1] = Lrp[-1] + 1000
    badL = types.SimpleNamespace(indptr=Lrp, indices=f.L.indices, data=f.L.data, dtype=f.L.dtype)
    subs = list(st.subdomains)
    subs[0] = dataclasses.replace(subs[0], factor=dataclasses.replace(f, L=badL))
    with pytest.raises(capi.S2LError) as e:
        capi.GpuSetup(ctx, dataclasses.replace(st, subdomains=subs))
    assert e.value.code == 1 and "monotone" in str(e.value)


def test_hbm_budget_refusal():
    from s2l_b200 import capi
    _, st = small_setup("poisson2d")
    c = capi.Context(0, hbm_budget=1 << 16)
    with pytest.raises(capi.S2LError) as e:
        capi.GpuSetup(c, st)
    assert e.value.code == 2
    c.close()


LAYOUTS = [
    {},
    {"tail_rows": 40},                       # force dense tails on small subdomains
    {"tail_max": 0},                         # no dense tail: the sweeps do all rows
    {"sweep_group": 8, "tail_rows": 17},
    {"sweep_group": 16},
    {"sweep_group": 32, "tail_rows": 3},
    {"chain_block": 1},                      # no chain blocks
    {"chain_block": 2, "sweep_group": 8},
    {"chain_block": 16, "tail_max": 0},      # long chain blocks over the whole factor
    {"chain_block": 16, "tail_rows": 5, "sweep_group": 16},
]


@pytest.mark.parametrize("layout", range(len(LAYOUTS)))
@pytest.mark.parametrize("name", ["poisson2d", "bubbles3d", "convdiff3d"])
def test_layouts_agree_with_oracle(ctx, rng, name, layout):
    """Every device layout of the same factors (dense tail split, sweep group width, chain blocks)
    gives the oracle's local solves and two-level apply to 1e-12."""
    from s2l_b200.capi import GpuSetup
    _, st = small_setup(name)
    opts = LAYOUTS[layout]
    g = GpuSetup(ctx, st, options=opts)
    if opts.get("tail_rows"):
        assert g.stat("tail_rows") == opts["tail_rows"] * st.nsub
    if opts.get("tail_max") == 0:
        assert g.stat("tail_rows") == 0
    if opts.get("chain_block") == 1:
        assert g.stat("chain_blocks") == 0
    o = OracleSetup(st)
    for i, s in enumerate(st.subdomains):
        b = rng.standard_normal(s.n_local)
        assert rel(g.local_solve(i, b), o.local_solve(i, b)) <= 1e-12
    r = rng.standard_normal(st.n)
    assert rel(g.apply(r), o.apply(r)) <= 1e-12
    g.close()


def test_forced_tail_single_precision(ctx, rng):
    from s2l_b200.capi import GpuSetup
    w, st = small_setup("convdiff3d", precision="single")
    g = GpuSetup(ctx, st, options={"tail_rows": 50})
    assert g.stat("tail_rows") > 0
    o = OracleSetup(st)
    for i, s in enumerate(st.subdomains):
        b = rng.standard_normal(s.n_local)
        assert rel(g.local_solve(i, b), o.local_solve(i, b)) <= 1e-5
    g.close()


@pytest.mark.parametrize("tpr", [1, 2, 4, 8, 16, 32])
def test_spmv_lanes_per_row(ctx, rng, tpr):
    """Every lanes-per-row choice of the product with A (1: chunk mode) gives the CSR product
    (1e-14), for one column and for a block of columns."""
    from s2l_b200.capi import GpuSetup
    _, st = small_setup("convdiff3d")
    g = GpuSetup(ctx, st, options={"spmv_tpr": tpr})
    assert g.stat("spmv_tpr") == tpr
    x = rng.standard_normal(st.n)
    assert rel(g.spmv(x), st.A @ x) <= 1e-14
    xs, res = g.gmres(st.b, restart=40, rtol=1e-8)
    assert res["converged"] and np.linalg.norm(st.b - st.A @ xs) <= 1.1e-8 * np.linalg.norm(st.b)
    B = np.random.default_rng(3).uniform(-1.0, 1.0, (4, st.n))
    X, rb = g.gmres_block(B, restart=40, rtol=1e-8)
    assert all(r["converged"] for r in rb)
    for j in range(4):
        assert np.linalg.norm(B[j] - st.A @ X[j]) <= 1.1e-8 * np.linalg.norm(B[j])
    g.close()
