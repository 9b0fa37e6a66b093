"""The algorithmic byte model behind bench.py's SpMV and per-solve rooflines (CPU)."""
import importlib.util
import os

import pytest

from conftest import REPO, small_setup


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_spmv_bytes(bench):
    _, st = small_setup("bubbles3d")
    n, nnz = st.n, st.A.nnz
    assert bench.spmv_bytes(st) == nnz * 12 + (n + 1) * 4 + 16 * n
    assert bench.spmv_bytes(st, 4) - bench.spmv_bytes(st) == 3 * 16 * n


def test_gmres_solve_bytes_terms(bench):
    _, st = small_setup("bubbles3d")  # deflated, boolean PoU
    n, n0 = st.n, st.n0
    ls, col = 1.0e6, 2.0e4
    basis = sum(s.n_owned * s.V.shape[1] for s in st.subdomains)
    fixed = (ls - col) + 2 * (st.A.nnz * 12 + (n + 1) * 4) + 2 * 8 * basis + 8 * n0 * n0

    def column(j):
        return col + 16 * n + 24 * n + 24 * n + 24 * n + 2 * (2 * (j + 1) * 8 * n + 16 * n)

    assert bench.gmres_solve_bytes(st, [0], 50, ls, col) == 0.0
    assert bench.gmres_solve_bytes(st, [1], 50, ls, col) == pytest.approx(fixed + column(0))
    assert bench.gmres_solve_bytes(st, [3], 2, ls, col) == pytest.approx(3 * fixed + 2 * column(0) + column(1))
    # two columns: the factors, matrix and basis once per step, the column terms twice; a column
    # that converged earlier stops adding its terms
    assert bench.gmres_solve_bytes(st, [2, 1], 50, ls, col) == pytest.approx(
        2 * fixed + 2 * column(0) + column(1))


def test_gmres_solve_bytes_one_level(bench):
    _, st = small_setup("poisson2d", coarse="none")
    n = st.n
    got = bench.gmres_solve_bytes(st, [1], 30, 5.0e5, 1.0e4)
    want = (5.0e5 - 1.0e4) + st.A.nnz * 12 + (n + 1) * 4 + 1.0e4 + 16 * n + 24 * n + 2 * (16 * n + 16 * n)
    assert got == pytest.approx(want)


def test_secondary_forms_run_within_the_budget(bench):
    """A form runs when its usual time fits in what is left of the run's budget, is skipped (with a
    record) when it does not, and an exception becomes an error record instead of ending the run."""
    assert bench.budgeted("f", 100, lambda: {"x": 1}, 500, 1500) == {"x": 1}
    assert "skipped" in bench.budgeted("f", 100, lambda: {"x": 1}, 50, 1500)

    def boom():
        raise RuntimeError("no room")
    assert bench.budgeted("f", 100, boom, 500, 1500)["error"].startswith("RuntimeError: no room")


def test_serving_mix_child_failure_is_a_record(bench):
    """The serving mix runs in a child process: a child that fails (here: no CUDA device, or any
    other error) gives an error record, the parent carries on."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU would run the whole serving mix")
    a = bench.parse(["--serve-mix", "10", "--budget-s", "600"])
    r = bench.serve_mix_child(a, 0)
    assert "error" in r and "stderr_tail" in r
