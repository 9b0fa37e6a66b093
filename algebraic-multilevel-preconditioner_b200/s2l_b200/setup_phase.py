"""Setup phase on the host: everything the solve phase uploads to the GPU once per matrix.

In the reference this is its own CPU code, run before the solve: decomposition
(``src/partition/domain_decomposer.cpp``), overlapping subdomains (``src/partition/subdomain.cpp``),
local factorizations (``src/linalg/local_solver.cpp``), the local generalized eigenproblems
(``src/preconditioner/local_eigensolver.cpp``), the coarse basis and E = R0 A R0^T
(``src/preconditioner/coarse_space.cpp``).  The GPU library only consumes its results.  This
module restates that setup with numpy/scipy so the solve phase can be driven stand-alone:

* overlap: the distance-``overlap`` neighbourhood in G(A + A^T) (the reference has distance 1,
  ``subdomain.cpp:163-233``; ``overlap=k`` is the extension the bubbly-pressure workload asks for);
* local numbering [owned (global order) | ghosts (sorted global ids)] (``subdomain.hpp:39-41``);
* lumping sums s(j) = sum_{k not in Omega_i} |A(j,k)| on the ghost rows (``subdomain.cpp:394-411``),
  A~_ii = A_ii - diag(s) (``local_block_splitting.cpp:9-21``);
* partition of unity: boolean or 1/multiplicity (``subdomain.cpp:281-302``);
* local factors: SuperLU (scipy) instead of Eigen SparseLU / SimplicialLLT; a symmetric matrix
  gets L L^T (symmetric minimum-degree ordering, no pivoting), anything else LU with COLAMD;
  ``local_precision='single'`` rounds the factors to float32;
* coarse vectors Z_i from B = D A_ii D and A~_ii with the reference's algorithm
  (``local_eigensolver.cpp:215-423``): kernel by block inverse iteration, (L cap K)^perp_K,
  then the largest-modulus eigenvalues of Pi_K (A~ + sigma I)^{-1} Pi_R B Pi_K (ARPACK here,
  Spectra there), |lambda| >= 1/tau selected, complex pairs split into real and imaginary parts;
* V_i = orth(D_i Z_i) by column-pivoted QR with a relative rank threshold (``coarse_space.cpp:51-75``);
* E = W^T A W with W = [R_1^T V_1, ..., R_N^T V_N] (``coarse_space.cpp:107-206``) and its inverse.
"""
from __future__ import annotations

import hashlib
import os
import pickle
from concurrent.futures import ProcessPoolExecutor
from dataclasses import dataclass, field, asdict
import multiprocessing as mp

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import partition as partmod


@dataclass
class SchwarzOptions:
    """The reference's preconditioner flags (``include/core/config.hpp:61-92``) + overlap."""
    one_level: str = "ras"            # ras | asm
    coarse: str = "deflated"          # deflated | additive | none
    pou: str = "boolean"              # boolean | multiplicity
    overlap: int = 1
    tau: float = 0.6
    nev: int = 300
    eig_tol: float = 1e-8
    eig_maxit: int = 1000
    shift_rel: float = 1e-13
    kernel_tol: float = 1e-8
    kernel_probe: int = 8
    dense_threshold: int = 400
    orth_tol: float = 1e-10
    local_factorization: str = "auto"  # auto | lu | cholesky
    local_precision: str = "double"    # double | single
    local_approx: str = "none"         # none (exact factors) | amg (one AMG V-cycle, --local-approx amg)
    amg_coarse_enough: int = 500       # --amg-coarse-enough: largest coarsest AMG level
    amg_sweeps: int = 1                # --amg-sweeps: Gauss-Seidel steps before / after the coarse correction
    amg_reuse: bool = False            # --amg-reuse: refactorization keeps the transfer operators
    amg_coarsening: str = "sa"         # --amg-coarsening: sa (smoothed aggregation) | rs (Ruge-Stuben)


@dataclass
class LocalFactor:
    """A_ii = P_in^T L U P_out^T in the sense: t = b[perm_in]; L u = t; U v = u; x = v[perm_out].

    kind 'lu': L unit lower (diagonal stored), U upper.  kind 'llt': L lower, U = L^T (not stored).
    kind 'ldlt': L unit lower, d the diagonal, U = diag(d) L^T (not stored).
    All matrices are CSR with sorted column indices; values float64 or float32.
    """
    kind: str
    L: sp.csr_matrix
    U: sp.csr_matrix | None
    perm_in: np.ndarray
    perm_out: np.ndarray
    d: np.ndarray | None = None

    @property
    def n(self) -> int:
        return self.L.shape[0]

    def upper(self) -> sp.csr_matrix:
        if self.kind == "lu":
            return self.U
        if self.kind == "llt":
            return self.L.T.tocsr()
        return (sp.diags(self.d) @ self.L.T).tocsr()

    def nnz(self) -> int:
        """Stored entries of the two triangular factors read by one solve."""
        if self.kind == "lu":
            return int(self.L.nnz + self.U.nnz)
        return int(2 * self.L.nnz)

    def solve(self, b: np.ndarray) -> np.ndarray:
        """Host solve in float64 (setup-time checks only; the solve phase runs on the GPU)."""
        t = np.asarray(b, dtype=np.float64)[self.perm_in]
        L = self.L.astype(np.float64)
        u = spla.spsolve_triangular(L, t, lower=True, unit_diagonal=(self.kind != "llt"))
        v = spla.spsolve_triangular(self.upper().astype(np.float64), u, lower=False)
        return v[self.perm_out]


@dataclass
class SubdomainData:
    """What the solve phase needs of subdomain i (``include/partition/subdomain.hpp:50-136``)."""
    begin: int                 # first owned global row (renumbered ordering)
    n_owned: int               # n_I
    ghosts: np.ndarray         # sorted global ids of Omega_Gamma (int64)
    D: np.ndarray              # partition of unity on Omega_i (n_i)
    factor: LocalFactor | None
    V: np.ndarray              # orthonormal coarse basis on Omega_i (n_i x m_i)
    Aii: sp.csr_matrix | None = None
    amg: object = None         # AMG hierarchy (s2l_b200.amg.AmgHierarchy) when factor is None

    @property
    def n_local(self) -> int:
        return self.n_owned + self.ghosts.size

    def l2g(self) -> np.ndarray:
        return np.concatenate([np.arange(self.begin, self.begin + self.n_owned, dtype=np.int64), self.ghosts])


@dataclass
class Setup:
    """Per-matrix setup of the two-level Schwarz preconditioner."""
    A: sp.csr_matrix           # renumbered global matrix (CSR, sorted columns)
    b: np.ndarray              # renumbered right-hand side
    ownership: np.ndarray      # nsub+1 offsets
    subdomains: list
    offsets: np.ndarray        # coarse offsets, nsub+1
    E: np.ndarray              # n0 x n0 coarse matrix
    opts: SchwarzOptions
    symmetric: bool
    new_to_old: np.ndarray | None = None
    description: str = ""
    stats: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.A.shape[0]

    @property
    def nsub(self) -> int:
        return len(self.subdomains)

    @property
    def n0(self) -> int:
        return int(self.offsets[-1])

    def Einv(self) -> np.ndarray:
        if self.n0 == 0:
            return np.zeros((0, 0))
        return np.linalg.inv(self.E)


# ----------------------------------------------------------------------------- helpers

def norm_estimate(M: sp.spmatrix) -> float:
    """sqrt(||M||_1 ||M||_inf) (``local_eigensolver.cpp:33-44``)."""
    if M.shape[0] == 0:
        return 0.0
    a = abs(M)
    return float(np.sqrt(np.max(np.asarray(a.sum(axis=0)).ravel()) * np.max(np.asarray(a.sum(axis=1)).ravel())))


def _orthonormalize(Y: np.ndarray) -> np.ndarray:
    q, _ = np.linalg.qr(Y)
    return q


def detect_kernel(solve, M: sp.spmatrix, thr: float, probe: int, forced_k: int, seed: int = 20230609) -> np.ndarray:
    """Numerical kernel by block inverse iteration (``local_eigensolver.cpp:64-101``)."""
    n = M.shape[0]
    p = min(max(probe, forced_k + 2), n)
    rng = np.random.default_rng(seed)
    while True:
        Y = _orthonormalize(rng.uniform(-1.0, 1.0, size=(n, p)))
        for _ in range(3):
            Y = _orthonormalize(solve(Y))
        R = M @ Y
        _, s, vh = np.linalg.svd(R, full_matrices=False)
        if forced_k >= 0:
            k = min(forced_k, p)
        else:
            k = int(np.sum(s <= thr))
        if forced_k < 0 and k == p and p < n:
            p = min(2 * p, n)
            continue
        return Y @ vh.T[:, p - k:] if k > 0 else np.zeros((n, 0))


def kernel_complement(B: sp.spmatrix, Q: np.ndarray, thr: float) -> np.ndarray:
    """(L cap K)^perp_K = Q * right singular vectors of B Q with nonzero singular values (``:103-118``)."""
    if Q.shape[1] == 0:
        return np.zeros((Q.shape[0], 0))
    BQ = B @ Q
    # thin SVD: only the right singular vectors (k x k) are used; the full one would also build the
    # n x n left factor (7 GB for a 30k-row subdomain)
    _, s, vh = np.linalg.svd(BQ, full_matrices=False)
    r = int(np.sum(s > thr))
    return Q @ vh.T[:, :r]


def select_eigenvectors(lam: np.ndarray, U: np.ndarray, nmax: int, tau: float):
    """|lambda| >= 1/tau among the first nmax by decreasing modulus; pairs -> Re, Im (``:126-153``)."""
    m = min(nmax, lam.size)
    thr = 1.0 / tau
    out = []
    for j in range(m):
        l = lam[j]
        if abs(l) < thr:
            continue
        if abs(l.imag) <= 1e-10 * abs(l):
            out.append(np.real(U[:, j]))
            continue
        if l.imag < 0.0:
            partner = any(q != j and abs(lam[q] - np.conj(l)) <= 1e-8 * abs(l) for q in range(m))
            if partner:
                continue
        out.append(np.real(U[:, j]))
        out.append(np.imag(U[:, j]))
    return out


def _assemble_Z(Kpart: np.ndarray, ev) -> np.ndarray:
    cols = [Kpart]
    for v in ev:
        nv = np.linalg.norm(v)
        cols.append((v / nv if nv > 0 else v)[:, None])
    return np.hstack(cols) if cols else Kpart


def local_coarse_vectors(Aii: sp.csr_matrix, Atil: sp.csr_matrix, D: np.ndarray, opts: SchwarzOptions,
                         symmetric: bool) -> tuple[np.ndarray, dict]:
    """Z_i of (3.2): [(L cap K)^perp_K | selected eigenvectors] (``local_eigensolver.cpp:215-226``)."""
    n = Aii.shape[0]
    Dm = sp.diags(D)
    B = (Dm @ Aii @ Dm).tocsr()
    nev = max(0, opts.nev)
    ncv = max(2 * nev + 1, nev + 20)
    info = {"n": n}
    if n <= opts.dense_threshold or ncv >= n:
        At = Atil.toarray()
        Bd = B.toarray()
        Uf, s, Vh = np.linalg.svd(At)
        thr = opts.kernel_tol * (s[0] if s.size else 0.0)
        r = int(np.sum(s > thr))
        Q = Vh.T[:, r:]
        Apinv = Vh.T[:, :r] @ np.diag(1.0 / s[:r]) @ Uf[:, :r].T
        Kpart = kernel_complement(B, Q, opts.kernel_tol * norm_estimate(B))
        ev = []
        nev_reg = max(0, opts.nev - Kpart.shape[1])
        if nev_reg > 0:
            T = Apinv @ Bd
            if Q.shape[1] > 0:
                T -= (T @ Q) @ Q.T
            lam, U = np.linalg.eig(T)
            order = np.argsort(-np.abs(lam), kind="stable")
            ev = select_eigenvectors(lam[order], U[:, order], nev_reg, opts.tau)
        info.update(dense=True, kernel_dim=Q.shape[1])
        return _assemble_Z(Kpart, ev), info

    normA = norm_estimate(Atil)
    sigma = opts.shift_rel * (normA if normA > 0 else 1.0)
    F = None
    for _ in range(4):
        try:
            F = spla.splu((Atil + sigma * sp.identity(n)).tocsc(), permc_spec="MMD_AT_PLUS_A")
            break
        except RuntimeError:
            sigma *= 1e3
    if F is None:
        raise RuntimeError("cannot factorize A~_ii + sigma I")
    thr = opts.kernel_tol * normA
    Q = detect_kernel(lambda Y: F.solve(np.asfortranarray(Y)), Atil, thr, opts.kernel_probe, -1)
    if symmetric or Q.shape[1] == 0:
        P = Q
    else:
        P = detect_kernel(lambda Y: F.solve(np.asfortranarray(Y), trans="T"), Atil.T.tocsr(), thr,
                          opts.kernel_probe, Q.shape[1])
    Kpart = kernel_complement(B, Q, opts.kernel_tol * norm_estimate(B))
    nev_reg = min(max(0, opts.nev - Kpart.shape[1]), n - 2)
    ev = []
    if nev_reg > 0:
        def op(x):
            x = np.asarray(x).ravel()
            v = x - Q @ (Q.T @ x) if Q.shape[1] else x
            w = B @ v
            if P.shape[1]:
                w = w - P @ (P.T @ w)
            z = F.solve(w)
            return z - Q @ (Q.T @ z) if Q.shape[1] else z

        T = spla.LinearOperator((n, n), matvec=op, dtype=np.float64)
        k = nev_reg
        ncv_k = min(max(max(2 * k + 1, k + 20), k + 2), n)
        v0 = np.ones(n) + 0.1 * np.sin(np.linspace(-1.0, 1.0, n))
        if Q.shape[1]:
            v0 -= Q @ (Q.T @ v0)
        if k >= n - 1:
            k = n - 2
        lam, U = spla.eigs(T, k=k, which="LM", ncv=ncv_k, tol=opts.eig_tol, maxiter=opts.eig_maxit, v0=v0)
        order = np.argsort(-np.abs(lam), kind="stable")
        ev = select_eigenvectors(lam[order], U[:, order], k, opts.tau)
    info.update(dense=False, kernel_dim=Q.shape[1], shift=sigma)
    return _assemble_Z(Kpart, ev), info


def factorize_local(Aii: sp.csr_matrix, symmetric: bool, request: str, precision: str) -> LocalFactor:
    """Exact factorization of A_ii with SuperLU (the reference uses Eigen, ``local_solver.cpp:95-153``)."""
    n = Aii.shape[0]
    A = Aii.tocsc()
    dt = np.float32 if precision == "single" else np.float64
    if symmetric and request in ("auto", "cholesky", "llt"):
        lu = spla.splu(A, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                       options=dict(SymmetricMode=True))
        dU = lu.U.diagonal()
        if np.array_equal(lu.perm_r, lu.perm_c) and np.all(dU > 0):
            L = (lu.L @ sp.diags(np.sqrt(dU))).tocsr()
            L.sort_indices()
            q = lu.perm_c.astype(np.int64)
            return LocalFactor("llt", L.astype(dt), None, np.argsort(q).astype(np.int32), q.astype(np.int32))
    lu = spla.splu(A, permc_spec="COLAMD")
    L = lu.L.tocsr()
    U = lu.U.tocsr()
    L.sort_indices()
    U.sort_indices()
    return LocalFactor("lu", L.astype(dt), U.astype(dt), np.argsort(lu.perm_r).astype(np.int32),
                       lu.perm_c.astype(np.int32))


def _subdomain_work(args):
    Aii, Atil, D, opts, symmetric, want_coarse = args
    if opts.local_approx == "amg":
        from .amg import build_hierarchy_native
        fac = build_hierarchy_native(Aii, coarse_enough=opts.amg_coarse_enough, sweeps=opts.amg_sweeps,
                                     coarsening=opts.amg_coarsening, single=opts.local_precision == "single")
    else:
        fac = factorize_local(Aii, symmetric, opts.local_factorization, opts.local_precision)
    Z, info = (local_coarse_vectors(Aii, Atil, D, opts, symmetric) if want_coarse
               else (np.zeros((Aii.shape[0], 0)), {}))
    return fac, Z, info


def orth_basis(DZ: np.ndarray, orth_tol: float) -> np.ndarray:
    """V = orth(D Z): column-pivoted Householder QR, rank |r_kk| > tol |r_00| (``coarse_space.cpp:56-63``)."""
    if DZ.shape[1] == 0:
        return np.zeros((DZ.shape[0], 0))
    Qf, R, _ = sla.qr(DZ, mode="economic", pivoting=True)
    d = np.abs(np.diag(R))
    r = int(np.sum(d > orth_tol * d[0])) if d.size and d[0] > 0 else 0
    return np.ascontiguousarray(Qf[:, :r])


# ----------------------------------------------------------------------------- main entry

def build_subdomain_structure(A: sp.csr_matrix, ownership: np.ndarray, overlap: int, pou: str):
    """Ghost lists, local matrices A_ii, lumping sums and D of every subdomain."""
    n = A.shape[0]
    nsub = ownership.size - 1
    S = (A + A.T).tocsr()
    S.sort_indices()
    g2l = np.full(n, -1, dtype=np.int64)
    ghosts_all = []
    for i in range(nsub):
        b, e = int(ownership[i]), int(ownership[i + 1])
        inside = np.arange(b, e, dtype=np.int64)
        frontier = inside
        ghosts = []
        for _ in range(max(1, overlap)):
            rows = S[frontier]
            nb = np.unique(rows.indices.astype(np.int64))
            new = np.setdiff1d(nb, inside, assume_unique=True)
            if new.size == 0:
                break
            ghosts.append(new)
            inside = np.union1d(inside, new)
            frontier = new
        ghosts_all.append(np.sort(np.concatenate(ghosts)) if ghosts else np.zeros(0, dtype=np.int64))
    mult = None
    if pou == "multiplicity":
        mult = np.ones(n)
        for g in ghosts_all:
            mult[g] += 1.0
    out = []
    for i in range(nsub):
        b, e = int(ownership[i]), int(ownership[i + 1])
        nI = e - b
        idx = np.concatenate([np.arange(b, e, dtype=np.int64), ghosts_all[i]])
        g2l[idx] = np.arange(idx.size)
        R = A[idx]
        R.sort_indices()
        lc = g2l[R.indices]
        keep = lc >= 0
        rows = np.repeat(np.arange(idx.size), np.diff(R.indptr))
        Aii = sp.csr_matrix((R.data[keep], (rows[keep], lc[keep])), shape=(idx.size, idx.size))
        Aii.sum_duplicates()
        Aii.sort_indices()
        lump = np.bincount(rows[~keep], weights=np.abs(R.data[~keep]), minlength=idx.size)[nI:]
        g2l[idx] = -1
        if pou == "boolean":
            D = np.zeros(idx.size)
            D[:nI] = 1.0
        else:
            D = 1.0 / mult[idx]
        out.append((b, nI, ghosts_all[i], Aii, lump, D))
    return out


_THREAD_LIMIT = None


def _one_thread_worker():
    """Initializer of a setup worker process: one BLAS / OpenMP thread (the pool's processes are
    the parallelism; a worker may be started at any time, whatever the parent's environment)."""
    global _THREAD_LIMIT
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    try:
        from threadpoolctl import threadpool_limits
        _THREAD_LIMIT = threadpool_limits(limits=1)  # kept: the limit holds while the object lives
    except ImportError:
        pass


def worker_pool(workers: int | None = None, tasks_per_worker: int | None = None) -> ProcessPoolExecutor:
    """A pool of spawned worker processes for the per-subdomain setup work (factorization and
    eigenproblem), one BLAS thread each; pass it to build_setup(pool=...) to set up several matrices
    without starting new processes for each.  With `tasks_per_worker` a worker is replaced after
    that many subdomains (off by default: the workers' memory stays small, about 1.4 GB for 16
    after the 2.1M-row convection-diffusion setup)."""
    return ProcessPoolExecutor(max_workers=workers or os.cpu_count() or 1, mp_context=mp.get_context("spawn"),
                               initializer=_one_thread_worker, max_tasks_per_child=tasks_per_worker)


def build_setup(A_orig: sp.csr_matrix, b_orig: np.ndarray, part: np.ndarray, nsub: int, opts: SchwarzOptions,
                symmetric: bool, workers: int | None = None, description: str = "",
                pool: ProcessPoolExecutor | None = None) -> Setup:
    ownership, n2o, _ = partmod.renumber(part, nsub)
    A = partmod.permute(A_orig.tocsr(), n2o)
    b = np.asarray(b_orig, dtype=np.float64)[n2o]
    struct = build_subdomain_structure(A, ownership, opts.overlap, opts.pou)
    want_coarse = opts.coarse != "none"
    jobs = []
    for (beg, nI, ghosts, Aii, lump, D) in struct:
        Atil = Aii.tolil(copy=True) if False else Aii.copy().tocsr()
        if lump.size:
            d = np.zeros(Aii.shape[0])
            d[nI:] = lump
            Atil = (Atil - sp.diags(d)).tocsr()
            Atil.sort_indices()
        jobs.append((Aii, Atil, D, opts, symmetric, want_coarse))
    if workers is None:
        workers = min(len(jobs), os.cpu_count() or 1)
    if pool is not None and len(jobs) > 1:
        # largest subdomains first, so the last jobs to finish are short ones
        order = sorted(range(len(jobs)), key=lambda i: -jobs[i][0].nnz)
        done = dict(zip(order, pool.map(_subdomain_work, [jobs[i] for i in order], chunksize=1)))
        results = [done[i] for i in range(len(jobs))]
    elif workers > 1 and len(jobs) > 1:
        saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
        for k in saved:
            os.environ[k] = "1"
        try:
            with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
                results = list(ex.map(_subdomain_work, jobs, chunksize=1))
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
    else:
        results = [_subdomain_work(j) for j in jobs]
    subs = []
    ms = []
    infos = []
    for (beg, nI, ghosts, Aii, lump, D), (fac, Z, info) in zip(struct, results):
        V = orth_basis(D[:, None] * Z, opts.orth_tol) if Z.shape[1] else np.zeros((Aii.shape[0], 0))
        if opts.pou == "boolean" and V.shape[1]:
            V[nI:, :] = 0.0
        if opts.local_approx == "amg":
            subs.append(SubdomainData(beg, nI, ghosts, D, None, np.ascontiguousarray(V), Aii, amg=fac))
        else:
            subs.append(SubdomainData(beg, nI, ghosts, D, fac, np.ascontiguousarray(V), Aii))
        ms.append(V.shape[1])
        infos.append(info)
    offsets = np.zeros(nsub + 1, dtype=np.int64)
    np.cumsum(ms, out=offsets[1:])
    E = coarse_matrix(A, subs, offsets) if want_coarse else np.zeros((0, 0))
    st = Setup(A, b, ownership, subs, offsets, E, opts, symmetric, n2o, description)
    st.stats = {"n0": int(offsets[-1]), "m_min": int(min(ms)) if ms else 0, "m_max": int(max(ms)) if ms else 0,
                "nnz_factors": int(sum(s.factor.nnz() if s.factor is not None else s.amg.nnz() for s in subs)),
                "kernel_subdomains": int(sum(1 for i in infos if i.get("kernel_dim", 0) > 0))}
    return st


def coarse_matrix(A: sp.csr_matrix, subs, offsets) -> np.ndarray:
    """E = R0 A R0^T = W^T A W, W(:, off_i + a) = R_i^T V_i(:, a) (``coarse_space.cpp:186-206``)."""
    n = A.shape[0]
    n0 = int(offsets[-1])
    if n0 == 0:
        return np.zeros((0, 0))
    rows, cols, vals = [], [], []
    for i, s in enumerate(subs):
        if s.V.shape[1] == 0:
            continue
        l2g = s.l2g()
        r, c = np.nonzero(s.V)
        rows.append(l2g[r])
        cols.append(offsets[i] + c)
        vals.append(s.V[r, c])
    W = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n0))
    AW = (A @ W).tocsc()
    E = (W.T.tocsr() @ AW).toarray()
    return E


# ----------------------------------------------------------------------------- named workloads

def setup_cache_path(key: dict) -> str | None:
    root = os.environ.get("S2L_CACHE_DIR")
    if not root:
        return None
    h = hashlib.sha1(repr(sorted(key.items())).encode()).hexdigest()[:16]
    return os.path.join(root, f"setup_{h}.pkl")


def cached(key: dict, make):
    """Build with ``make()`` or load a pickled copy from $S2L_CACHE_DIR (setup is deterministic)."""
    path = setup_cache_path(key)
    if path and os.path.exists(path):
        with open(path, "rb") as f:
            return pickle.load(f)
    st = make()
    if path:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "wb") as f:
            pickle.dump(st, f, protocol=pickle.HIGHEST_PROTOCOL)
        os.replace(tmp, path)
    return st


def with_factor_precision(st: Setup, precision: str) -> Setup:
    """Shallow copy of a setup whose local factors are stored in ``precision`` ('single'/'double').

    The factors are rounded from the FP64 factorization (the reference factorizes in float when
    ``--local-precision single``, ``src/linalg/local_solver.cpp:66-84``; rounding an FP64 factor
    is the mixed-precision form used here); everything else is shared.
    """
    import copy
    dt = np.float32 if precision == "single" else np.float64
    out = copy.copy(st)
    out.opts = copy.copy(st.opts)
    out.opts.local_precision = precision
    subs = []
    for s in st.subdomains:
        f = s.factor
        nf = LocalFactor(f.kind, f.L.astype(dt), f.U.astype(dt) if f.U is not None else None, f.perm_in, f.perm_out,
                         f.d.astype(dt) if f.d is not None else None)
        ns = copy.copy(s)
        ns.factor = nf
        subs.append(ns)
    out.subdomains = subs
    return out


def refactor_amg_setup(st: Setup, A_new: sp.csr_matrix) -> Setup:
    """The setup after the reference's Refactorize with AMG local solvers, for new values of A
    (renumbered ordering, same pattern): every subdomain's hierarchy is set up again on its new
    A_ii (``AmgSolver::refactorize``, ``src/linalg/inexact_solver.cpp:77-89``: a new hierarchy, or
    with ``amg_reuse`` the kept transfer operators and new Galerkin products), the coarse basis is
    kept and E = W^T A_new W recomputed with it (``CoarseSpace::refresh``,
    ``src/preconditioner/coarse_space.cpp:95-105, 186-206``)."""
    import copy
    from .amg import build_hierarchy_native, rebuild_hierarchy
    A_new = sp.csr_matrix(A_new, dtype=np.float64)
    A_new.sort_indices()
    if A_new.shape != st.A.shape:
        raise ValueError(f"size changed: {A_new.shape} != {st.A.shape}")
    o = st.opts
    subs = []
    for sd in st.subdomains:
        if sd.amg is None:
            raise ValueError("refactor_amg_setup: a subdomain without an AMG hierarchy")
        idx = sd.l2g()
        Aii = sp.csr_matrix(A_new[idx][:, idx])
        Aii.sort_indices()
        single = o.local_precision == "single"
        if o.amg_reuse:
            H = rebuild_hierarchy(sd.amg, Aii, single=single)
        else:
            H = build_hierarchy_native(Aii, coarse_enough=o.amg_coarse_enough, sweeps=o.amg_sweeps,
                                       coarsening=o.amg_coarsening, single=single)
        ns = copy.copy(sd)
        ns.Aii = Aii
        ns.amg = H
        subs.append(ns)
    out = copy.copy(st)
    out.A = A_new
    out.subdomains = subs
    out.E = coarse_matrix(A_new, subs, st.offsets) if st.n0 else st.E
    out.stats = dict(st.stats)
    out.stats["nnz_factors"] = int(sum(sd.amg.nnz() for sd in subs))
    return out
