"""ctypes wrapper of the C oracle (s2l_oracle.c).  TEST INFRASTRUCTURE ONLY.

``OracleSetup`` takes the same host ``Setup`` the GPU library is uploaded from and offers the same
calls as ``s2l_b200.capi.GpuSetup`` (spmv, local_solve, coarse_apply, one_level_apply, apply,
gmres, bicgstab), computed sequentially on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libs2l_oracle.so")

_lib = None


class OResult(C.Structure):
    _fields_ = [("converged", C.c_int), ("breakdown", C.c_int), ("iterations", C.c_int), ("restarts", C.c_int),
                ("rel_residual", C.c_double), ("true_rel_residual", C.c_double),
                ("initial_residual_of", C.c_double), ("final_residual_of", C.c_double), ("history_len", C.c_int),
                ("history", C.POINTER(C.c_double))]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "s2l_oracle.c")):
        build()
    lib = C.CDLL(LIB)
    vp = C.c_void_p
    lib.oracle_setup_create.restype = vp
    lib.oracle_setup_create.argtypes = [C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.oracle_setup_destroy.argtypes = [vp]
    lib.oracle_set_matrix.argtypes = [vp, vp, vp, vp]
    lib.oracle_add_subdomain.argtypes = [vp, C.c_int, C.c_int64, C.c_int, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp,
                                         vp, vp, vp, vp, vp, vp, vp, C.c_int, vp]
    lib.oracle_set_coarse.argtypes = [vp, C.c_int64, vp, vp]
    lib.oracle_set_coarse.restype = C.c_int
    for f in ("oracle_spmv", "oracle_one_level", "oracle_coarse_apply", "oracle_apply"):
        getattr(lib, f).argtypes = [vp, vp, vp]
    lib.oracle_local_solve.argtypes = [vp, C.c_int, vp, vp]
    lib.oracle_gmres.argtypes = [vp, vp, vp, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_double, C.POINTER(OResult)]
    lib.oracle_bicgstab.argtypes = [vp, vp, vp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                    C.POINTER(OResult)]
    lib.oracle_dense_lu.restype = C.c_int
    lib.oracle_dense_lu.argtypes = [C.c_int, vp, vp]
    lib.oracle_amg_apply.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.oracle_add_subdomain_amg.restype = C.c_int
    lib.oracle_add_subdomain_amg.argtypes = [vp, C.c_int, C.c_int64, C.c_int, C.c_int, vp, vp, C.c_int, C.c_int, vp,
                                             vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int, vp, C.c_int, vp]
    lib.oracle_refactor.restype = C.c_int
    lib.oracle_refactor.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    _lib = lib
    return lib


def _a(x):
    return C.c_void_p(x.ctypes.data) if x is not None else None


ONE_LEVEL = {"ras": 0, "asm": 1}
COARSE = {"none": 0, "additive": 1, "deflated": 2}
POU = {"boolean": 0, "multiplicity": 1}
FACTOR = {"lu": 0, "llt": 1, "ldlt": 2}


class OracleSetup:
    def __init__(self, st, one_level=None, coarse=None, pou=None):
        lib = self.lib = load()
        o = st.opts
        coarse = coarse or o.coarse
        self.n = st.n
        self.h = lib.oracle_setup_create(st.n, st.nsub, ONE_LEVEL[one_level or o.one_level], COARSE[coarse],
                                         POU[pou or o.pou])
        self._keep = []
        A = st.A
        rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
        ci = np.ascontiguousarray(A.indices, dtype=np.int64)
        av = np.ascontiguousarray(A.data, dtype=np.float64)
        lib.oracle_set_matrix(self.h, _a(rp), _a(ci), _a(av))
        self.local_sizes = []
        for i, s in enumerate(st.subdomains):
            if getattr(s, "amg", None) is not None:
                self._add_amg(lib, i, s, coarse)
                self.local_sizes.append(s.n_local)
                continue
            f = s.factor
            single = 1 if f.L.dtype == np.float32 else 0
            vt = np.float32 if single else np.float64
            arrs = dict(
                gh=np.ascontiguousarray(s.ghosts, dtype=np.int64), D=np.ascontiguousarray(s.D, dtype=np.float64),
                pin=np.ascontiguousarray(f.perm_in, dtype=np.int32), pout=np.ascontiguousarray(f.perm_out, dtype=np.int32),
                Lp=np.ascontiguousarray(f.L.indptr, dtype=np.int64), Li=np.ascontiguousarray(f.L.indices, dtype=np.int32),
                Lx=np.ascontiguousarray(f.L.data, dtype=vt))
            if f.kind == "lu":
                arrs.update(Up=np.ascontiguousarray(f.U.indptr, dtype=np.int64),
                            Ui=np.ascontiguousarray(f.U.indices, dtype=np.int32),
                            Ux=np.ascontiguousarray(f.U.data, dtype=vt))
            d = np.ascontiguousarray(f.d, dtype=vt) if f.kind == "ldlt" else None
            m = s.V.shape[1] if coarse != "none" else 0
            V = np.asfortranarray(s.V, dtype=np.float64) if m else None
            lib.oracle_add_subdomain(self.h, i, int(s.begin), int(s.n_owned), int(s.ghosts.size), _a(arrs["gh"]),
                                     _a(arrs["D"]), FACTOR[f.kind], single, _a(arrs["pin"]), _a(arrs["pout"]),
                                     _a(arrs["Lp"]), _a(arrs["Li"]), _a(arrs["Lx"]), _a(arrs.get("Up")),
                                     _a(arrs.get("Ui")), _a(arrs.get("Ux")), _a(d), m, _a(V))
            self.local_sizes.append(s.n_local)
        if coarse != "none":
            off = np.ascontiguousarray(st.offsets, dtype=np.int64)
            E = np.ascontiguousarray(st.E, dtype=np.float64) if st.n0 else np.zeros(1)
            if not lib.oracle_set_coarse(self.h, int(st.n0), _a(off), _a(E)):
                raise RuntimeError("oracle: singular coarse matrix")

    def _add_amg(self, lib, i, s, coarse):
        H = s.amg
        nlev = len(H.levels)
        keep = self._keep

        def arr(x, dt):
            a = np.ascontiguousarray(x, dtype=dt)
            keep.append(a)
            return a

        def ptrs(mats, part, dt):
            out = (C.c_void_p * max(nlev, 1))()
            for l, M in enumerate(mats):
                out[l] = arr(getattr(M, part), dt).ctypes.data if M is not None else None
            keep.append(out)
            return C.cast(out, C.c_void_p)

        A = [l.A for l in H.levels]
        P = [l.P for l in H.levels]
        R = [l.R for l in H.levels]
        nrow = arr([M.shape[0] for M in A] or [0], np.int32)
        nc = 0 if H.coarse is None else H.coarse.shape[0]
        Cm = arr(H.coarse if H.coarse is not None else np.zeros(1), np.float64)
        m = s.V.shape[1] if coarse != "none" else 0
        V = arr(np.asfortranarray(s.V).ravel(order="F") if m else np.zeros(1), np.float64)
        ok = lib.oracle_add_subdomain_amg(
            self.h, i, int(s.begin), int(s.n_owned), int(s.ghosts.size), _a(arr(s.ghosts, np.int64)),
            _a(arr(s.D, np.float64)), nlev, int(H.sweeps), _a(nrow),
            ptrs(A, "indptr", np.int64), ptrs(A, "indices", np.int32), ptrs(A, "data", np.float64),
            ptrs(P, "indptr", np.int64), ptrs(P, "indices", np.int32), ptrs(P, "data", np.float64),
            ptrs(R, "indptr", np.int64), ptrs(R, "indices", np.int32), ptrs(R, "data", np.float64),
            nc, _a(Cm) if nc else None, m, _a(V))
        if not ok:
            raise RuntimeError("oracle: singular coarsest AMG level")

    def _v(self, f, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        f(self.h, _a(x), _a(y))
        return y

    def spmv(self, x):
        return self._v(self.lib.oracle_spmv, x)

    def apply(self, r):
        return self._v(self.lib.oracle_apply, r)

    def one_level_apply(self, r):
        return self._v(self.lib.oracle_one_level, r)

    def coarse_apply(self, r):
        return self._v(self.lib.oracle_coarse_apply, r)

    def local_solve(self, i, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.local_sizes[i])
        self.lib.oracle_local_solve(self.h, i, _a(b), _a(x))
        return x

    def _res(self, res, hist):
        return {"converged": bool(res.converged), "breakdown": bool(res.breakdown), "iterations": res.iterations,
                "restarts": res.restarts, "rel_residual": res.rel_residual,
                "true_rel_residual": res.true_rel_residual, "history": hist[:res.history_len].copy(),
                "initial_residual_of": res.initial_residual_of, "final_residual_of": res.final_residual_of}

    STOP = {"l2": 0, "openfoam": 1}

    def gmres(self, b, x0=None, restart=30, rtol=1e-8, maxit=1000, flexible=False, strict=False, history_cap=4096,
              stop_norm="l2", atol=0.0):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        hist = np.zeros(history_cap)
        res = OResult()
        res.history = hist.ctypes.data_as(C.POINTER(C.c_double))
        self.lib.oracle_gmres(self.h, _a(b), _a(x), restart, rtol, maxit, int(flexible), int(strict), history_cap,
                              self.STOP[stop_norm], atol, C.byref(res))
        return x, self._res(res, hist)

    def bicgstab(self, b, x0=None, rtol=1e-8, maxit=1000, strict=False, history_cap=4096, stop_norm="l2", atol=0.0):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        hist = np.zeros(history_cap)
        res = OResult()
        res.history = hist.ctypes.data_as(C.POINTER(C.c_double))
        self.lib.oracle_bicgstab(self.h, _a(b), _a(x), rtol, maxit, int(strict), history_cap, self.STOP[stop_norm],
                                 atol, C.byref(res))
        return x, self._res(res, hist)

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_setup_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refactor_factor(fac, Aii):
    """New factor values for the local matrix Aii on fac's kept pattern and permutations.

    The reference's LocalSolver::refactorize (``src/linalg/local_solver.cpp:111-118``), restated
    by ``oracle_refactor``: LL^T, or LU with the setup's row order (no new pivoting).  The result
    keeps fac's value type.  Raises ValueError on a failed pivot or an entry outside the pattern.
    """
    import scipy.sparse as sp
    from s2l_b200.setup_phase import LocalFactor
    lib = load()
    if fac.kind not in ("lu", "llt"):
        raise ValueError("refactorization supports LU and LL^T factors")
    n = fac.n
    ipout = np.argsort(fac.perm_out)
    Ah = sp.csr_matrix(Aii)[fac.perm_in][:, ipout].tocsc()
    Ah.sort_indices()
    Ap = np.ascontiguousarray(Ah.indptr, dtype=np.int64)
    Ai = np.ascontiguousarray(Ah.indices, dtype=np.int32)
    Ax = np.ascontiguousarray(Ah.data, dtype=np.float64)
    L = fac.L.astype(np.float64).tocsr()
    Lp = np.ascontiguousarray(L.indptr, dtype=np.int64)
    Li = np.ascontiguousarray(L.indices, dtype=np.int32)
    Lx = np.zeros(L.nnz)
    Up = Ui = Ux = None
    if fac.kind == "lu":
        U = fac.U.astype(np.float64).tocsr()
        Up = np.ascontiguousarray(U.indptr, dtype=np.int64)
        Ui = np.ascontiguousarray(U.indices, dtype=np.int32)
        Ux = np.zeros(U.nnz)
    rc = lib.oracle_refactor(n, 0 if fac.kind == "lu" else 1, _a(Ap), _a(Ai), _a(Ax), _a(Lp), _a(Li), _a(Lx),
                             _a(Up), _a(Ui), _a(Ux))
    if rc == -(n + 1):
        raise ValueError("an entry of the local matrix lies outside the factor pattern")
    if rc:
        raise ValueError(f"refactorization: bad pivot in column {-rc - 1}")
    dt = fac.L.dtype
    Ln = sp.csr_matrix((Lx.astype(dt), Li, Lp), shape=(n, n))
    Un = sp.csr_matrix((Ux.astype(dt), Ui, Up), shape=(n, n)) if Ux is not None else None
    return LocalFactor(fac.kind, Ln, Un, fac.perm_in, fac.perm_out)


def refactor_setup(st, A_new):
    """The setup after the reference's Refactorize on the new matrix A_new (renumbered, same pattern).

    Local factors refactorized on their patterns (``refactor_factor``), the coarse basis kept and
    E = W^T A_new W recomputed with it (``CoarseSpace::refresh``,
    ``src/preconditioner/coarse_space.cpp:95-105, 186-206``).
    """
    import dataclasses
    import scipy.sparse as sp
    from s2l_b200.setup_phase import coarse_matrix
    A_new = sp.csr_matrix(A_new)
    subs = []
    for s in st.subdomains:
        idx = s.l2g()
        Aii = A_new[idx][:, idx]
        subs.append(dataclasses.replace(s, factor=refactor_factor(s.factor, Aii), Aii=Aii))
    E = coarse_matrix(A_new, subs, st.offsets) if st.n0 else st.E
    return dataclasses.replace(st, A=A_new, subdomains=subs, E=E)


def amg_apply(H, b):
    """One V-cycle of the AMG hierarchy H (s2l_b200.amg.AmgHierarchy) from x = 0, on the CPU
    (``oracle_amg_apply``: the reference's inexact local solve)."""
    lib = load()
    nlev = len(H.levels)
    keep = []

    def arr(x, dt):
        a = np.ascontiguousarray(x, dtype=dt)
        keep.append(a)
        return a

    def ptrs(mats, part, dt):
        out = (C.c_void_p * max(nlev, 1))()
        for l, M in enumerate(mats):
            if M is None:
                out[l] = None
                continue
            a = arr(getattr(M, part), dt)
            out[l] = a.ctypes.data
        return out

    A = [l.A for l in H.levels]
    P = [l.P for l in H.levels]
    R = [l.R for l in H.levels]
    nc = 0 if H.coarse is None else H.coarse.shape[0]
    nrow = arr([M.shape[0] for M in A] + [nc], np.int32)
    CLU = arr(H.coarse if H.coarse is not None else np.zeros((1, 1)), np.float64).copy()
    keep.append(CLU)
    piv = arr(np.zeros(max(nc, 1)), np.int32)
    if nc and not lib.oracle_dense_lu(nc, _a(CLU), _a(piv)):
        raise ValueError("singular coarse AMG level")
    n = H.n
    b = arr(b, np.float64)
    x = np.zeros(n)
    lib.oracle_amg_apply(nlev, H.sweeps, _a(nrow), ptrs(A, "indptr", np.int64), ptrs(A, "indices", np.int32),
                         ptrs(A, "data", np.float64), ptrs(P, "indptr", np.int64), ptrs(P, "indices", np.int32),
                         ptrs(P, "data", np.float64), ptrs(R, "indptr", np.int64), ptrs(R, "indices", np.int32),
                         ptrs(R, "data", np.float64), _a(CLU), _a(piv), _a(b), _a(x))
    return x
