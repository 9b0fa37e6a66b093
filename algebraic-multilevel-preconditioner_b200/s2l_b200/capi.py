"""ctypes binding of the C ABI in include/s2l_gpu.h (the library is libs2l_gpu.so, built in-tree).

``GpuSetup`` uploads a host ``Setup`` (setup_phase) once and exposes the solve-phase calls.
There is no CPU fallback: if the library or a CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from .setup_phase import Setup

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(HERE, "lib", "libs2l_gpu.so")

S2L_OK = 0
ERRORS = {1: "BADARG", 2: "OOM", 3: "CUDA", 4: "NUMERIC", 5: "TIMEOUT", 6: "BREAKDOWN", 7: "STATE"}
ONE_LEVEL = {"ras": 0, "asm": 1}
COARSE = {"none": 0, "additive": 1, "deflated": 2}
POU = {"boolean": 0, "multiplicity": 1}
FACTOR = {"lu": 0, "llt": 1, "ldlt": 2}
PTR_HOST, PTR_DEVICE = 0, 1

# every symbol include/s2l_gpu.h declares
EXPORTED = [
    "s2l_gpu_create", "s2l_gpu_destroy", "s2l_gpu_last_error", "s2l_gpu_setup_begin", "s2l_gpu_set_matrix",
    "s2l_gpu_add_subdomain", "s2l_gpu_set_coarse", "s2l_gpu_setup_end", "s2l_gpu_setup_destroy",
    "s2l_gpu_setup_bytes", "s2l_gpu_spmv", "s2l_gpu_local_solve", "s2l_gpu_coarse_apply",
    "s2l_gpu_one_level_apply", "s2l_gpu_apply", "s2l_gpu_gmres", "s2l_gpu_bicgstab", "s2l_gpu_set_stream",
    "s2l_gpu_profile_enable", "s2l_gpu_profile_get", "s2l_gpu_local_solve_bytes", "s2l_gpu_setup_option",
    "s2l_gpu_setup_stat", "s2l_gpu_coarse_apply_noalloc", "s2l_gpu_solve_batch", "s2l_gpu_serve_start",
    "s2l_gpu_submit", "s2l_gpu_poll", "s2l_gpu_wait", "s2l_gpu_cancel", "s2l_gpu_ticket_info",
    "s2l_gpu_ticket_free", "s2l_gpu_apply_block", "s2l_gpu_gmres_block", "s2l_gpu_update_matrix",
    "s2l_gpu_refactor", "s2l_gpu_add_subdomain_amg", "s2l_amg_build", "s2l_amg_rebuild", "s2l_amg_shape",
    "s2l_amg_matrix", "s2l_amg_coarse", "s2l_amg_free", "s2l_gpu_serve_batching",
]
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_CANCELED = 0, 1, 2, 3
ERR_TIMEOUT, ERR_CANCELED = 5, 8


class KrylovOpts(C.Structure):
    _fields_ = [("restart", C.c_int), ("rtol", C.c_double), ("maxit", C.c_int), ("flexible", C.c_int),
                ("strict_true_residual", C.c_int), ("history_cap", C.c_int), ("stop_norm", C.c_int),
                ("atol", C.c_double)]


class Result(C.Structure):
    _fields_ = [("converged", C.c_int), ("breakdown", C.c_int), ("iterations", C.c_int), ("restarts", C.c_int),
                ("rel_residual", C.c_double), ("true_rel_residual", C.c_double), ("history_len", C.c_int),
                ("history", C.POINTER(C.c_double)), ("initial_residual_of", C.c_double),
                ("final_residual_of", C.c_double)]


class S2LError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"s2l_gpu error {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH):
    """Load libs2l_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run algebraic-multilevel-preconditioner_b200/build.py")
    lib = C.CDLL(path)
    vp = C.c_void_p
    i64p = C.POINTER(C.c_int64)
    i32p = C.POINTER(C.c_int32)
    dp = C.POINTER(C.c_double)
    sig = {
        "s2l_gpu_create": ([C.c_int, C.c_size_t, C.POINTER(vp)], C.c_int),
        "s2l_gpu_destroy": ([vp], C.c_int),
        "s2l_gpu_last_error": ([vp], C.c_char_p),
        "s2l_gpu_setup_begin": ([vp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
        "s2l_gpu_set_matrix": ([vp, i64p, i64p, dp], C.c_int),
        "s2l_gpu_add_subdomain": ([vp, C.c_int, C.c_int64, C.c_int, C.c_int, i64p, dp, C.c_int, C.c_int, i32p,
                                   i32p, i64p, i32p, vp, i64p, i32p, vp, vp, C.c_int, dp], C.c_int),
        "s2l_gpu_set_coarse": ([vp, C.c_int64, i64p, dp], C.c_int),
        "s2l_gpu_setup_end": ([vp], C.c_int),
        "s2l_gpu_setup_destroy": ([vp], C.c_int),
        "s2l_gpu_setup_bytes": ([vp, C.POINTER(C.c_size_t)], C.c_int),
        "s2l_gpu_spmv": ([vp, vp, vp, C.c_int], C.c_int),
        "s2l_gpu_local_solve": ([vp, C.c_int, vp, vp, C.c_int], C.c_int),
        "s2l_gpu_coarse_apply": ([vp, vp, vp, C.c_int], C.c_int),
        "s2l_gpu_one_level_apply": ([vp, vp, vp, C.c_int], C.c_int),
        "s2l_gpu_apply": ([vp, vp, vp, C.c_int], C.c_int),
        "s2l_gpu_gmres": ([vp, vp, vp, C.c_int, C.POINTER(KrylovOpts), C.POINTER(Result)], C.c_int),
        "s2l_gpu_bicgstab": ([vp, vp, vp, C.c_int, C.POINTER(KrylovOpts), C.POINTER(Result)], C.c_int),
        "s2l_gpu_set_stream": ([vp, vp], C.c_int),
        "s2l_gpu_profile_enable": ([vp, C.c_int], C.c_int),
        "s2l_gpu_profile_get": ([vp, C.c_char_p, dp, C.POINTER(C.c_long)], C.c_int),
        "s2l_gpu_local_solve_bytes": ([vp, dp], C.c_int),
        "s2l_gpu_setup_option": ([vp, C.c_char_p, C.c_double], C.c_int),
        "s2l_gpu_setup_stat": ([vp, C.c_char_p, dp], C.c_int),
        "s2l_gpu_coarse_apply_noalloc": ([vp, vp, vp], C.c_int),
        "s2l_gpu_solve_batch": ([vp, C.c_int, C.c_int, C.POINTER(vp), C.POINTER(vp), C.c_int, C.POINTER(KrylovOpts),
                                 C.POINTER(Result), C.POINTER(C.c_int)], C.c_int),
        "s2l_gpu_serve_start": ([vp, C.c_int], C.c_int),
        "s2l_gpu_serve_batching": ([vp, C.c_int], C.c_int),
        "s2l_gpu_submit": ([vp, C.c_int, vp, vp, C.c_int, C.POINTER(KrylovOpts), C.POINTER(Result), C.POINTER(vp)],
                           C.c_int),
        "s2l_gpu_poll": ([vp, C.POINTER(C.c_int)], C.c_int),
        "s2l_gpu_wait": ([vp, C.c_double, C.POINTER(C.c_int)], C.c_int),
        "s2l_gpu_cancel": ([vp], C.c_int),
        "s2l_gpu_ticket_info": ([vp, dp, dp, C.POINTER(C.c_char_p)], C.c_int),
        "s2l_gpu_ticket_free": ([vp], C.c_int),
        "s2l_gpu_apply_block": ([vp, C.c_int, vp, vp, C.c_int], C.c_int),
        "s2l_gpu_update_matrix": ([vp, vp, C.c_int], C.c_int),
        "s2l_gpu_refactor": ([vp, vp, C.c_int], C.c_int),
        "s2l_gpu_add_subdomain_amg": ([vp, C.c_int, C.c_int64, C.c_int, C.c_int, vp, vp, C.c_int, C.c_int, vp,
                                       vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int, vp, C.c_int, vp], C.c_int),
        "s2l_gpu_gmres_block": ([vp, C.c_int, vp, vp, C.c_int, C.POINTER(KrylovOpts), C.POINTER(Result)], C.c_int),
        "s2l_amg_build": ([C.c_int64, vp, vp, vp, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
        "s2l_amg_rebuild": ([vp, vp, vp, vp, C.POINTER(vp)], C.c_int),
        "s2l_amg_shape": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int64)], C.c_int),
        "s2l_amg_matrix": ([vp, C.c_int, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(vp),
                            C.POINTER(vp), C.POINTER(vp)], C.c_int),
        "s2l_amg_coarse": ([vp, C.POINTER(vp)], C.c_int),
        "s2l_amg_free": ([vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _vp(a):
    """void* of a numpy array or a device pointer (int)."""
    if isinstance(a, int):
        return C.c_void_p(a)
    return C.c_void_p(a.ctypes.data)


class Context:
    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.s2l_gpu_create(device, hbm_budget, C.byref(h))
        if rc != S2L_OK:
            raise S2LError(rc, "s2l_gpu_create failed (no CUDA device?)")
        self.h = h
        self._setups = weakref.WeakSet()  # closed before the context (a setup must not outlive it)

    def error(self) -> str:
        return self.lib.s2l_gpu_last_error(self.h).decode()

    def check(self, rc):
        if rc != S2L_OK:
            raise S2LError(rc, self.error())

    def serve_start(self, workers: int = 4, batching: int = -1):
        """Start the native worker threads of the asynchronous solves (GpuSetup.submit).  batching:
        slots of the continuous-batching block runners (-1 automatic, 0 off: every GMRES request
        alone on its worker)."""
        self.check(self.lib.s2l_gpu_serve_start(self.h, workers))
        self.serve_batching(batching)

    def serve_batching(self, slots: int):
        self.check(self.lib.s2l_gpu_serve_batching(self.h, slots))

    def close(self):
        if self.h:
            for g in list(self._setups):
                g.close()
            self.lib.s2l_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _result_dict(res: "Result", hist: np.ndarray) -> dict:
    return {"converged": bool(res.converged), "breakdown": bool(res.breakdown), "iterations": res.iterations,
            "restarts": res.restarts, "rel_residual": res.rel_residual, "true_rel_residual": res.true_rel_residual,
            "history": hist[:res.history_len].copy(), "initial_residual_of": res.initial_residual_of,
            "final_residual_of": res.final_residual_of}


class Ticket:
    """An asynchronous solve (s2l_gpu_submit); keeps b, x and the result buffers alive until freed."""

    def __init__(self, setup: "GpuSetup", h, keep):
        self.setup, self.lib, self.h, self._keep = setup, setup.lib, h, keep

    def state(self) -> int:
        v = C.c_int()
        self.setup.ctx.check(self.lib.s2l_gpu_poll(self.h, C.byref(v)))
        return v.value

    def cancel(self):
        self.lib.s2l_gpu_cancel(self.h)

    def wait(self, timeout: float = -1.0):
        """(x, result dict, status) once finished; raises TimeoutError if not finished in time."""
        st = C.c_int()
        rc = self.lib.s2l_gpu_wait(self.h, timeout, C.byref(st))
        if rc == ERR_TIMEOUT:
            raise TimeoutError("solve not finished")
        self.setup.ctx.check(rc)
        x, res, hist = self._keep["x"], self._keep["res"], self._keep["hist"]
        return x, _result_dict(res, hist), st.value

    def info(self) -> dict:
        q, r, e = C.c_double(), C.c_double(), C.c_char_p()
        self.setup.ctx.check(self.lib.s2l_gpu_ticket_info(self.h, C.byref(q), C.byref(r), C.byref(e)))
        return {"queue_ms": q.value, "run_ms": r.value, "error": (e.value or b"").decode()}

    def free(self):
        if self.h is not None and self.lib.s2l_gpu_ticket_free(self.h) == S2L_OK:
            self.h = None

    def __del__(self):
        try:
            if self.h is not None:
                self.cancel()
                self.lib.s2l_gpu_wait(self.h, -1.0, None)
                self.free()
        except Exception:
            pass


class GpuSetup:
    """One matrix's setup on the GPU (the drop-in for the reference's TwoLevelSchwarz + Krylov)."""

    def __init__(self, ctx: Context, st: Setup, one_level=None, coarse=None, pou=None, options=None):
        self.ctx = ctx
        ctx._setups.add(self)
        self.lib = ctx.lib
        self.n = st.n
        self.nsub = st.nsub
        opts = st.opts
        h = C.c_void_p()
        ctx.check(self.lib.s2l_gpu_setup_begin(ctx.h, st.n, st.nsub, ONE_LEVEL[one_level or opts.one_level],
                                                COARSE[coarse or opts.coarse], POU[pou or opts.pou], C.byref(h)))
        self.h = h
        try:
            options = dict(options or {})
            if opts.local_approx == "amg" and opts.local_precision == "single":
                options.setdefault("amg_single", 1)  # the hierarchy's values are floats: V-cycle in float
            for k, v in options.items():
                ctx.check(self.lib.s2l_gpu_setup_option(h, k.encode(), float(v)))
            self._upload(st, coarse or opts.coarse)
        except Exception:
            self.close()
            raise

    def _upload(self, st: Setup, coarse: str):
        lib, ctx = self.lib, self.ctx
        A = st.A
        rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
        ci = np.ascontiguousarray(A.indices, dtype=np.int64)
        av = np.ascontiguousarray(A.data, dtype=np.float64)
        ctx.check(lib.s2l_gpu_set_matrix(self.h, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(av, C.c_double)))
        self.local_sizes = []
        for i, s in enumerate(st.subdomains):
            if getattr(s, "amg", None) is not None:
                ctx.check(self._add_amg(i, s, coarse))
                self.local_sizes.append(s.n_local)
                continue
            f = s.factor
            real = 1 if f.L.dtype == np.float32 else 0
            vt = np.float32 if real else np.float64
            Lrp = np.ascontiguousarray(f.L.indptr, dtype=np.int64)
            Lci = np.ascontiguousarray(f.L.indices, dtype=np.int32)
            Lv = np.ascontiguousarray(f.L.data, dtype=vt)
            if f.kind == "lu":
                Urp = np.ascontiguousarray(f.U.indptr, dtype=np.int64)
                Uci = np.ascontiguousarray(f.U.indices, dtype=np.int32)
                Uv = np.ascontiguousarray(f.U.data, dtype=vt)
                up = (_p(Urp, C.c_int64), _p(Uci, C.c_int32), _vp(Uv))
            else:
                up = (None, None, None)
            d = np.ascontiguousarray(f.d, dtype=vt) if f.kind == "ldlt" else None
            gh = np.ascontiguousarray(s.ghosts, dtype=np.int64)
            D = np.ascontiguousarray(s.D, dtype=np.float64)
            pin = np.ascontiguousarray(f.perm_in, dtype=np.int32)
            pout = np.ascontiguousarray(f.perm_out, dtype=np.int32)
            m = s.V.shape[1] if coarse != "none" else 0
            V = np.asfortranarray(s.V, dtype=np.float64) if m else np.zeros(1)
            rc = lib.s2l_gpu_add_subdomain(self.h, i, int(s.begin), int(s.n_owned), int(gh.size), _p(gh, C.c_int64),
                                           _p(D, C.c_double), FACTOR[f.kind], real, _p(pin, C.c_int32),
                                           _p(pout, C.c_int32), _p(Lrp, C.c_int64), _p(Lci, C.c_int32), _vp(Lv),
                                           *up, _vp(d) if d is not None else None, m, _p(V, C.c_double))
            ctx.check(rc)
            self.local_sizes.append(s.n_local)
        if coarse != "none":
            off = np.ascontiguousarray(st.offsets, dtype=np.int64)
            E = np.ascontiguousarray(st.E, dtype=np.float64)
            if E.size == 0:
                E = np.zeros(1)
            ctx.check(lib.s2l_gpu_set_coarse(self.h, int(st.n0), _p(off, C.c_int64), _p(E, C.c_double)))
        ctx.check(lib.s2l_gpu_setup_end(self.h))

    # ---- helpers
    def _vec(self, x, n):
        if isinstance(x, int):
            return x, PTR_DEVICE
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != n:
            raise ValueError(f"vector of size {x.size}, expected {n}")
        return x, PTR_HOST

    def _call2(self, fn, x, n_in, n_out, out=None):
        xv, kind = self._vec(x, n_in)
        if kind == PTR_DEVICE:
            if out is None or not isinstance(out, int):
                raise ValueError("device input needs a device output pointer")
            self.ctx.check(fn(self.h, C.c_void_p(xv), C.c_void_p(out), PTR_DEVICE))
            return out
        y = np.empty(n_out) if out is None else out
        self.ctx.check(fn(self.h, _vp(xv), _vp(y), PTR_HOST))
        return y

    # ---- solve phase
    def spmv(self, x, out=None):
        return self._call2(self.lib.s2l_gpu_spmv, x, self.n, self.n, out)

    def apply(self, r, out=None):
        return self._call2(self.lib.s2l_gpu_apply, r, self.n, self.n, out)

    def coarse_apply(self, r, out=None):
        return self._call2(self.lib.s2l_gpu_coarse_apply, r, self.n, self.n, out)

    def coarse_apply_noalloc(self, r_dev: int, x0_dev: int):
        """x0 = R0^T E^-1 R0 r with the library's static scratch (device pointers, enqueued on the
        setup's stream; the caller synchronizes)."""
        self.ctx.check(self.lib.s2l_gpu_coarse_apply_noalloc(self.h, C.c_void_p(r_dev), C.c_void_p(x0_dev)))

    def one_level_apply(self, r, out=None):
        return self._call2(self.lib.s2l_gpu_one_level_apply, r, self.n, self.n, out)

    def local_solve(self, i, b):
        n = self.local_sizes[i] if 0 <= i < len(self.local_sizes) else max(1, np.size(b))
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(n)
        self.ctx.check(self.lib.s2l_gpu_local_solve(self.h, i, _vp(b), _vp(x), PTR_HOST))
        return x

    STOP = {"l2": 0, "openfoam": 1}

    def _krylov(self, fn, b, x0, restart, rtol, maxit, flexible, strict, history_cap, device_out=None,
                stop_norm="l2", atol=0.0):
        o = KrylovOpts(restart, rtol, maxit, 1 if flexible else 0, 1 if strict else 0, history_cap,
                       self.STOP[stop_norm], atol)
        hist = np.zeros(max(history_cap, 1))
        res = Result()
        res.history = _p(hist, C.c_double)
        if isinstance(b, int):
            self.ctx.check(fn(self.h, C.c_void_p(b), C.c_void_p(device_out), PTR_DEVICE, C.byref(o), C.byref(res)))
            x = device_out
        else:
            b = np.ascontiguousarray(b, dtype=np.float64)
            if x0 is None:
                x = np.zeros(self.n)
            elif isinstance(x0, np.ndarray) and x0.dtype == np.float64 and x0.flags.c_contiguous and x0.size == self.n:
                x = x0  # used in place (keeps a pinned buffer pinned)
            else:
                x = np.array(x0, dtype=np.float64)
            self.ctx.check(fn(self.h, _vp(b), _vp(x), PTR_HOST, C.byref(o), C.byref(res)))
        out = {"converged": bool(res.converged), "breakdown": bool(res.breakdown), "iterations": res.iterations,
               "restarts": res.restarts, "rel_residual": res.rel_residual,
               "true_rel_residual": res.true_rel_residual, "history": hist[:res.history_len].copy(),
               "initial_residual_of": res.initial_residual_of, "final_residual_of": res.final_residual_of}
        return x, out

    def gmres(self, b, x0=None, restart=30, rtol=1e-8, maxit=1000, flexible=False, strict=False, history_cap=4096,
              device_out=None, stop_norm="l2", atol=0.0):
        return self._krylov(self.lib.s2l_gpu_gmres, b, x0, restart, rtol, maxit, flexible, strict, history_cap,
                            device_out, stop_norm, atol)

    def bicgstab(self, b, x0=None, rtol=1e-8, maxit=1000, strict=False, history_cap=4096, device_out=None,
                 stop_norm="l2", atol=0.0):
        return self._krylov(self.lib.s2l_gpu_bicgstab, b, x0, 1, rtol, maxit, False, strict, history_cap,
                            device_out, stop_norm, atol)

    METHOD = {"gmres": 0, "bicgstab": 1}

    def _opts(self, restart, rtol, maxit, flexible, strict, history_cap, stop_norm, atol):
        return KrylovOpts(restart, rtol, maxit, 1 if flexible else 0, 1 if strict else 0, history_cap,
                          self.STOP[stop_norm], atol)

    def solve_batch(self, bs, method="gmres", restart=30, rtol=1e-8, maxit=1000, flexible=False, strict=False,
                    history_cap=4096, stop_norm="l2", atol=0.0, x0s=None):
        """k solves at once (s2l_gpu_solve_batch) from host vectors: list of (x, result dict, status)."""
        k = len(bs)
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
        xs = [np.zeros(self.n) if x0s is None else np.array(x0s[j], dtype=np.float64) for j in range(k)]
        o = self._opts(restart, rtol, maxit, flexible, strict, history_cap, stop_norm, atol)
        res = (Result * k)()
        hists = [np.zeros(max(history_cap, 1)) for _ in range(k)]
        for j in range(k):
            res[j].history = _p(hists[j], C.c_double)
        pb = (C.c_void_p * k)(*[b.ctypes.data for b in bs])
        px = (C.c_void_p * k)(*[x.ctypes.data for x in xs])
        st = (C.c_int * k)()
        rc = self.lib.s2l_gpu_solve_batch(self.h, self.METHOD[method], k, pb, px, PTR_HOST, C.byref(o), res, st)
        if rc != S2L_OK and all(v == S2L_OK for v in st):
            self.ctx.check(rc)
        return [(xs[j], _result_dict(res[j], hists[j]), st[j]) for j in range(k)]

    def update_matrix(self, values):
        """New values of A (same pattern, renumbered CSR order); the preconditioner is kept."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.ctx.check(self.lib.s2l_gpu_update_matrix(self.h, _vp(v), PTR_HOST))

    def _add_amg(self, i, s, coarse):
        """Subdomain i with its AMG hierarchy (s2l_gpu_add_subdomain_amg)."""
        H = s.amg
        keep = self._keep_amg = getattr(self, "_keep_amg", [])
        nlev = len(H.levels)

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
        gh = arr(s.ghosts, np.int64)
        D = arr(s.D, np.float64)
        m = s.V.shape[1] if coarse != "none" else 0
        V = np.asfortranarray(s.V, dtype=np.float64) if m else np.zeros(1)
        keep.append(V)
        return self.lib.s2l_gpu_add_subdomain_amg(
            self.h, i, int(s.begin), int(s.n_owned), int(gh.size), _vp(gh), _vp(D), nlev, int(H.sweeps), _vp(nrow),
            ptrs(A, "indptr", np.int64), ptrs(A, "indices", np.int32), ptrs(A, "data", np.float64),
            ptrs(P, "indptr", np.int64), ptrs(P, "indices", np.int32), ptrs(P, "data", np.float64),
            ptrs(R, "indptr", np.int64), ptrs(R, "indices", np.int32), ptrs(R, "data", np.float64),
            nc, _vp(Cm) if nc else None, m, _vp(V))

    def refactor(self, values):
        """New values of A (same pattern, renumbered CSR order, host array or a device pointer) and
        the preconditioner refactorized for them on the device (s2l_gpu_refactor; the setup needs
        the option refactor=1)."""
        if isinstance(values, int):
            self.ctx.check(self.lib.s2l_gpu_refactor(self.h, C.c_void_p(values), PTR_DEVICE))
            return
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.ctx.check(self.lib.s2l_gpu_refactor(self.h, _vp(v), PTR_HOST))

    def apply_block(self, R):
        """Z = M^-1 R for the k rows of R (k x n, host), one block call (s2l_gpu_apply_block)."""
        R = np.ascontiguousarray(np.atleast_2d(R), dtype=np.float64)
        Z = np.empty_like(R)
        self.ctx.check(self.lib.s2l_gpu_apply_block(self.h, R.shape[0], _vp(R), _vp(Z), PTR_HOST))
        return Z

    def gmres_block(self, B, X0=None, restart=30, rtol=1e-8, maxit=1000, flexible=False, strict=False,
                    history_cap=4096, device_out=None):
        """k right-hand sides in one lockstep block GMRES (s2l_gpu_gmres_block).

        Host: B is k x n (rows are right-hand sides); returns (X k x n, [result dict per row]).
        Device: B and device_out are device pointers to k * n doubles (pass k=... via B as (ptr, k))."""
        o = self._opts(restart, rtol, maxit, flexible, strict, history_cap, "l2", 0.0)
        if isinstance(B, tuple):  # (device pointer, k)
            ptr, k = B
            res = (Result * k)()
            hists = [np.zeros(max(history_cap, 1)) for _ in range(k)]
            for j in range(k):
                res[j].history = _p(hists[j], C.c_double)
            self.ctx.check(self.lib.s2l_gpu_gmres_block(self.h, k, C.c_void_p(ptr), C.c_void_p(device_out), PTR_DEVICE,
                                                        C.byref(o), res))
            return device_out, [_result_dict(res[j], hists[j]) for j in range(k)]
        B = np.ascontiguousarray(np.atleast_2d(B), dtype=np.float64)
        k = B.shape[0]
        if X0 is None:
            X = np.zeros_like(B)
        elif isinstance(X0, np.ndarray) and X0.dtype == np.float64 and X0.flags.c_contiguous and X0.shape == B.shape:
            X = X0  # used in place (keeps a pinned buffer pinned)
        else:
            X = np.array(X0, dtype=np.float64)
        res = (Result * k)()
        hists = [np.zeros(max(history_cap, 1)) for _ in range(k)]
        for j in range(k):
            res[j].history = _p(hists[j], C.c_double)
        self.ctx.check(self.lib.s2l_gpu_gmres_block(self.h, k, _vp(B), _vp(X), PTR_HOST, C.byref(o), res))
        return X, [_result_dict(res[j], hists[j]) for j in range(k)]

    def submit(self, b, x0=None, method="gmres", restart=30, rtol=1e-8, maxit=1000, flexible=False, strict=False,
               history_cap=4096, stop_norm="l2", atol=0.0) -> Ticket:
        """Queue one solve on the context's worker threads (Context.serve_start) and return at once."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        o = self._opts(restart, rtol, maxit, flexible, strict, history_cap, stop_norm, atol)
        hist = np.zeros(max(history_cap, 1))
        res = Result()
        res.history = _p(hist, C.c_double)
        t = C.c_void_p()
        self.ctx.check(self.lib.s2l_gpu_submit(self.h, self.METHOD[method], _vp(b), _vp(x), PTR_HOST, C.byref(o),
                                               C.byref(res), C.byref(t)))
        return Ticket(self, t, {"b": b, "x": x, "res": res, "hist": hist, "opts": o})

    def set_stream(self, stream_ptr: int | None):
        self.ctx.check(self.lib.s2l_gpu_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def set_option(self, name: str, value: float):
        """A setup option that may change after the upload ("spin_limit", "spin_sleep_ns",
        "sweep_prefetch")."""
        self.ctx.check(self.lib.s2l_gpu_setup_option(self.h, name.encode(), float(value)))

    PROF = {"spmv": 1, "local_solve": 2, "coarse": 4, "combine": 8, "krylov_vec": 16, "all": 31}

    def profile(self, classes=("all",)):
        """Time the given kernel classes with CUDA events (empty: off); resets counters."""
        mask = 0
        for c in classes:
            mask |= self.PROF[c]
        self.ctx.check(self.lib.s2l_gpu_profile_enable(self.h, mask))

    def launches(self) -> int:
        return self.profile_get("launches")[1]

    def profile_get(self, name):
        ms = C.c_double()
        n = C.c_long()
        self.ctx.check(self.lib.s2l_gpu_profile_get(self.h, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def local_solve_bytes(self) -> float:
        b = C.c_double()
        self.ctx.check(self.lib.s2l_gpu_local_solve_bytes(self.h, C.byref(b)))
        return b.value

    def stat(self, name: str) -> float:
        v = C.c_double()
        self.ctx.check(self.lib.s2l_gpu_setup_stat(self.h, name.encode(), C.byref(v)))
        return v.value

    def device_bytes(self) -> int:
        b = C.c_size_t()
        self.ctx.check(self.lib.s2l_gpu_setup_bytes(self.h, C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h:  # never after its context is destroyed (Context.close closes its setups first)
                self.lib.s2l_gpu_setup_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NativeAmg:
    """An AMG hierarchy built by the library on the host (s2l_amg_build / s2l_amg_rebuild: the
    reference's AMGCL setup restated in C++, no device needed)."""
    CODES = {"sa": 0, "rs": 1}

    def __init__(self, h, lib):
        self.h, self.lib = h, lib

    SINGLE = 16  # S2L_AMG_SINGLE

    @classmethod
    def build(cls, A, coarse_enough: int = 500, coarsening: str = "sa", single: bool = False) -> "NativeAmg":
        """single: the setup in single precision (--local-precision single), every value a float."""
        import scipy.sparse as sp
        lib = load()
        A = sp.csr_matrix(A, dtype=np.float64)
        A.sort_indices()
        rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
        ci = np.ascontiguousarray(A.indices, dtype=np.int32)
        v = np.ascontiguousarray(A.data, dtype=np.float64)
        h = C.c_void_p()
        code = cls.CODES[coarsening] | (cls.SINGLE if single else 0)
        rc = lib.s2l_amg_build(A.shape[0], _vp(rp), _vp(ci), _vp(v), int(coarse_enough), code, C.byref(h))
        if rc != S2L_OK:
            raise S2LError(rc, "s2l_amg_build")
        return cls(h, lib)

    def rebuild(self, A) -> "NativeAmg":
        """New values of the same pattern, the transfer operators kept."""
        import scipy.sparse as sp
        A = sp.csr_matrix(A, dtype=np.float64)
        A.sort_indices()
        rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
        ci = np.ascontiguousarray(A.indices, dtype=np.int32)
        v = np.ascontiguousarray(A.data, dtype=np.float64)
        h = C.c_void_p()
        rc = self.lib.s2l_amg_rebuild(self.h, _vp(rp), _vp(ci), _vp(v), C.byref(h))
        if rc != S2L_OK:
            raise S2LError(rc, "s2l_amg_rebuild")
        return NativeAmg(h, self.lib)

    def _matrix(self, level, which):
        import scipy.sparse as sp
        rows, cols = C.c_int64(), C.c_int64()
        rp, ci, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        rc = self.lib.s2l_amg_matrix(self.h, level, which, C.byref(rows), C.byref(cols), C.byref(rp), C.byref(ci),
                                     C.byref(v))
        if rc != S2L_OK:
            raise S2LError(rc, "s2l_amg_matrix")
        if rows.value == 0:
            return None
        n = rows.value
        indptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int64)), (n + 1,)).copy()
        nnz = int(indptr[-1])
        indices = (np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), (nnz,)).copy() if nnz
                   else np.zeros(0, np.int32))
        data = np.ctypeslib.as_array(C.cast(v, C.POINTER(C.c_double)), (nnz,)).copy() if nnz else np.zeros(0)
        return sp.csr_matrix((data, indices, indptr), shape=(n, cols.value))

    def hierarchy(self, sweeps: int = 1):
        """The levels as an s2l_b200.amg.AmgHierarchy (copies)."""
        from .amg import AmgHierarchy, AmgLevel
        nlev, nc = C.c_int(), C.c_int64()
        self.lib.s2l_amg_shape(self.h, C.byref(nlev), C.byref(nc))
        H = AmgHierarchy(sweeps=int(sweeps))
        for l in range(nlev.value):
            H.levels.append(AmgLevel(self._matrix(l, 0), self._matrix(l, 1), self._matrix(l, 2)))
        if nc.value:
            d = C.c_void_p()
            self.lib.s2l_amg_coarse(self.h, C.byref(d))
            H.coarse = np.ctypeslib.as_array(C.cast(d, C.POINTER(C.c_double)), (nc.value, nc.value)).copy()
        return H

    def close(self):
        if self.h:
            self.lib.s2l_amg_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
