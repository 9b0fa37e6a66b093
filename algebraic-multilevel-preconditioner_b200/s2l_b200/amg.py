"""AMG hierarchy of a local matrix: the inexact local solver of the reference (``--local-approx amg``).

The reference approximates A_ii^-1 by one V-cycle of AMGCL (``src/linalg/inexact_solver.cpp:45-178``:
``amgcl::amg`` with the builtin backend, smoothed aggregation, Gauss-Seidel smoothing, one cycle
from x = 0 per application, coarsest level at most ``coarse_enough`` unknowns solved directly).
AMGCL (MIT licence, vendored with the reference under ``external/amgcl``) is third-party code; this
module restates its published setup algorithm for the configuration the reference builds:

* strength of connection (``coarsening/plain_aggregates.hpp``): off-diagonal a_ij is strong when
  eps^2 a_ii a_jj < a_ij^2, eps = 0.08 (a float) on the finest level, halved on every coarser one
  (``coarsening/smoothed_aggregation.hpp``);
* plain aggregation, in row order: an unaggregated row with strong connections starts an
  aggregate with its strong neighbours (taking them from earlier aggregates too), then the
  unaggregated strong neighbours of those neighbours; rows without strong connections belong to
  no aggregate; empty aggregates are squeezed out;
* tentative prolongation P0(i, aggregate(i)) = 1;
* smoothing P = (I - omega D_F^-1 A_F) P0 with omega = 2/3 and the filtered matrix A_F (weak
  off-diagonal entries added to the diagonal): P(i, :) = sum over the strong and diagonal entries
  of row i, in column order, of ((1 - omega) on the diagonal, -omega a_ij / d_F(i) elsewhere) P0(j, :);
* R = P^T, coarse operator R (A P) by row-wise sparse products (``coarsening/detail/galerkin.hpp``,
  ``detail/spgemm.hpp``: Saad's algorithm, the accumulation order of scipy's product too);
* levels are added while a level has more than ``coarse_enough`` rows; the last one is solved
  directly (AMGCL's skyline LU; any exact solve agrees to rounding).

With ``--amg-coarsening rs`` the levels come from AMGCL's classic Ruge-Stuben coarsening
(``coarsening/ruge_stuben.hpp``, default parameters): negative strong couplings
(eps_str = 0.25), C/F splitting by decreasing measure in AMGCL's bucket order, direct
interpolation with truncation (eps_tr = 0.2) and rescaling, R = P^T, the same Galerkin product.

The cycle itself (Gauss-Seidel, residual, restriction, coarse correction) is applied by the solve
phase; its CPU restatement is the oracle's ``oracle_amg_apply``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

EPS_STRONG = np.float32(0.08)
OMEGA = 1.0 * (2.0 / 3.0)  # relax (1) times 2/3: no spectral-radius estimate in the reference's setup


@dataclass
class AmgLevel:
    A: sp.csr_matrix                  # operator of the level (sorted columns)
    P: sp.csr_matrix | None = None    # prolongation from the next level (rows of this level)
    R: sp.csr_matrix | None = None    # restriction to the next level


@dataclass
class AmgHierarchy:
    levels: list = field(default_factory=list)
    coarse: np.ndarray | None = None  # the coarsest operator, dense, solved directly (None: smoothed only)
    sweeps: int = 1

    @property
    def n(self) -> int:
        return self.levels[0].A.shape[0] if self.levels else self.coarse.shape[0]

    def nnz(self) -> int:
        """Stored entries of every operator and transfer matrix (what one V-cycle reads)."""
        t = 0
        for l in self.levels:
            t += l.A.nnz + (l.P.nnz + l.R.nnz if l.P is not None else 0)
        if self.coarse is not None:
            t += self.coarse.size
        return int(t)


def _sorted_csr(M) -> sp.csr_matrix:
    M = sp.csr_matrix(M)
    M.sort_indices()
    return M


def _aggregates(A: sp.csr_matrix, eps: np.float32):
    """Strong connections (per stored entry) and aggregate ids (-2: none) and their count."""
    n = A.shape[0]
    rp, ci, va = A.indptr, A.indices, A.data
    dia = A.diagonal()
    eps2 = float(np.float32(eps) * np.float32(eps))  # the product of two floats, in float
    rows = np.repeat(np.arange(n), np.diff(rp))
    strong = (ci != rows) & ((eps2 * dia[rows]) * dia[ci] < va * va)
    UNDEF, REMOVED = -1, -2
    has_strong = np.add.reduceat(strong.astype(np.int64), rp[:-1]) if n else np.zeros(0, np.int64)
    has_strong[np.diff(rp) == 0] = 0
    aid = np.where(has_strong > 0, UNDEF, REMOVED).astype(np.int64)
    count = 0
    rp_l, ci_l, st_l = rp.tolist(), ci.tolist(), strong.tolist()
    aid_l = aid.tolist()
    for i in range(n):
        if aid_l[i] != UNDEF:
            continue
        cur = count
        count += 1
        aid_l[i] = cur
        neib = []
        for j in range(rp_l[i], rp_l[i + 1]):
            c = ci_l[j]
            if st_l[j] and aid_l[c] != REMOVED:
                aid_l[c] = cur
                neib.append(c)
        for c in neib:
            for j in range(rp_l[c], rp_l[c + 1]):
                cc = ci_l[j]
                if st_l[j] and aid_l[cc] == UNDEF:
                    aid_l[cc] = cur
    aid = np.asarray(aid_l, dtype=np.int64)
    if count == 0:
        return strong, aid, 0
    used = np.zeros(count, dtype=np.int64)
    used[aid[aid >= 0]] = 1
    cs = np.cumsum(used)
    if cs[-1] < count:  # aggregates emptied by later ones: renumber without gaps
        aid = np.where(aid >= 0, cs[np.maximum(aid, 0)] - 1, aid)
        count = int(cs[-1])
    return strong, aid, count


def _transfer(A: sp.csr_matrix, eps: np.float32):
    """(P, R) of one level, or None when no row has a strong connection."""
    n = A.shape[0]
    strong, aid, count = _aggregates(A, eps)
    if count == 0:
        return None
    rp, ci, va = A.indptr, A.indices, A.data
    rows = np.repeat(np.arange(n), np.diff(rp))
    keep = (ci == rows) | strong                      # entries of the filtered matrix's pattern
    # filtered diagonal: the diagonal plus the weak entries, summed in row order
    weak_or_diag = ~strong
    dia_f = np.zeros(n)
    for i in range(n):  # sequential sum in the row's order (as the reference's loop)
        s = 0.0
        for j in range(rp[i], rp[i + 1]):
            if weak_or_diag[j]:
                s += va[j]
        dia_f[i] = s
    scale = np.where(dia_f != 0.0, -OMEGA * (1.0 / np.where(dia_f != 0.0, dia_f, 1.0)), 0.0)
    vals = np.where(ci == rows, 1.0 - OMEGA, scale[rows] * va)
    target = aid[ci]
    sel = (keep & (target >= 0)).tolist()
    vals_l, tgt_l = vals.tolist(), target.tolist()
    # P(i, aggregate) = sum of vals over the selected entries of row i, in row order
    pp, pc, pv = [0], [], []
    for i in range(n):
        acc = {}
        for j in range(rp[i], rp[i + 1]):
            if sel[j]:
                t = tgt_l[j]
                acc[t] = acc[t] + vals_l[j] if t in acc else vals_l[j]
        for t in sorted(acc):
            pc.append(t)
            pv.append(acc[t])
        pp.append(len(pc))
    P = sp.csr_matrix((np.asarray(pv), np.asarray(pc, dtype=np.int64), np.asarray(pp, dtype=np.int64)),
                      shape=(n, count))
    R = _sorted_csr(P.T)
    return P, R


# Ruge-Stuben (--amg-coarsening rs, AMGCL's coarsening/ruge_stuben.hpp with its default parameters)
RS_EPS_STRONG = float(np.float32(0.25))  # a_ij strong when a_ij < eps_str * min_k a_ik (negative couplings)
RS_EPS_TRUNC = float(np.float32(0.2))    # the float 0.2f as the double it widens to
_TINY = 2.0 * float(np.finfo(np.float64).eps)  # AMGCL's detail::eps<double>(1)
_U, _F, _C = 0, 1, 2


def _rs_strength(A: sp.csr_matrix):
    """Strong couplings per stored entry and the initial C/F marks: a row without a negative
    off-diagonal entry is F with no strong coupling; else a_ij (j != i) is strong when
    a_ij < eps_str * min_k a_ik."""
    n = A.shape[0]
    rp, ci, va = A.indptr, A.indices, A.data
    rows = np.repeat(np.arange(n), np.diff(rp))
    off = ci != rows
    amin = np.zeros(n)
    np.minimum.at(amin, rows[off], va[off])  # min(0, off-diagonal entries): exact in any order
    weak_row = np.abs(amin) < _TINY
    thr = amin * RS_EPS_STRONG
    strong = off & (va < thr[rows]) & ~weak_row[rows]
    cf = [_F if w else _U for w in weak_row.tolist()]
    return strong, cf


def _rs_split(A: sp.csr_matrix, strong: np.ndarray, cf: list) -> list:
    """Classic C/F splitting by decreasing measure lambda_i (the number of undecided variables
    that depend strongly on i, F ones counted twice), with AMGCL's bucket order: variables sit in
    groups of equal lambda, by increasing index at the start; the last variable of the highest
    group becomes C, the undecided variables depending on it F, and the measures move by one
    between adjacent groups (a rise to the end of the group above, a drop to the start of the
    group below)."""
    n = A.shape[0]
    rp, ci = A.indptr.tolist(), A.indices.tolist()
    st = strong.tolist()
    # transposed strength graph: for column c, the rows that depend strongly on c, by row
    tp = [0] * (n + 1)
    for j, s in enumerate(st):
        if s:
            tp[ci[j] + 1] += 1
    for i in range(n):
        tp[i + 1] += tp[i]
    tcol = [0] * tp[n]
    fill = tp[:n]
    for i in range(n):
        for j in range(rp[i], rp[i + 1]):
            if st[j]:
                c = ci[j]
                tcol[fill[c]] = i
                fill[c] += 1
    lam = [sum(1 if cf[k] == _U else 2 for k in tcol[tp[i]:tp[i + 1]]) for i in range(n)]
    size = max(n, max(lam, default=0) + 1)
    ptr = [0] * (size + 1)
    cnt = [0] * size
    for v in lam:
        ptr[v + 1] += 1
    for k in range(size):
        ptr[k + 1] += ptr[k]
    i2n = [0] * n
    n2i = [0] * n
    for i in range(n):
        v = lam[i]
        pos = ptr[v] + cnt[v]
        cnt[v] += 1
        i2n[pos] = i
        n2i[i] = pos

    def move(x, old_pos, new_pos):
        y = i2n[new_pos]
        n2i[x], n2i[y] = new_pos, old_pos
        i2n[old_pos], i2n[new_pos] = y, x

    for top in range(n - 1, -1, -1):
        i = i2n[top]
        li = lam[i]
        if li == 0:
            return [_C if m == _U else m for m in cf]
        cnt[li] -= 1
        if cf[i] == _F:
            continue
        cf[i] = _C
        for c in tcol[tp[i]:tp[i + 1]]:
            if cf[c] != _U:
                continue
            cf[c] = _F
            for aj in range(rp[c], rp[c + 1]):  # the undecided variables c depends on rise by one
                if not st[aj]:
                    continue
                a = ci[aj]
                la = lam[a]
                if cf[a] != _U or la + 1 >= n:
                    continue
                move(a, n2i[a], ptr[la] + cnt[la] - 1)
                cnt[la] -= 1
                cnt[la + 1] += 1
                ptr[la + 1] = ptr[la] + cnt[la]
                lam[a] = la + 1
        for j in range(rp[i], rp[i + 1]):  # the undecided variables i depends on drop by one
            if not st[j]:
                continue
            c = ci[j]
            lc = lam[c]
            if cf[c] != _U or lc == 0:
                continue
            move(c, n2i[c], ptr[lc])
            cnt[lc] -= 1
            cnt[lc - 1] += 1
            ptr[lc] += 1
            lam[c] = lc - 1
    return cf


def _rs_transfer(A: sp.csr_matrix):
    """(P, R) of one Ruge-Stuben level (direct interpolation with truncation), or None without
    C variables.  Row i of P: 1 at i's coarse index for C; for F, a_ij scaled by alpha (negative
    a_ij) or beta (positive) over the strong C couplings that survive truncation (outside
    [eps_tr * min, eps_tr * max] of them), alpha = -|sum of negative a_ik| / (|a_ii| |sum of the
    negative strong C ones|) rescaled for what truncation dropped, beta likewise; positive
    couplings without a strong positive C coupling are lumped into the diagonal."""
    n = A.shape[0]
    strong, cf = _rs_strength(A)
    cf = _rs_split(A, strong, cf)
    cidx = [0] * n
    nc = 0
    for i in range(n):
        if cf[i] == _C:
            cidx[i] = nc
            nc += 1
    if nc == 0:
        return None
    rp, ci, va, st = A.indptr.tolist(), A.indices.tolist(), A.data.tolist(), strong.tolist()
    pp, pc, pv = [0], [], []
    for i in range(n):
        if cf[i] == _C:
            pc.append(cidx[i])
            pv.append(1.0)
            pp.append(len(pc))
            continue
        lo = hi = 0.0
        for j in range(rp[i], rp[i + 1]):
            if st[j] and cf[ci[j]] == _C:
                lo = min(lo, va[j])
                hi = max(hi, va[j])
        lo *= RS_EPS_TRUNC
        hi *= RS_EPS_TRUNC
        dia = a_num = a_den = b_num = b_den = d_neg = d_pos = 0.0
        for j in range(rp[i], rp[i + 1]):
            c, v = ci[j], va[j]
            if c == i:
                dia = v
                continue
            sc = st[j] and cf[c] == _C
            if v < 0.0:
                a_num += v
                if sc:
                    a_den += v
                    if lo < v:
                        d_neg += v
            else:
                b_num += v
                if sc:
                    b_den += v
                    if v < hi:
                        d_pos += v
        cf_neg = abs(a_den) / abs(a_den - d_neg) if abs(a_den - d_neg) > _TINY else 1.0
        cf_pos = abs(b_den) / abs(b_den - d_pos) if abs(b_den - d_pos) > _TINY else 1.0
        if 0.0 < b_num and abs(b_den) < _TINY:
            dia += b_num
        alpha = -cf_neg * abs(a_num) / (abs(dia) * abs(a_den)) if abs(a_den) > _TINY else 0.0
        beta = -cf_pos * abs(b_num) / (abs(dia) * abs(b_den)) if abs(b_den) > _TINY else 0.0
        for j in range(rp[i], rp[i + 1]):
            c, v = ci[j], va[j]
            if not (st[j] and cf[c] == _C) or lo <= v <= hi:
                continue
            pc.append(cidx[c])
            pv.append((alpha if v < 0.0 else beta) * v)
        pp.append(len(pc))
    P = _sorted_csr(sp.csr_matrix((np.asarray(pv, dtype=np.float64), np.asarray(pc, dtype=np.int64),
                                   np.asarray(pp, dtype=np.int64)), shape=(n, nc)))
    return P, _sorted_csr(P.T)


def build_hierarchy(A, coarse_enough: int = 500, sweeps: int = 1, coarsening: str = "sa") -> AmgHierarchy:
    """The reference's AMG setup for one local matrix (see the module docstring); coarsening "sa"
    (smoothed aggregation) or "rs" (Ruge-Stuben, ``--amg-coarsening rs``)."""
    if coarsening not in ("sa", "rs"):
        raise ValueError(f"unknown AMG coarsening '{coarsening}' (sa|rs)")
    A = _sorted_csr(sp.csr_matrix(A, dtype=np.float64))
    H = AmgHierarchy(sweeps=int(sweeps))
    eps = EPS_STRONG
    direct = True
    while A is not None and A.shape[0] > coarse_enough:
        lvl = AmgLevel(A)
        H.levels.append(lvl)
        if coarsening == "rs":
            tr = _rs_transfer(A)
        else:
            tr = _transfer(A, eps)
            eps = np.float32(eps * np.float32(0.5))
        if tr is None:  # nothing to aggregate: the last level is smoothed only
            A = None
            direct = False
            break
        lvl.P, lvl.R = tr
        A = _sorted_csr(lvl.R @ (A @ lvl.P))
    if A is None or A.shape[0] > coarse_enough:
        direct = False
    if direct:
        H.coarse = A.toarray()
    return H


def rebuild_hierarchy(H: AmgHierarchy, A, single: bool = False) -> AmgHierarchy:
    """The hierarchy of new values of the same matrix with H's transfer operators kept: every
    coarser operator is recomputed as R (A P) and the coarsest is solved directly again
    (AMGCL's ``amg::rebuild``, ``amg.hpp:250-269``, ``level::rebuild``; the reference's
    refactorize() with ``--amg-reuse``, ``src/linalg/inexact_solver.cpp:77-89``)."""
    A = _sorted_csr(sp.csr_matrix(A, dtype=np.float64))
    if H.n != A.shape[0]:
        raise ValueError(f"rebuild: {A.shape[0]} rows, the hierarchy has {H.n}")
    out = AmgHierarchy(sweeps=H.sweeps)
    if single:  # the Galerkin products in float, as AMGCL<float> rebuilds them (values stored widened)
        A = A.astype(np.float32).astype(np.float64)
    for lvl in H.levels:
        out.levels.append(AmgLevel(A, lvl.P, lvl.R))
        if lvl.P is None:
            A = None
        elif single:
            f = np.float32
            A = _sorted_csr((lvl.R.astype(f) @ (A.astype(f) @ lvl.P.astype(f))).astype(np.float64))
        else:
            A = _sorted_csr(lvl.R @ (A @ lvl.P))
    if H.coarse is not None:
        out.coarse = A.toarray()
    return out


def build_hierarchy_native(A, coarse_enough: int = 500, sweeps: int = 1, coarsening: str = "sa",
                           single: bool = False) -> AmgHierarchy:
    """build_hierarchy computed by the library's host setup (s2l_amg_build, the same algorithms in
    C++, bit-identical levels) when libs2l_gpu.so is built, else by the Python restatement; used by
    the setup producer, where the Python loops would dominate the setup of large subdomains.
    single: the setup in single precision (--local-precision single; the library's host setup only)."""
    try:
        from . import capi
        N = capi.NativeAmg.build(A, coarse_enough, coarsening, single=single)
    except FileNotFoundError:
        if single:
            raise
        return build_hierarchy(A, coarse_enough=coarse_enough, sweeps=sweeps, coarsening=coarsening)
    try:
        return N.hierarchy(sweeps=sweeps)
    finally:
        N.close()
