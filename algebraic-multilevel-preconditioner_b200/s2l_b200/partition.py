"""Partition of the unknowns into subdomains and the part-contiguous renumbering.

The reference calls METIS_PartGraphKway on G(A + A^T) (``src/partition/graph_partitioner.cpp``),
which is not available here.  The setup phase of this package uses a deterministic recursive
coordinate bisection of the grid cells instead (compact, balanced parts); the oracle build feeds
the same partition vector to the reference, so both sides decompose identically.

``renumber`` follows ``src/partition/domain_decomposer.cpp:254-268``: the unknowns of part p get
the contiguous range [ownership[p], ownership[p+1]) and keep their original order inside a part.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def rcb(coords: np.ndarray, nparts: int, imbalance: float = 0.0, seed: int = 0) -> np.ndarray:
    """Recursive coordinate bisection.

    Splits along the longest extent, at the fraction k/nparts of the points (k = nparts // 2), so
    every part gets n/nparts points.  ``imbalance`` > 0 moves each cut by a seeded random fraction
    of up to ``imbalance`` of the smaller side, giving uneven parts (sizes still deterministic).
    """
    n = coords.shape[0]
    part = np.zeros(n, dtype=np.int32)
    rng = np.random.default_rng(seed)
    stack = [(np.arange(n), 0, nparts)]
    while stack:
        idx, first, np_ = stack.pop()
        if np_ == 1:
            part[idx] = first
            continue
        c = coords[idx]
        ext = c.max(axis=0) - c.min(axis=0)
        ax = int(np.argmax(ext))
        k = np_ // 2
        frac = k / np_
        if imbalance > 0.0:
            frac *= 1.0 + imbalance * (2.0 * rng.random() - 1.0) * min(frac, 1 - frac) / max(frac, 1e-12)
            frac = min(max(frac, 0.05), 0.95)
        # stable order: by coordinate, ties by original index
        order = np.lexsort((idx, c[:, ax]))
        cut = int(round(frac * idx.size))
        cut = min(max(cut, k), idx.size - (np_ - k))
        stack.append((idx[order[cut:]], first + k, np_ - k))
        stack.append((idx[order[:cut]], first, k))
    return part


def bfs_bisection(A: sp.csr_matrix, nparts: int) -> np.ndarray:
    """Graph-only fallback (no coordinates): recursive bisection of a breadth-first order."""
    from scipy.sparse.csgraph import breadth_first_order

    S = (A + A.T).tocsr()
    n = A.shape[0]
    part = np.zeros(n, dtype=np.int32)
    stack = [(np.arange(n), 0, nparts)]
    while stack:
        idx, first, np_ = stack.pop()
        if np_ == 1:
            part[idx] = first
            continue
        sub = S[idx][:, idx]
        order = breadth_first_order(sub, int(np.argmin(np.diff(sub.indptr))), directed=False,
                                    return_predecessors=False)
        if order.size < idx.size:  # disconnected: append the rest in index order
            rest = np.setdiff1d(np.arange(idx.size), order)
            order = np.concatenate([order, rest])
        k = np_ // 2
        cut = int(round(k / np_ * idx.size))
        stack.append((idx[order[cut:]], first + k, np_ - k))
        stack.append((idx[order[:cut]], first, k))
    return part


def renumber(part: np.ndarray, nparts: int):
    """ownership (nparts+1), new_to_old, old_to_new (``domain_decomposer.cpp:254-268``)."""
    counts = np.bincount(part, minlength=nparts).astype(np.int64)
    if np.any(counts == 0):
        raise RuntimeError("the partition produced an empty subdomain")
    ownership = np.zeros(nparts + 1, dtype=np.int64)
    np.cumsum(counts, out=ownership[1:])
    new_to_old = np.argsort(part, kind="stable").astype(np.int64)
    old_to_new = np.empty_like(new_to_old)
    old_to_new[new_to_old] = np.arange(part.size, dtype=np.int64)
    return ownership, new_to_old, old_to_new


def permute(A: sp.csr_matrix, new_to_old: np.ndarray) -> sp.csr_matrix:
    """P A P^T with sorted column indices (``domain_decomposer.cpp:166-197``)."""
    Ap = A[new_to_old][:, new_to_old].tocsr()
    Ap.sort_indices()
    return Ap
