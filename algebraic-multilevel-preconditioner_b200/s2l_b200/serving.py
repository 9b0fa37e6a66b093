"""Serving loop of the solve phase on one GPU.

Requests name a matrix by key.  The engine keeps one device setup per key (least recently used
first out), reuses it for every request on that matrix and along a sequence of values of it
(``update``: the reference's UpdateLevel::Reuse, preconditioner kept, or Refactorize on the
device), and runs the solves on the
native worker threads of the context (``s2l_gpu_serve_start``), so requests that arrive while
others are on the GPU overlap with them.  GMRES requests on one matrix are batched continuously
(``s2l_gpu_serve_batching``): they share the Arnoldi steps of a block runner, joining it as slots
free up and leaving it as they converge.  Memory is admitted by the context's HBM budget: a
solve whose buffers do not fit waits in the library for a workspace of its setup to come free,
and a new setup that does not fit evicts idle setups (those with no queued or running solve)
until it does.
"""
from __future__ import annotations

import threading
from collections import OrderedDict

from . import capi


class Engine:
    def __init__(self, device: int = 0, hbm_budget: int = 0, workers: int = 4, batching: int = -1):
        self.ctx = capi.Context(device, int(hbm_budget))
        self.ctx.serve_start(workers, batching=batching)
        self._cache: OrderedDict[object, capi.GpuSetup] = OrderedDict()
        self._lock = threading.Lock()
        self.builds = 0  # device setups created (cache misses)
        self.evictions = 0

    def setup(self, key, make, options=None) -> capi.GpuSetup:
        """The device setup of matrix `key`; `make()` returns its host setup on a miss."""
        with self._lock:
            g = self._cache.get(key)
            if g is not None:
                self._cache.move_to_end(key)
                return g
        st = make()
        while True:
            try:
                g = capi.GpuSetup(self.ctx, st, options=options)
                break
            except capi.S2LError as e:
                if e.code != 2 or not self._evict_one():  # 2: S2L_ERR_OOM (budget)
                    raise
        with self._lock:
            other = self._cache.get(key)
            if other is not None:  # built concurrently by another request: keep the first
                g.close()
                self._cache.move_to_end(key)
                return other
            self._cache[key] = g
            self.builds += 1
        return g

    def _evict_one(self) -> bool:
        """Release the least recently used setup that has nothing queued or running."""
        with self._lock:
            for key, g in list(self._cache.items()):
                if g.lib.s2l_gpu_setup_destroy(g.h) == capi.S2L_OK:
                    g.h = None
                    del self._cache[key]
                    self.evictions += 1
                    return True
        return False

    def update(self, key, values, level: str = "reuse") -> None:
        """Next matrix of a sequence on `key` (new values of A, same pattern).  level "reuse" keeps
        the preconditioner (UpdateLevel::Reuse); "refactorize" refactorizes it on the device
        (UpdateLevel::Refactorize; the setup must have been made with options {"refactor": 1})."""
        with self._lock:
            g = self._cache[key]
        if level == "reuse":
            g.update_matrix(values)
        elif level == "refactorize":
            g.refactor(values)
        else:
            raise ValueError(f"unknown update level {level!r}")

    def submit(self, key, make, b, x0=None, method="gmres", options=None, **kw) -> capi.Ticket:
        """Queue one solve of matrix `key` and return its ticket at once."""
        return self.setup(key, make, options).submit(b, x0=x0, method=method, **kw)

    def resident(self):
        with self._lock:
            return list(self._cache.keys())

    def close(self):
        with self._lock:
            for g in self._cache.values():
                g.close()
            self._cache.clear()
        self.ctx.close()
