import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "algebraic-multilevel-preconditioner_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libs2l_gpu.so")


_SETUPS = {}


def small_setup(name: str, **kw):
    """Small seeded setups of the three workload families, built once per test session."""
    from s2l_b200 import workloads as W
    from s2l_b200.setup_phase import SchwarzOptions
    key = (name, tuple(sorted(kw.items())))
    if key in _SETUPS:
        return _SETUPS[key]
    if name == "poisson2d":
        w = W.poisson2d(kw.get("nx", 40), kw.get("nsub", 4))
    elif name == "bubbles3d":
        w = W.bubbles3d(kw.get("nx", 16), kw.get("nsub", 8), nbubbles=kw.get("nbubbles", 6),
                        overlap=kw.get("overlap", 2), precision=kw.get("precision", "double"))
    elif name == "convdiff3d":
        w = W.convdiff3d(kw.get("nx", 14), kw.get("nsub", 8), precision=kw.get("precision", "double"))
        w.opts.nev = kw.get("nev", 8)
    else:
        raise ValueError(name)
    if "precision" in kw:
        w.opts.local_precision = kw["precision"]
    for k in ("one_level", "coarse", "pou", "overlap", "local_approx", "amg_coarse_enough", "amg_sweeps",
              "amg_coarsening"):
        if k in kw:
            setattr(w.opts, k, kw[k])
    st = W.build(w, workers=1, use_cache=False)
    _SETUPS[key] = (w, st)
    return w, st


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
