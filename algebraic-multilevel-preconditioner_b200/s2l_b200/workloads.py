"""Named workloads of the solve phase (seeded, synthetic).

* ``poisson2d``: 2D 5-point Poisson 200x200 (n = 40,000), 8 subdomains, overlap 1, nev 20,
  RAS + additive coarse term, exact LU, GMRES(30), rtol 1e-8 (the reference's own CPU case).
* ``bubbles3d``: 3D 7-point variable-coefficient pressure Poisson 100^3 (n = 1.0M),
  beta = 1/rho, rho = 1e-3 in 200 seeded spheres of radius 3-8 cells, 64 subdomains, overlap 2,
  nev 20, deflated RAS, local L L^T, GMRES(50), rtol 1e-8, U[-1,1] right-hand side.
* ``convdiff3d``: 3D upwind convection-diffusion 128^3 (n = 2.1M) on a seeded divergence-free
  4-mode Fourier field with cell Peclet 0.1-10, 128 subdomains, overlap 1, nev 24, FP32 LU
  factors, flexible GMRES(40).

Every workload takes a ``scale`` so tests can run the same family at small sizes.
"""
from __future__ import annotations

from dataclasses import dataclass, field, asdict

import numpy as np

from . import partition as partmod
from . import problems
from .rng import random_rhs
from .setup_phase import SchwarzOptions, build_setup, cached


@dataclass
class Workload:
    name: str
    kind: str                    # laplace2d | laplace3d | bubbles3d | convdiff3d
    nx: int
    nsub: int
    opts: SchwarzOptions
    krylov: str = "gmres"
    restart: int = 30
    rtol: float = 1e-8
    flexible: bool = False
    seed: int = 12345
    nbubbles: int = 200
    radius_cells: tuple | None = (3.0, 8.0)
    rho_ratio: float = 1000.0
    imbalance: float = 0.0
    time: float = 0.0
    extra: dict = field(default_factory=dict)

    def key(self) -> dict:
        d = asdict(self)
        d["opts"] = tuple(sorted(asdict(self.opts).items()))
        d["extra"] = tuple(sorted(self.extra.items()))
        d["version"] = 3
        return d


def poisson2d(nx=200, nsub=8) -> Workload:
    return Workload("poisson2d", "laplace2d", nx, nsub,
                    SchwarzOptions(one_level="ras", coarse="additive", pou="boolean", overlap=1, nev=20,
                                   local_factorization="lu"), restart=30)


def bubbles3d(nx=100, nsub=64, nbubbles=200, overlap=2, precision="double") -> Workload:
    return Workload("bubbles3d", "bubbles3d", nx, nsub,
                    SchwarzOptions(one_level="ras", coarse="deflated", pou="boolean", overlap=overlap, nev=20,
                                   local_factorization="cholesky", local_precision=precision),
                    restart=50, nbubbles=nbubbles)


def convdiff3d(nx=128, nsub=128, precision="single") -> Workload:
    return Workload("convdiff3d", "convdiff3d", nx, nsub,
                    SchwarzOptions(one_level="ras", coarse="deflated", pou="boolean", overlap=1, nev=24,
                                   local_factorization="lu", local_precision=precision),
                    restart=40, flexible=True)


def reference_generator(kind: str, nx=32, nsub=8, **extra) -> Workload:
    """A workload on one of the reference's own generators (``--generate convdiff2d`` etc.):
    kind reference_convdiff2d | reference_convdiff3d | reference_coupled2d | reference_coupled3d;
    extra: nu, ncomp, pulse, pulse_period.  Deflated RAS, LU factors, GMRES(40)."""
    return Workload(kind, kind, nx, nsub,
                    SchwarzOptions(one_level="ras", coarse="deflated", pou="boolean", overlap=1, nev=8,
                                   local_factorization="lu"), restart=40, extra=dict(extra))


def make_problem(w: Workload):
    if w.kind == "laplace2d":
        return problems.laplace(2, w.nx)
    if w.kind == "laplace3d":
        return problems.laplace(3, w.nx)
    if w.kind == "bubbles3d":
        return problems.bubbles(3, w.nx, nbubbles=w.nbubbles, rho_ratio=w.rho_ratio, radius_cells=w.radius_cells,
                                time=w.time, seed=w.extra.get("bubble_seed", 2024))
    if w.kind == "convdiff3d":
        return problems.convdiff_fourier(w.nx, seed=w.extra.get("field_seed", 7))
    if w.kind in ("reference_convdiff2d", "reference_convdiff3d", "reference_coupled2d", "reference_coupled3d"):
        # the reference's own --generate convdiff{2d,3d} / coupled{2d,3d}; with a pulse the
        # convection changes with the time step (a nonsymmetric sequence on one pattern)
        e = w.extra
        return problems.convdiff(3 if w.kind.endswith("3d") else 2, w.nx, nu=e.get("nu", 1.0),
                                 ncomp=e.get("ncomp", 4), pulse=e.get("pulse", 0.0), time=w.time,
                                 pulse_period=e.get("pulse_period", 20), coupled="coupled" in w.kind)
    raise ValueError(f"unknown workload kind {w.kind}")


def make_partition(w: Workload, prob) -> np.ndarray:
    """Subdomain of every unknown: cells by recursive coordinate bisection, the unknowns of a cell
    (coupled problems) with their cell."""
    part = partmod.rcb(prob.cell_coords().astype(np.float64), w.nsub, imbalance=w.imbalance)
    per_cell = prob.A.shape[0] // part.size
    return np.repeat(part, per_cell) if per_cell > 1 else part


def build(w: Workload, workers=None, use_cache=True, pool=None):
    """Problem + partition + setup (cached under $S2L_CACHE_DIR when set); `pool`: a process pool of
    setup_phase.worker_pool for the per-subdomain work."""
    def make():
        prob = make_problem(w)
        part = make_partition(w, prob)
        b = random_rhs(prob.n, w.seed)
        st = build_setup(prob.A, b, part, w.nsub, w.opts, prob.symmetric, workers=workers,
                         description=prob.description, pool=pool)
        st.stats["part"] = part
        return st
    if use_cache:
        return cached(w.key(), make)
    return make()
