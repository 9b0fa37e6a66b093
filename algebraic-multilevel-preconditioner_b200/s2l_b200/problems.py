"""Finite-volume test matrices of the solve phase, generated on the host (setup phase).

Restates the reference's generators (``src/utils/matrix_generators.cpp``):

* ``laplace(dim, ...)``: 5/7-point Laplacian, unit conductivity, Dirichlet faces only at
  y = 0/1 in 2D and z = 0/1 in 3D, zero flux elsewhere (``matrix_generators.cpp:57-193``,
  Dirichlet rows at ``:162-168``).
* ``bubbles(dim, ...)``: variable-coefficient pressure Poisson, beta = 1/rho, rho blended by
  the smoothed gas fraction of rising bubbles, p = 0 on the top face
  (``matrix_generators.cpp:195-306``; bubble field ``include/utils/bubble_field.hpp:43-158``).
  Extension: ``radius_cells=(rmin, rmax)`` draws one radius per bubble, in cells, from the
  same seeded engine right after that bubble's four reference draws.
* ``convdiff_fourier(...)``: 3D first-order upwind convection-diffusion with a seeded
  divergence-free Fourier velocity field (no counterpart in the reference, which only has the
  fixed field of ``matrix_generators.cpp:136-160``); face fluxes come from a vector potential so
  the discrete divergence of every cell is exactly zero.

Cells are numbered ``i + nx*(j + ny*k)``; every generator returns the cell coordinates so a
geometric partitioner can split the grid.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from .rng import MT19937_64


@dataclass
class Problem:
    A: sp.csr_matrix
    dims: tuple
    symmetric: bool
    description: str
    rhs_generated: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.A.shape[0]

    def cell_coords(self) -> np.ndarray:
        """Integer (i, j, k) of every cell, shape (n, 3)."""
        nx, ny, nz = self.dims
        c = np.arange(nx * ny * nz, dtype=np.int64)
        return np.stack([c % nx, (c // nx) % ny, c // (nx * ny)], axis=1)


def _faces(nx, ny, nz, dim):
    """Interior faces (P, N, direction) with N = P + stride, direction 0/1/2."""
    c = np.arange(nx * ny * nz, dtype=np.int64)
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    out = []
    m = i + 1 < nx
    out.append((c[m], c[m] + 1, 0))
    m = j + 1 < ny
    out.append((c[m], c[m] + nx, 1))
    if dim == 3:
        m = k + 1 < nz
        out.append((c[m], c[m] + nx * ny, 2))
    return out, (i, j, k)


def laplace(dim: int, nx: int, ny: int = 0, nz: int = 0) -> Problem:
    ny = ny or nx
    nz = (nz or nx) if dim == 3 else 1
    hx, hy = 1.0 / nx, 1.0 / ny
    hz = 1.0 / nz if dim == 3 else 1.0
    n = nx * ny * nz
    faces, (i, j, k) = _faces(nx, ny, nz, dim)
    geom = [hy * hz / hx, hx * hz / hy, hx * hy / hz]
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for P, N, d in faces:
        g = geom[d]
        rows += [P, N]
        cols += [N, P]
        vals += [np.full(P.size, -g), np.full(P.size, -g)]
        np.add.at(diag, P, g)
        np.add.at(diag, N, g)
    rhs = np.zeros(n)
    if dim == 2:
        gd = hx / (0.5 * hy)
        diag[j == 0] += gd
        diag[j == ny - 1] += gd
        rhs[j == ny - 1] += gd * 1.0
    else:
        gd = hx * hy / (0.5 * hz)
        diag[k == 0] += gd
        diag[k == nz - 1] += gd
        rhs[k == 0] += gd * 1.0
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    desc = f"laplace{dim}d {nx}x{ny}" + (f"x{nz}" if dim == 3 else "") + f" (n={n}, nnz={A.nnz})"
    return Problem(A, (nx, ny, nz), True, desc, rhs)


def _segment_distance(px, py, ax, ay, bx, by):
    vx, vy = bx - ax, by - ay
    t = np.clip(((px - ax) * vx + (py - ay) * vy) / (vx * vx + vy * vy), 0.0, 1.0)
    dx, dy = px - (ax + t * vx), py - (ay + t * vy)
    return np.sqrt(dx * dx + dy * dy)


def kappa(x, y):
    """The reference's heterogeneous diffusivity (``MatrixGenerator::kappa``,
    ``src/utils/matrix_generators.cpp:33-44``): 2 in a rectangle, 0.06 in two channels and in a
    periodic lattice of square inclusions, 1 elsewhere."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    px, py = np.fmod(x, 0.2) - 0.1, np.fmod(y, 0.2) - 0.1
    k = np.where((np.abs(px) < 0.035) & (np.abs(py) < 0.035), 6e-2, 1.0)
    k = np.where(_segment_distance(x, y, 0.55, 0.62, 0.90, 0.35) < 0.03, 6e-2, k)
    k = np.where(_segment_distance(x, y, 0.15, 0.62, 0.75, 0.70) < 0.04, 6e-2, k)
    return np.where((x >= 0.10) & (x <= 0.45) & (y >= 0.12) & (y <= 0.30), 2.0, k)


def convdiff(dim: int, nx: int, ny: int = 0, nz: int = 0, nu: float = 1.0, ncomp: int = 1, pulse: float = 0.0,
             time: float = 0.0, pulse_period: int = 20, coupled: bool = False) -> Problem:
    """The reference's convdiff{2d,3d} and coupled{2d,3d} generators (``--generate``,
    ``src/utils/matrix_generators.cpp:57-192``): upwind finite volumes of -div(nu kappa grad u) +
    div(V u) with the Section-4.2 velocity (exact face integrals of V.n, scaled by
    1 + pulse sin(2 pi t / period)), harmonic-mean diffusivity on x/y faces, Dirichlet faces
    (2D: y = 0 -> 0, y = 1 -> 1; 3D: z = 0 -> 1, z = 1 -> 0); `coupled` repeats it for ncomp
    components (viscosity nu (1 + c)) with a nonsymmetric cyclic coupling between them."""
    ny = ny or nx
    nz = (nz or nx) if dim == 3 else 1
    nc = max(1, ncomp) if coupled else 1
    hx, hy = 1.0 / nx, 1.0 / ny
    hz = 1.0 / nz if dim == 3 else 1.0
    ncell = nx * ny * nz
    n = ncell * nc
    conv = 1.0 + pulse * np.sin(2.0 * np.pi * time / max(1, pulse_period))
    c = np.arange(ncell, dtype=np.int64)
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    kP = kappa((i + 0.5) * hx, (j + 0.5) * hy)
    x0, x1, y0, y1 = i * hx, (i + 1) * hx, j * hy, (j + 1) * hy
    z0, z1 = k * hz, (k + 1) * hz

    def P1(t):
        return t * t - t

    rows, cols, vals = [], [], []
    rhs = np.zeros(n)

    def face(m, N, geom, F):
        P = c[m]
        F = F * conv
        for comp in range(nc):
            D = nu * (1.0 + comp) * geom
            p, q = P * nc + comp, N * nc + comp
            rows.extend([p, p, q, q])
            cols.extend([p, q, q, p])
            vals.extend([D + np.maximum(F, 0.0), -D - np.maximum(-F, 0.0), D + np.maximum(-F, 0.0),
                         -D - np.maximum(F, 0.0)])

    m = i + 1 < nx
    kN = kappa((i[m] + 1.5) * hx, (j[m] + 0.5) * hy)
    kf = 2.0 * kP[m] * kN / (kP[m] + kN)
    xf = x1[m]
    if dim == 2:
        F = xf * (1.0 - xf) * (P1(y1[m]) - P1(y0[m]))
    else:
        F = 2.0 * xf * (1.0 - xf) * (P1(y1[m]) - P1(y0[m])) * 0.5 * (z1[m] * z1[m] - z0[m] * z0[m])
    face(m, c[m] + 1, kf * (hy * hz) / hx, F)
    m = j + 1 < ny
    kN = kappa((i[m] + 0.5) * hx, (j[m] + 1.5) * hy)
    kf = 2.0 * kP[m] * kN / (kP[m] + kN)
    yf = y1[m]
    F = -yf * (1.0 - yf) * (P1(x1[m]) - P1(x0[m])) * (1.0 if dim == 2 else (z1[m] - z0[m]))
    face(m, c[m] + nx, kf * (hx * hz) / hy, F)
    if dim == 3:
        m = k + 1 < nz
        zf = z1[m]
        F = -zf * (1.0 - zf) * (P1(x1[m]) - P1(x0[m])) * (P1(y1[m]) - P1(y0[m]))
        face(m, c[m] + nx * ny, kP[m] * (hx * hy) / hz, F)
    if dim == 2:
        bnd = [(j == 0, kP * hx / (0.5 * hy), 0.0), (j == ny - 1, kP * hx / (0.5 * hy), 1.0)]
    else:
        bnd = [(k == 0, kP * hx * hy / (0.5 * hz), 1.0), (k == nz - 1, kP * hx * hy / (0.5 * hz), 0.0)]
    for m, geom, ub in bnd:
        for comp in range(nc):
            D = nu * (1.0 + comp) * geom[m]
            p = c[m] * nc + comp
            rows.append(p)
            cols.append(p)
            vals.append(D)
            np.add.at(rhs, p, D * ub)
    if nc > 1:
        gamma = nu * (hy / hx if dim == 2 else hy * hz / hx)
        for comp in range(nc):
            p = c * nc + comp
            rows.extend([p, p])
            cols.extend([p, c * nc + (comp + 1) % nc])
            vals.extend([np.full(ncell, gamma), np.full(ncell, -gamma)])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    name = ("coupled" if coupled else "convdiff") + f"{dim}d"
    desc = f"{name} {nx}x{ny}" + (f"x{nz}" if dim == 3 else "") + f" nu={nu:g}" + \
        (f" ncomp={nc}" if nc > 1 else "") + (f" pulse={pulse:g} t={time:g}" if pulse != 0.0 else "") + \
        f" (n={n}, nnz={A.nnz})"
    return Problem(A, (nx, ny, nz), False, desc, rhs)


def bubble_alpha(dim, nx, ny, nz, nbubbles, radius, cfl, time, seed, radius_cells=None):
    """Gas fraction of every cell (``include/utils/bubble_field.hpp:56-117,150-156``).

    alpha = 0.5 (1 - tanh((d - R)/w)), w = one cell, maximum over the bubbles and their periodic
    copies, evaluated only inside the index box of half-width R + 4w around each copy.
    """
    nz = nz if dim == 3 else 1
    n_ = [nx, ny, nz]
    h = [1.0 / nx, 1.0 / ny, (1.0 / nz) if dim == 3 else 1.0]
    nv = nz if dim == 3 else ny
    hv = 1.0 / nv
    w = max(h[0], max(h[1], h[2] if dim == 3 else h[1]))
    g = MT19937_64(seed)
    rise = cfl * hv * time
    vdir = 2 if dim == 3 else 1
    alpha = np.zeros(nx * ny * nz)
    for _ in range(nbubbles):
        x0, y0, z0, ph = g.uniform(4)
        R = radius
        if radius_cells is not None:
            lo, hi = radius_cells
            R = (lo + (hi - lo) * g.uniform(1)[0]) * w
        x0 = R + (1.0 - 2.0 * R) * x0
        y0 = R + (1.0 - 2.0 * R) * y0
        phase = 2.0 * np.pi * ph
        wob = 0.5 * R * np.sin(2.0 * np.pi * time / 40.0 + phase)
        xw = x0 + wob
        xc = R if xw < R else (1.0 - R if 1.0 - R < xw else xw)
        if dim == 3:
            c = [xc, y0, z0 + rise]
        else:
            c = [xc, z0 + rise, 0.5]
        c[vdir] -= np.floor(c[vdir])
        reach = R + 4.0 * w
        for image in (-1, 0, 1):
            cc = list(c)
            cc[vdir] += image
            lo_, hi_ = [0, 0, 0], [0, 0, 0]
            empty = False
            for d in range(dim):
                lo_[d] = max(0, int(np.floor((cc[d] - reach) / h[d])))
                hi_[d] = min(n_[d] - 1, int(np.floor((cc[d] + reach) / h[d])))
                empty = empty or lo_[d] > hi_[d]
            if empty:
                continue
            ii = np.arange(lo_[0], hi_[0] + 1)
            jj = np.arange(lo_[1], hi_[1] + 1)
            kk = np.arange(lo_[2], hi_[2] + 1) if dim == 3 else np.array([0])
            K, J, I = np.meshgrid(kk, jj, ii, indexing="ij")
            dx = (I + 0.5) * h[0] - cc[0]
            dy = (J + 0.5) * h[1] - cc[1]
            dz = ((K + 0.5) * h[2] - cc[2]) if dim == 3 else 0.0
            dist = np.sqrt(dx * dx + dy * dy + dz * dz)
            prof = 0.5 * (1.0 - np.tanh((dist - R) / w))
            idx = (I + nx * (J + ny * K)).ravel()
            alpha[idx] = np.maximum(alpha[idx], prof.ravel())
    return alpha


def bubbles(dim: int, nx: int, ny: int = 0, nz: int = 0, nbubbles: int = 50, radius: float = 0.06,
            rho_ratio: float = 1000.0, cfl: float = 0.5, time: float = 0.0, seed: int = 2024,
            radius_cells=None) -> Problem:
    ny = ny or nx
    nz = (nz or nx) if dim == 3 else 1
    hx, hy = 1.0 / nx, 1.0 / ny
    hz = 1.0 / nz if dim == 3 else 1.0
    n = nx * ny * nz
    alpha = bubble_alpha(dim, nx, ny, nz, nbubbles, radius, cfl, time, seed, radius_cells)
    rho_g = 1.0 / rho_ratio
    beta = 1.0 / (alpha * rho_g + (1.0 - alpha))
    c = np.arange(n, dtype=np.int64)
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    gx, gy, gz = hy * hz / hx, hx * hz / hy, hx * hy / hz
    # neighbours in the reference's column order: k-1, j-1, i-1, P, i+1, j+1, k+1
    nb = []
    if dim == 3:
        nb.append((k > 0, -nx * ny, gz))
    nb.append((j > 0, -nx, gy))
    nb.append((i > 0, -1, gx))
    nb_hi = [(i + 1 < nx, 1, gx), (j + 1 < ny, nx, gy)]
    if dim == 3:
        nb_hi.append((k + 1 < nz, nx * ny, gz))
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for m, off, geom in nb + nb_hi:
        P = c[m]
        N = P + off
        coef = 0.5 * (beta[P] + beta[N]) * geom
        rows.append(P)
        cols.append(N)
        vals.append(-coef)
        diag[P] = diag[P] + coef
    top = (k == nz - 1) if dim == 3 else (j == ny - 1)
    gtop = hx * hy / (0.5 * hz) if dim == 3 else hx * hz / (0.5 * hy)
    diag[top] = diag[top] + beta[top] * gtop
    rows.append(c)
    cols.append(c)
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sort_indices()
    rhs = (hx * hy * hz) * alpha
    desc = (f"bubbles{dim}d {nx}x{ny}" + (f"x{nz}" if dim == 3 else "") +
            f" rho_ratio={rho_ratio:g} nb={nbubbles} " +
            (f"R={radius_cells[0]}-{radius_cells[1]} cells" if radius_cells else f"R={radius:g}") +
            f" t={time:g} (n={n}, nnz={A.nnz})")
    return Problem(A, (nx, ny, nz), True, desc, rhs, {"alpha": alpha})


def convdiff_fourier(nx: int, ny: int = 0, nz: int = 0, modes: int = 4, peclet=(0.1, 10.0),
                     nu: float = 1.0, seed: int = 7) -> Problem:
    """3D upwind convection-diffusion on a seeded divergence-free Fourier velocity field.

    The velocity is u = curl(psi) with psi a sum of ``modes`` seeded sine modes; the flux of every
    face is the circulation of psi around that face (Stokes), so the net flux out of every cell is
    exactly zero up to rounding.  The field is scaled so that the cell Peclet number
    |u| h / nu spans ``peclet``: the amplitude of each mode is drawn log-uniformly in that range.
    Dirichlet faces at z = 0 (u = 1) and z = 1 (u = 0), zero flux elsewhere, as the reference's
    3D convection-diffusion (``matrix_generators.cpp:162-168``).
    """
    ny = ny or nx
    nz = nz or nx
    hx, hy, hz = 1.0 / nx, 1.0 / ny, 1.0 / nz
    n = nx * ny * nz
    g = MT19937_64(seed)
    # psi(x) = sum_m a_m * e_m * sin(2 pi k_m . x + phi_m) at the grid nodes
    ks, amps, dirs, phis = [], [], [], []
    lp0, lp1 = np.log(peclet[0]), np.log(peclet[1])
    for _ in range(modes):
        r = g.uniform(8)
        kv = 1 + np.floor(r[0:3] * 3.0)
        d = r[3:6] - 0.5
        d /= np.linalg.norm(d) + 1e-300
        pe = np.exp(lp0 + (lp1 - lp0) * r[6])
        # |u| ~ amp * 2 pi |k|; cell Peclet = |u| h / nu
        amp = pe * nu / (hx * 2.0 * np.pi * np.linalg.norm(kv))
        ks.append(kv)
        dirs.append(d)
        amps.append(amp)
        phis.append(2.0 * np.pi * r[7])

    def psi(x, y, z):
        out = np.zeros(x.shape + (3,))
        for kv, d, a, ph in zip(ks, dirs, amps, phis):
            s = a * np.sin(2.0 * np.pi * (kv[0] * x + kv[1] * y + kv[2] * z) + ph)
            out += s[..., None] * d
        return out

    # psi on the edges: average of the two node values times the edge length (trapezoid)
    xn = np.arange(nx + 1) * hx
    yn = np.arange(ny + 1) * hy
    zn = np.arange(nz + 1) * hz
    Zn, Yn, Xn = np.meshgrid(zn, yn, xn, indexing="ij")
    P = psi(Xn, Yn, Zn)  # (nz+1, ny+1, nx+1, 3)
    # edge integrals: along x (component 0), along y (1), along z (2)
    Ex = 0.5 * (P[:, :, :-1, 0] + P[:, :, 1:, 0]) * hx  # (nz+1, ny+1, nx)
    Ey = 0.5 * (P[:, :-1, :, 1] + P[:, 1:, :, 1]) * hy  # (nz+1, ny, nx+1)
    Ez = 0.5 * (P[:-1, :, :, 2] + P[1:, :, :, 2]) * hz  # (nz, ny+1, nx+1)
    # flux through the x-face at node-plane i (normal +x): circulation of psi around its boundary
    Fx = (Ey[:-1, :, :] + Ez[:, 1:, :] - Ey[1:, :, :] - Ez[:, :-1, :])  # (nz, ny, nx+1)
    Fy = (Ez[:, :, :-1] + Ex[1:, :, :] - Ez[:, :, 1:] - Ex[:-1, :, :])  # (nz, ny+1, nx)
    Fz = (Ex[:, :-1, :] + Ey[:, :, 1:] - Ex[:, 1:, :] - Ey[:, :, :-1])  # (nz+1, ny, nx)
    c = np.arange(n, dtype=np.int64)
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    rows, cols, vals = [], [], []
    diag = np.zeros(n)

    def face(m, off, Dgeom, F):
        Pc = c[m]
        Nc = Pc + off
        rows.extend([Pc, Nc])
        cols.extend([Nc, Pc])
        vals.extend([-Dgeom - np.maximum(-F, 0.0), -Dgeom - np.maximum(F, 0.0)])
        np.add.at(diag, Pc, Dgeom + np.maximum(F, 0.0))
        np.add.at(diag, Nc, Dgeom + np.maximum(-F, 0.0))

    m = i + 1 < nx
    face(m, 1, nu * hy * hz / hx, Fx[k[m], j[m], i[m] + 1])
    m = j + 1 < ny
    face(m, nx, nu * hx * hz / hy, Fy[k[m], j[m] + 1, i[m]])
    m = k + 1 < nz
    face(m, nx * ny, nu * hx * hy / hz, Fz[k[m] + 1, j[m], i[m]])
    gd = nu * hx * hy / (0.5 * hz)
    rhs = np.zeros(n)
    diag[k == 0] += gd
    rhs[k == 0] += gd
    diag[k == nz - 1] += gd
    rows.append(c)
    cols.append(c)
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    div = np.zeros(n)
    div += Fx[k, j, i + 1] - Fx[k, j, i] + Fy[k, j + 1, i] - Fy[k, j, i] + Fz[k + 1, j, i] - Fz[k, j, i]
    umax = np.max(np.abs(np.concatenate([Fx.ravel() / (hy * hz), Fy.ravel() / (hx * hz), Fz.ravel() / (hx * hy)])))
    desc = f"convdiff3d-fourier {nx}x{ny}x{nz} modes={modes} Pe_cell<={umax * hx / nu:.3g} (n={n}, nnz={A.nnz})"
    return Problem(A, (nx, ny, nz), False, desc, rhs, {"max_div": float(np.max(np.abs(div))), "umax": umax})
