"""Synthetic initial data of the benchmark workloads (host arrays, cell order
ic = i * ny + j).  Nothing here is measured; it only builds inputs.

riemann2d_case3   four-quadrant Riemann problem, zephyr's Riemann2D(3)
                  (phys/tests/test_2D.cpp:26-31, quadrant rules 72-110), point
                  values at cell centres.
fourier_smooth    smooth periodic data: rho = 1 + 0.2 f, u = 0.3 f, v = 0.3 f,
                  p = 1 + 0.1 f, each f = sum_{m=1..8} a_m sin(2 pi m x + phi_m)
                  sin(2 pi m y + psi_m), a_m ~ U(0,1)/8, phi, psi ~ U(0, 2 pi),
                  drawn (a_m, phi_m, psi_m) for m = 1..8 from numpy's PCG64
                  with seeds 1, 2, 3, 4 for rho, u, v, p.
transfer_disks    volume fractions of disks for the VOF transport (Transfer):
                  the transfer problem's disk (problems/transfer.cpp:334-354,
                  radius 0.1 at (0.15, 0.5) in [0, 1] x [0, 0.7]) or a seeded
                  field of disks; cell fractions by sub x sub midpoint
                  sampling of the cells that the circles cross.
blast_cell_means  the AMR blast: rho = 1, u = v = 0, p = 1e-5 except p = 1e3
                  for r < 0.01 around (0.5, 0.5); cell means of the
                  conservative state by n x n midpoint sub-sampling of each
                  cell (the sub-sampled initialisation of smf_test_2D.cpp:77-87,
                  IVP::*_mean), for the cells of an adaptive mesh.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .smf import Boundaries, Boundary, IdealGas, Rectangle


@dataclass
class Workload:
    name: str
    gen: Rectangle
    eos: object
    state: tuple  # (rho, vx, vy, p, e)


def _centres(gen: Rectangle):
    X = gen.x_min + ((gen.x_max - gen.x_min) * np.arange(gen.nx() + 1)) / gen.nx()
    Y = gen.y_min + ((gen.y_max - gen.y_min) * np.arange(gen.ny() + 1)) / gen.ny()
    cx = 0.25 * (((X[:-1] + X[1:]) + X[:-1]) + X[1:])
    cy = 0.25 * (((Y[:-1] + Y[:-1]) + Y[1:]) + Y[1:])
    return cx, cy


def riemann2d_case3(n: int = 256) -> Workload:
    gen = Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Boundaries(Boundary.ZOE, Boundary.ZOE, Boundary.ZOE, Boundary.ZOE))
    gen.set_nx(n)
    eos = IdealGas(1.4)
    cx, cy = _centres(gen)
    x = np.repeat(cx, gen.ny())
    y = np.tile(cy, gen.nx())
    # (rho, u, v, p) of quadrants 1 (NE), 2 (NW), 3 (SW), 4 (SE): test_2D.cpp:26-31
    q = {1: (1.5, 0.0, 0.0, 1.5), 2: (0.5323, 1.206, 0.0, 0.3), 3: (0.138, 1.206, 1.206, 0.029),
         4: (0.5323, 0.0, 1.206, 0.3)}
    xj = yj = 0.5
    # The reference tests the quadrants in the order 1, 2, 3, 4 with >= / <=.
    quad = np.where((x >= xj) & (y >= yj), 1,
                    np.where((x <= xj) & (y >= yj), 2, np.where((x <= xj) & (y <= yj), 3, 4)))
    rho = np.choose(quad - 1, [q[k][0] for k in (1, 2, 3, 4)]).astype(np.float64)
    u = np.choose(quad - 1, [q[k][1] for k in (1, 2, 3, 4)]).astype(np.float64)
    v = np.choose(quad - 1, [q[k][2] for k in (1, 2, 3, 4)]).astype(np.float64)
    p = np.choose(quad - 1, [q[k][3] for k in (1, 2, 3, 4)]).astype(np.float64)
    e = p / ((eos.gamma - 1.0) * rho)  # ideal_gas.cpp:50-57
    return Workload("riemann2d_case3", gen, eos, (rho, u, v, p, e))


def _fourier(seed: int, cx, cy, modes: int = 8):
    rng = np.random.default_rng(seed)
    f = np.zeros((cx.size, cy.size))
    for m in range(1, modes + 1):
        a = rng.uniform(0.0, 1.0) / 8.0
        phi = rng.uniform(0.0, 2.0 * np.pi)
        psi = rng.uniform(0.0, 2.0 * np.pi)
        f += a * np.outer(np.sin(2.0 * np.pi * m * cx + phi), np.sin(2.0 * np.pi * m * cy + psi))
    return f.reshape(-1)


def fourier_smooth(n: int = 2048) -> Workload:
    gen = Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Boundaries(Boundary.PERIODIC, Boundary.PERIODIC, Boundary.PERIODIC, Boundary.PERIODIC))
    gen.set_nx(n)
    eos = IdealGas(1.4)
    cx, cy = _centres(gen)
    rho = 1.0 + 0.2 * _fourier(1, cx, cy)
    u = 0.3 * _fourier(2, cx, cy)
    v = 0.3 * _fourier(3, cx, cy)
    p = 1.0 + 0.1 * _fourier(4, cx, cy)
    e = p / ((eos.gamma - 1.0) * rho)
    return Workload("fourier_smooth", gen, eos, (rho, u, v, p, e))


@dataclass
class MmWorkload:
    name: str
    nx: int
    ny: int
    box: tuple        # x_min, x_max, y_min, y_max
    bounds: tuple     # left, right, bottom, top (zephyr Boundary codes)
    materials: tuple  # (kind, name) per material, e.g. ("stiffened", "Water")
    rho: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    p: np.ndarray
    beta: np.ndarray  # mass fractions, (n_cells, 4)


def shock_water_column(n: int = 1024, sub: int = 8) -> MmWorkload:
    """Two-material shock / water-column interaction on [0, 0.1]^2 m.

    Material 0 is water (StiffenedGas "Water": gamma 4.4, P0 6e8 Pa), material
    1 air (IdealGas "Air": gamma 1.4).  A water column of radius 0.01 m sits at
    the centre at rest in air (rho 1.2 kg/m^3, p 1e5 Pa); a planar shock in the
    air with post-shock pressure 1e6 Pa (Rankine-Hugoniot state) starts at
    x = 0.005 m and moves in +x.  Left/right boundaries ZOE, bottom/top WALL.
    Cells cut by the column get the water volume fraction alpha from sub x sub
    sample points, density alpha rho_w + (1 - alpha) rho_a and the matching
    mass fractions; energy, temperature and true densities then come from the
    mixture closure when the states are loaded."""
    box = (0.0, 0.1, 0.0, 0.1)
    h = (box[1] - box[0]) / n
    xc = box[0] + (np.arange(n) + 0.5) * h
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")  # cell ic = i * n + j
    x, y = xc[i].ravel(), xc[j].ravel()
    # water volume fraction by sub-sampling
    s = (np.arange(sub) + 0.5) / sub - 0.5
    inside = np.zeros(n * n)
    for a in s:
        for b in s:
            inside += ((x + a * h - 0.05) ** 2 + (y + b * h - 0.05) ** 2) < 0.01 ** 2
    alpha = inside / (sub * sub)
    g, p1, rho1, p2 = 1.4, 1.0e5, 1.2, 1.0e6
    rho2 = rho1 * ((g + 1) * p2 + (g - 1) * p1) / ((g - 1) * p2 + (g + 1) * p1)
    u2 = (p2 - p1) / np.sqrt((p2 - p1) / (1 / rho1 - 1 / rho2))
    shocked = x < 0.005
    rho_a = np.where(shocked, rho2, rho1)
    rho_w = 1000.0
    rho = alpha * rho_w + (1 - alpha) * rho_a
    beta = np.zeros((n * n, 4))
    beta[:, 0] = alpha * rho_w / rho
    beta[:, 1] = 1.0 - beta[:, 0]
    beta[alpha >= 1.0, :2] = (1.0, 0.0)
    beta[alpha <= 0.0, :2] = (0.0, 1.0)
    vx = np.where(shocked & (alpha <= 0.0), u2, 0.0)
    p = np.where(shocked & (alpha <= 0.0), p2, p1)
    return MmWorkload("shock_water_column", n, n, box, (2, 2, 1, 1), (("stiffened", "Water"), ("ideal", "Air")),
                      rho, vx, np.zeros(n * n), p, beta)


BLAST_R0 = 0.01
BLAST_P_IN, BLAST_P_OUT = 1.0e3, 1.0e-5


def blast_cell_means(map_x, map_y, n_sub: int = 20, gamma: float = 1.4):
    """(rho, vx, vy, p, e) of the blast for cells given by their 9 map points
    (axis-aligned rectangles: corners at map points 0 and 8).  The mean total
    energy of a cell is the sub-sample mean of p / (gamma - 1); cells the
    circle does not cross take the centre value."""
    x0, x1 = map_x[0::9], map_x[8::9]
    y0, y1 = map_y[0::9], map_y[8::9]
    n = x0.size
    # distance range of each rectangle from the centre
    dx_near = np.maximum(np.maximum(0.5 - x1, x0 - 0.5), 0.0)
    dy_near = np.maximum(np.maximum(0.5 - y1, y0 - 0.5), 0.0)
    dx_far = np.maximum(np.abs(x0 - 0.5), np.abs(x1 - 0.5))
    dy_far = np.maximum(np.abs(y0 - 0.5), np.abs(y1 - 0.5))
    r_near, r_far = np.hypot(dx_near, dy_near), np.hypot(dx_far, dy_far)
    frac = (r_far < BLAST_R0).astype(np.float64)
    cut = np.where((r_near < BLAST_R0) & (r_far >= BLAST_R0))[0]
    if cut.size:
        t = (np.arange(n_sub) + 0.5) / n_sub
        sx = x0[cut, None] + (x1 - x0)[cut, None] * t[None, :]
        sy = y0[cut, None] + (y1 - y0)[cut, None] * t[None, :]
        inside = np.hypot(sx[:, :, None] - 0.5, sy[:, None, :] - 0.5) < BLAST_R0
        frac[cut] = inside.mean(axis=(1, 2))
    E = (frac * BLAST_P_IN + (1.0 - frac) * BLAST_P_OUT) / (gamma - 1.0)
    rho = np.ones(n)
    p = (gamma - 1.0) * E
    return rho, np.zeros(n), np.zeros(n), p, p / ((gamma - 1.0) * rho)


def transfer_disks(nx: int, ny: int, box=(0.0, 1.0, 0.0, 0.7), disks=((0.15, 0.5, 0.1),), sub: int = 8) -> np.ndarray:
    """Volume fraction of the union of `disks` (cx, cy, R) in every cell of the
    nx by ny rectangle `box` (cell order ic = i * ny + j); cells a circle
    crosses are sampled at sub x sub midpoints."""
    x0, x1, y0, y1 = box
    X = x0 + ((x1 - x0) * np.arange(nx + 1)) / nx
    Y = y0 + ((y1 - y0) * np.arange(ny + 1)) / ny
    u = np.zeros((nx, ny))
    t = (np.arange(sub) + 0.5) / sub
    for cx, cy, R in disks:
        i0 = max(int(np.searchsorted(X, cx - R)) - 1, 0)
        i1 = min(int(np.searchsorted(X, cx + R)) + 1, nx)
        j0 = max(int(np.searchsorted(Y, cy - R)) - 1, 0)
        j1 = min(int(np.searchsorted(Y, cy + R)) + 1, ny)
        if i0 >= i1 or j0 >= j1:
            continue
        xa, xb = X[i0:i1][:, None], X[i0 + 1:i1 + 1][:, None]
        ya, yb = Y[j0:j1][None, :], Y[j0 + 1:j1 + 1][None, :]
        # nearest and farthest point of each cell from the centre
        dnx = np.maximum(np.maximum(xa - cx, cx - xb), 0.0)
        dny = np.maximum(np.maximum(ya - cy, cy - yb), 0.0)
        dfx = np.maximum(np.abs(xa - cx), np.abs(xb - cx))
        dfy = np.maximum(np.abs(ya - cy), np.abs(yb - cy))
        near = dnx ** 2 + dny ** 2
        far = dfx ** 2 + dfy ** 2
        blk = u[i0:i1, j0:j1]
        blk[far <= R * R] = 1.0
        cut = np.argwhere((near < R * R) & (far > R * R))
        for a, b in cut:
            sx = X[i0 + a] + (X[i0 + a + 1] - X[i0 + a]) * t
            sy = Y[j0 + b] + (Y[j0 + b + 1] - Y[j0 + b]) * t
            inside = (sx[:, None] - cx) ** 2 + (sy[None, :] - cy) ** 2 < R * R
            blk[a, b] = max(blk[a, b], inside.mean())
    return np.ascontiguousarray(u.ravel())


def transfer_disk_field(nx: int, ny: int, box=(0.0, 1.0, 0.0, 1.0), count: int = 64, seed: int = 7,
                        sub: int = 8) -> np.ndarray:
    """A seeded field of `count` disks (radii 0.01-0.04) for the transport
    benchmark: more interface than the single disk at the same size."""
    rng = np.random.default_rng(seed)
    x0, x1, y0, y1 = box
    disks = [(x0 + (x1 - x0) * (0.1 + 0.8 * rng.random()), y0 + (y1 - y0) * (0.1 + 0.8 * rng.random()),
              0.01 + 0.03 * rng.random()) for _ in range(count)]
    return transfer_disks(nx, ny, box, disks, sub)
