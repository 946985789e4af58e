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
