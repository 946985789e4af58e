"""TEST INFRASTRUCTURE ONLY: restatement of the adaptive configuration's
refinement criterion for checking the GPU (zg_amr_set_flags_gradient).

The criterion has no counterpart in the reference (its SmFluid::set_flags
uses neighbour jumps, math/solver/sm_fluid.cpp:517-559); the benchmark
defines it: refine where |grad rho| h / rho > 0.05, coarsen where it is
below 0.01, keep otherwise.  Here grad rho is the reference's unlimited
least-squares gradient (math/cfd/gradient.h:226-282, density only, in 2-D:
weights w = S / |dr . n|^3 with dr the vector to the neighbour's centre, or
to the mirror of the cell centre in a boundary face, amr_faces.h:197-199; the
third row and column of the 3x3 system are the identity in 2-D, and a
vanishing A11 is replaced by 1 as in gradient.h:267-273), and h is the
square root of the cell area.

Works on the slot arrays of an adaptive mesh (8 face slots per cell, slot k
of cell i at 8 i + k, boundary code -1 for an undefined slot), as
zephyr_b200.smf.EuMesh.amr_arrays() and oracle.ref_mesh.RefEuMesh return
them.
"""
from __future__ import annotations

import numpy as np

BC_INNER = 0
BC_UNDEFINED = -1


def criterion(mesh: dict, rho) -> np.ndarray:
    """|grad rho| h / rho of every cell."""
    cx, cy = np.asarray(mesh["cx"], float), np.asarray(mesh["cy"], float)
    vol = np.asarray(mesh["vol"], float)
    n = len(cx)
    fb = np.asarray(mesh["boundary"]).reshape(n, 8)
    nb = np.asarray(mesh["neib"]).reshape(n, 8)
    fnx = np.asarray(mesh["nx"], float).reshape(n, 8)
    fny = np.asarray(mesh["ny"], float).reshape(n, 8)
    fcx = np.asarray(mesh["fx"], float).reshape(n, 8)
    fcy = np.asarray(mesh["fy"], float).reshape(n, 8)
    fa = np.asarray(mesh["area"], float).reshape(n, 8)
    rho = np.asarray(rho, float)
    A00 = np.zeros(n)
    A01 = np.zeros(n)
    A10 = np.zeros(n)
    A11 = np.zeros(n)
    Fx = np.zeros(n)
    Fy = np.zeros(n)
    for s in range(8):
        act = fb[:, s] != BC_UNDEFINED
        inner = fb[:, s] == BC_INNER
        periodic_or_boundary = ~inner
        j = np.where(act, nb[:, s], 0)
        # neighbour value: a boundary slot (WALL / ZOE) takes the cell's own
        # density; an inner or periodic slot the neighbour's
        boundary = periodic_or_boundary & (fb[:, s] != 3)
        rn = np.where(boundary, rho, rho[j])
        # neighbour centre: the neighbour's, or the mirror in the face
        d = (fcx[:, s] - cx) * fnx[:, s] + (fcy[:, s] - cy) * fny[:, s]
        mx, my = cx + (2.0 * d) * fnx[:, s], cy + (2.0 * d) * fny[:, s]
        ncx = np.where(inner, cx[j], mx)
        ncy = np.where(inner, cy[j], my)
        rx, ry = ncx - cx, ncy - cy
        dn = rx * fnx[:, s] + ry * fny[:, s]
        nxx, nyy = dn * fnx[:, s], dn * fny[:, s]
        an = np.sqrt(nxx * nxx + nyy * nyy)
        with np.errstate(divide="ignore", invalid="ignore"):
            w = np.where(act, fa[:, s] / (an * an * an), 0.0)
        dF = np.where(act, rn - rho, 0.0)
        A00 += w * nxx * rx
        A01 += w * nxx * ry
        A10 += w * nyy * rx
        A11 += w * nyy * ry
        Fx += w * dF * nxx
        Fy += w * dF * nyy
    A11 = np.where(np.abs(A11) < 1e-8, 1.0, A11)
    inv = 1.0 / (A11 * A00 - A01 * A10)
    gx = (A11 * Fx - A01 * Fy) * inv
    gy = (-A10 * Fx + A00 * Fy) * inv
    return np.sqrt(gx * gx + gy * gy) * np.sqrt(vol) / rho


def flags(mesh: dict, rho, refine: float = 0.05, coarsen: float = 0.01) -> np.ndarray:
    """1 refine, -1 coarsen, 0 keep."""
    c = criterion(mesh, rho)
    return np.where(c > refine, 1, np.where(c < coarsen, -1, 0)).astype(np.int32)
