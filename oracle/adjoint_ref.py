"""CPU restatement of the adjoint mode's forward (TEST INFRASTRUCTURE ONLY):
Heun steps at a fixed dt on a uniform periodic rectangle with limited
least-squares slopes (smooth van Albada limiter), HLLC fluxes with Davis wave
speeds, ideal gas; J = mean pressure over the probe box.  numpy, vectorised;
used to pin the GPU forward of zg_adj_forward."""
from __future__ import annotations

import numpy as np


def prim(U, gamma):
    r, mx, my, E = U
    return np.array([r, mx / r, my / r, (gamma - 1.0) * (E - 0.5 * ((mx * mx + my * my) / r))])


def slope(wm, w0, wp, inv2h, eps):
    # (phi(-dL, dR) dR - phi(-dR, dL) dL) / (2h) with phi(a, b) = (a (a + b) + eps) / (a^2 + b^2 + eps):
    # both limiter values share the denominator dL^2 + dR^2 + eps
    a, b = wm - w0, wp - w0
    return inv2h * ((a - b) * (2.0 * a * b - eps)) / (a * a + b * b + eps)


def phys(r, u, v, p, rE):
    return np.array([r * u, r * u * u + p, r * u * v, (rE + p) * u])


def hllc(L, R, gamma):
    rL, uL, vL, pL = L
    rR, uR, vR, pR = R
    gm1 = gamma - 1.0
    rEL = pL / gm1 + 0.5 * (rL * (uL * uL + vL * vL))
    rER = pR / gm1 + 0.5 * (rR * (uR * uR + vR * vR))
    cL, cR = np.sqrt(gamma * pL / rL), np.sqrt(gamma * pR / rR)
    SL = np.minimum(uL - cL, uR - cR)
    SR = np.maximum(uL + cL, uR + cR)
    FL, FR = phys(rL, uL, vL, pL, rEL), phys(rR, uR, vR, pR, rER)
    with np.errstate(all="ignore"):
        aL, aR = rL * (SL - uL), rR * (SR - uR)
        SC = (pL - pR + aR * uR - aL * uL) / (aR - aL)
        rsL, rsR = aL / (SL - SC), aR / (SR - SC)
        EsL = rEL / rL + (SC - uL) * (SC + pL / aL)
        EsR = rER / rR + (SC - uR) * (SC + pR / aR)
        QL = np.array([rL, rL * uL, rL * vL, rEL])
        QR = np.array([rR, rR * uR, rR * vR, rER])
        QsL = np.array([rsL, rsL * SC, rsL * vL, rsL * EsL])
        QsR = np.array([rsR, rsR * SC, rsR * vR, rsR * EsR])
        F = 0.5 * (FL + FR + SL * (QsL - QL) + np.abs(SC) * (QsL - QsR) + SR * (QsR - QR))
    F = np.where(SL >= 0.0, FL, np.where(SR <= 0.0, FR, F))
    return F


def operator(U, gamma, hx, hy, eps):
    W = prim(U, gamma)
    gx = slope(np.roll(W, 1, axis=1), W, np.roll(W, -1, axis=1), 0.5 / hx, eps)
    gy = slope(np.roll(W, 1, axis=2), W, np.roll(W, -1, axis=2), 0.5 / hy, eps)
    # x faces between i and i + 1
    a = W + gx * (0.5 * hx)
    b = np.roll(W - gx * (0.5 * hx), -1, axis=1)
    Fx = hllc(a, b, gamma)
    # y faces between j and j + 1, face frame (rho, v, -u, p)
    a = W + gy * (0.5 * hy)
    b = np.roll(W - gy * (0.5 * hy), -1, axis=2)
    Fl = hllc(np.array([a[0], a[2], -a[1], a[3]]), np.array([b[0], b[2], -b[1], b[3]]), gamma)
    Fy = np.array([Fl[0], -Fl[2], Fl[1], Fl[3]])
    div = hy * (Fx - np.roll(Fx, 1, axis=1)) + hx * (Fy - np.roll(Fy, 1, axis=2))
    return -div / (hx * hy)


def run(rho, u, v, p, nx, ny, box=(0.0, 1.0, 0.0, 1.0), gamma=1.4, dt=1e-3, steps=10, eps=1e-8,
        probe=(0.6, 0.7, 0.6, 0.7)):
    """J after `steps` Heun steps from the primitive initial state (flat
    arrays, cell (i, j) at i * ny + j)."""
    hx, hy = (box[1] - box[0]) / nx, (box[3] - box[2]) / ny
    sh = (nx, ny)
    r, uu, vv, pp = (np.asarray(a, float).reshape(sh) for a in (rho, u, v, p))
    U = np.array([r, r * uu, r * vv, pp / (gamma - 1.0) + 0.5 * (r * (uu * uu + vv * vv))])
    for _ in range(steps):
        Us = U + dt * operator(U, gamma, hx, hy, eps)
        U = 0.5 * U + 0.5 * Us + 0.5 * dt * operator(Us, gamma, hx, hy, eps)
    P = prim(U, gamma)[3]
    cx = box[0] + (np.arange(nx) + 0.5) * hx
    cy = box[2] + (np.arange(ny) + 0.5) * hy
    mask = ((cx[:, None] >= probe[0]) & (cx[:, None] <= probe[1]) & (cy[None, :] >= probe[2]) &
            (cy[None, :] <= probe[3]))
    return float(P[mask].sum() / mask.sum()), U
