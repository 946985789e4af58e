"""Adjoint mode over the C ABI (``zg_adj_*``; no counterpart in the
reference): J = mean pressure over a probe box after Heun steps at a fixed dt
on a uniform periodic rectangle, and its gradient with respect to the initial
density field and gamma by a discrete adjoint with checkpoints.

Fields are CUDA tensors (float64, nx * ny cells, cell (i, j) at i * ny + j),
passed to the library as device pointers; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

from ._lib import AdjParams, ZgError, load


class Adjoint:
    def __init__(self, nx, ny, box=(0.0, 1.0, 0.0, 1.0), device=0, stream=None):
        self._lib = load()
        self.h = C.c_void_p()
        rc = self._lib.zg_adj_create(C.byref(self.h), device, nx, ny, *box)
        if rc != 0:
            raise ZgError(rc, "zg_adj_create failed")
        self.nx, self.ny = nx, ny
        if stream is not None:
            self._lib.zg_adj_set_stream(self.h, C.c_void_p(stream))

    @staticmethod
    def params(steps=100, checkpoint_every=10, gamma=1.4, dt=0.0, limiter_eps=1e-8, probe=(0.6, 0.7, 0.6, 0.7),
               precision=0):
        """zg_adj_params; precision 0 = FP64, 1 = MIXED (zg_precision)."""
        p = AdjParams()
        load().zg_adj_default_params(C.byref(p))
        p.steps, p.checkpoint_every, p.gamma, p.dt, p.limiter_eps = steps, checkpoint_every, gamma, dt, limiter_eps
        p.precision = int(precision)
        for k in range(4):
            p.probe[k] = probe[k]
        return p

    def _check(self, rc):
        if rc != 0:
            raise ZgError(rc, (self._lib.zg_adj_last_error(self.h) or b"").decode())

    @staticmethod
    def _ptrs(*ts):
        for t in ts:
            if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float64"):
                raise ValueError("fields must be contiguous float64 CUDA tensors")
        return [C.c_void_p(t.data_ptr()) for t in ts]

    def cfl_dt(self, gamma, CFL, rho, u, v, p):
        dt = C.c_double()
        self._check(self._lib.zg_adj_cfl_dt(self.h, gamma, CFL, *self._ptrs(rho, u, v, p), C.byref(dt)))
        return dt.value

    def forward(self, prm, rho, u, v, p):
        J = C.c_double()
        self._check(self._lib.zg_adj_forward(self.h, C.byref(prm), *self._ptrs(rho, u, v, p), C.byref(J)))
        return J.value

    def gradient(self, prm, rho, u, v, p, grad_rho):
        """J, fills grad_rho (CUDA tensor like rho) and returns (J, dJ/dgamma)."""
        J, gg = C.c_double(), C.c_double()
        ptrs = self._ptrs(rho, u, v, p, grad_rho)
        self._check(self._lib.zg_adj_gradient(self.h, C.byref(prm), *ptrs[:4], C.byref(J), ptrs[4], C.byref(gg)))
        return J.value, gg.value

    def launch_count(self):
        n = C.c_longlong()
        self._lib.zg_adj_launch_count(self.h, C.byref(n))
        return n.value

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self._lib.zg_adj_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
