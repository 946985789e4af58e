"""zephyr_b200 -- zephyr's explicit finite-volume step on one B200.

The CUDA kernels and the C ABI live in ``csrc/`` and build into the in-tree
``libzephyr_gpu.so``; ``smf`` mirrors the reference's SmFluid / EuMesh API on
top of that ABI, and ``workloads`` generates the synthetic initial data.
"""
from ._lib import LIB_PATH, ZgError, load
from .smf import (Boundaries, Boundary, EuMesh, Fluxes, IdealGas, Kernels, Parts, Precision, Rectangle, Scheme,
                  SmFluid, StiffenedGas)

__all__ = [
    "LIB_PATH", "ZgError", "load", "Boundaries", "Boundary", "EuMesh", "Fluxes", "IdealGas", "Kernels", "Parts",
    "Precision", "Rectangle", "Scheme", "SmFluid", "StiffenedGas",
]
