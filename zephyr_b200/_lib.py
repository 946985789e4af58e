"""ctypes binding of ``libzephyr_gpu.so`` (the C ABI in include/zephyr_gpu.h).

The shared library is built in-tree by ``zephyr_b200.build``.  There is no
fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libzephyr_gpu.so"

ZG_OK = 0
_ERR_NAMES = {-1: "ZG_ERR_ARG", -2: "ZG_ERR_CUDA", -3: "ZG_ERR_STATE", -4: "ZG_ERR_ALLOC", -5: "ZG_ERR_NUMERIC",
              -6: "ZG_ERR_TOO_LARGE"}


class ZgError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {message}")
        self.code = code


class SmfParams(C.Structure):
    _fields_ = [
        ("eos_kind", C.c_int),
        ("gamma", C.c_double),
        ("P0", C.c_double),
        ("e0", C.c_double),
        ("flux", C.c_int),
        ("limiter", C.c_int),
        ("accuracy", C.c_int),
        ("scheme", C.c_int),
        ("precision", C.c_int),
        ("kernels", C.c_int),
        ("CFL", C.c_double),
        ("max_dt", C.c_double),
    ]


class MeshView(C.Structure):
    _fields_ = [(n, t) for n, t in (
        ("n_cells", C.c_int),
        ("center_x", C.POINTER(C.c_double)), ("center_y", C.POINTER(C.c_double)),
        ("volume", C.POINTER(C.c_double)), ("incircle", C.POINTER(C.c_double)),
        ("face_boundary", C.POINTER(C.c_int)), ("face_neib", C.POINTER(C.c_int)),
        ("face_nx", C.POINTER(C.c_double)), ("face_ny", C.POINTER(C.c_double)),
        ("face_cx", C.POINTER(C.c_double)), ("face_cy", C.POINTER(C.c_double)),
        ("face_area", C.POINTER(C.c_double)))]


_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_V = C.c_void_p


class AmrStats(C.Structure):
    """zg_amr_stats"""
    _fields_ = [(n, C.c_int) for n in ("max_level", "capacity", "n_before", "n_after", "n_coarse", "n_refine",
                                        "n_large")]


class AmrCells(C.Structure):
    """zg_amr_cells (host arrays; NULL members are skipped)"""
    _fields_ = [(n, t) for n, t in (
        ("center_x", _P), ("center_y", _P), ("volume", _P), ("incircle", _P), ("map_x", _P), ("map_y", _P),
        ("level", _I), ("flag", _I), ("b_idx", _I), ("z_idx", _I), ("face_boundary", _I), ("face_neib", _I),
        ("face_nx", _P), ("face_ny", _P), ("face_cx", _P), ("face_cy", _P), ("face_area", _P))]

# name -> (restype, argtypes); every symbol include/zephyr_gpu.h declares.
class Material(C.Structure):
    """zg_material"""
    _fields_ = [("kind", C.c_int), ("gamma", C.c_double), ("P0", C.c_double), ("e0", C.c_double),
                ("Cv", C.c_double), ("T0", C.c_double), ("rho_ref", C.c_double)]


class MmfParams(C.Structure):
    """zg_mmf_params"""
    _fields_ = [("n_materials", C.c_int), ("materials", Material * 4), ("crp_mode", C.c_int),
                ("accuracy", C.c_int), ("CFL", C.c_double), ("max_dt", C.c_double), ("split", C.c_int),
                ("precision", C.c_int), ("limiter", C.c_int)]


class TrParams(C.Structure):
    """zg_tr_params"""
    _fields_ = [("method", C.c_int), ("CFL", C.c_double), ("velocity", C.c_int), ("vel", C.c_double * 3)]


class OutVar(C.Structure):
    """zg_out_var"""
    _fields_ = [("name", C.c_char_p), ("source", C.c_int), ("component", C.c_int), ("host", C.POINTER(C.c_double))]


class AdjParams(C.Structure):
    """zg_adj_params"""
    _fields_ = [("gamma", C.c_double), ("dt", C.c_double), ("steps", C.c_int), ("checkpoint_every", C.c_int),
                ("limiter_eps", C.c_double), ("probe", C.c_double * 4), ("precision", C.c_int)]


SIGNATURES = {
    "zg_smf_default_params": (None, [C.POINTER(SmfParams)]),
    "zg_limiter_from_name": (C.c_int, [C.c_char_p]),
    "zg_create": (C.c_int, [C.POINTER(_V), C.c_int]),
    "zg_destroy": (C.c_int, [_V]),
    "zg_last_error": (C.c_char_p, [_V]),
    "zg_set_stream": (C.c_int, [_V, _V]),
    "zg_mesh_rectangle": (C.c_int, [_V, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _I]),
    "zg_mesh_n_cells": (C.c_int, [_V, _I]),
    "zg_mesh_upload": (C.c_int, [_V, C.POINTER(MeshView)]),
    "zg_mesh_set_axial": (C.c_int, [_V, _P, _P]),
    "zg_amr_enable": (C.c_int, [_V, C.c_int, C.c_int]),
    "zg_amr_set_distributor": (C.c_int, [_V, C.c_int]),
    "zg_amr_put_flags": (C.c_int, [_V, _I]),
    "zg_amr_set_flags_gradient": (C.c_int, [_V, C.c_double, C.c_double, _I]),
    "zg_amr_refine": (C.c_int, [_V]),
    "zg_amr_info": (C.c_int, [_V, C.POINTER(AmrStats)]),
    "zg_amr_download": (C.c_int, [_V, C.POINTER(AmrCells)]),
    "zg_smf_configure": (C.c_int, [_V, C.POINTER(SmfParams)]),
    "zg_smf_set_max_dt": (C.c_int, [_V, C.c_double]),
    "zg_state_upload": (C.c_int, [_V, _P, _P, _P, _P, _P]),
    "zg_state_download": (C.c_int, [_V, _P, _P, _P, _P, _P]),
    "zg_wait_upload": (C.c_int, [_V, _I]),
    "zg_wait_download": (C.c_int, [_V, _I]),
    "zg_smf_update": (C.c_int, [_V]),
    "zg_smf_update_n": (C.c_int, [_V, C.c_int]),
    "zg_smf_dt": (C.c_int, [_V, _P]),
    "zg_smf_set_flags": (C.c_int, [_V, _I]),
    "zg_smf_gradients": (C.c_int, [_V, _P, _P]),
    "zg_state_rows": (C.c_int, [_V, C.c_int, C.c_int, _P, _I, C.c_int]),
    "zg_smf_cfl_min": (C.c_int, [_V, _P]),
    "zg_launch_count": (C.c_int, [_V, C.POINTER(C.c_longlong)]),
    "zg_synchronize": (C.c_int, [_V]),
    "zg_set_timing": (C.c_int, [_V, C.c_int]),
    "zg_kernel_times": (C.c_int, [_V, _P, C.POINTER(C.c_longlong)]),
    "zg_kernel_name": (C.c_char_p, [C.c_int]),
    "zg_material_named": (C.c_int, [C.c_int, C.c_char_p, C.POINTER(Material)]),
    "zg_mmf_default_params": (None, [C.POINTER(MmfParams)]),
    "zg_mmf_configure": (C.c_int, [_V, C.POINTER(MmfParams)]),
    "zg_mmf_state_upload": (C.c_int, [_V, _P]),
    "zg_mmf_state_download": (C.c_int, [_V, _P]),
    "zg_mmf_make_states": (C.c_int, [_V, _P, _P, _P, _P, _P]),
    "zg_mmf_update": (C.c_int, [_V]),
    "zg_mmf_update_n": (C.c_int, [_V, C.c_int]),
    "zg_mmf_dt": (C.c_int, [_V, _P]),
    "zg_mmf_set_flags": (C.c_int, [_V, _I]),
    "zg_mmf_grad_a": (C.c_int, [_V, _P]),
    "zg_mmf_interface": (C.c_int, [_V, _P, _P]),
    "zg_tr_default_params": (None, [C.POINTER(TrParams)]),
    "zg_tr_configure": (C.c_int, [_V, C.POINTER(TrParams)]),
    "zg_tr_upload": (C.c_int, [_V, _P]),
    "zg_tr_download": (C.c_int, [_V, _P, _P, _P]),
    "zg_tr_update_interface": (C.c_int, [_V, C.c_int]),
    "zg_tr_compute_dt": (C.c_int, [_V, _P]),
    "zg_tr_set_dt": (C.c_int, [_V, C.c_double]),
    "zg_tr_get_dt": (C.c_int, [_V, _P]),
    "zg_tr_update": (C.c_int, [_V, C.c_int]),
    "zg_tr_advance": (C.c_int, [_V, C.c_int, C.c_int, C.c_double, _P]),
    "zg_tr_set_flags": (C.c_int, [_V, _I]),
    "zg_vtu_write": (C.c_int, [_V, C.c_char_p, C.POINTER(OutVar), C.c_int]),
    "zg_pvd_open": (C.c_int, [C.POINTER(_V), C.c_char_p, C.c_char_p]),
    "zg_pvd_save": (C.c_int, [_V, _V, C.POINTER(OutVar), C.c_int, C.c_double]),
    "zg_pvd_close": (C.c_int, [_V]),
    "zg_adj_default_params": (None, [C.POINTER(AdjParams)]),
    "zg_adj_create": (C.c_int, [C.POINTER(_V), C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                C.c_double]),
    "zg_adj_destroy": (C.c_int, [_V]),
    "zg_adj_last_error": (C.c_char_p, [_V]),
    "zg_adj_set_stream": (C.c_int, [_V, _V]),
    "zg_adj_launch_count": (C.c_int, [_V, C.POINTER(C.c_longlong)]),
    "zg_adj_cfl_dt": (C.c_int, [_V, C.c_double, C.c_double, _V, _V, _V, _V, _P]),
    "zg_adj_forward": (C.c_int, [_V, C.POINTER(AdjParams), _V, _V, _V, _V, _P]),
    "zg_adj_gradient": (C.c_int, [_V, C.POINTER(AdjParams), _V, _V, _V, _V, _P, _V, _P]),
    "zg_rect_step_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, _I, C.POINTER(SmfParams), C.POINTER(_V), C.POINTER(_V), _V,
                                       _V]),
}

# enum zg_kernel_kind
KERNEL_KINDS = ["dt", "flux1", "grad", "stage1", "stage2", "heun_a", "heun_b", "flags", "mm_dt", "mm_recover",
                "mm_flux", "mm_crp", "mm_closure", "tr_dt", "tr_flux", "tr_update", "tr_normals", "tr_adjust",
                "mm_grad", "mm_stage1", "mm_stage2", "step"]

_lib = None


def load():
    """Load the library (once) and declare the signatures."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA extension first "
                "(python -m zephyr_b200.build); there is no CPU fallback")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(ctx, rc: int):
    if rc != ZG_OK:
        msg = load().zg_last_error(ctx) if ctx else b""
        raise ZgError(rc, (msg or b"").decode(errors="replace"))
    return rc
