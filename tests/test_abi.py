"""The C ABI library loads, exports every symbol include/zephyr_gpu.h
declares, and its host-only entry points behave (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import pytest

import zephyr_b200 as Z
from zephyr_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "zephyr_gpu.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "zg_smf_update" in names and "zg_create" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = Z.load()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in zephyr_gpu.h but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_default_params_match_smfluid_constructor():
    """sm_fluid.cpp:16-23: HLLC, MC, CFL 0.5, no dt cap; set_accuracy default 1."""
    lib = Z.load()
    p = _lib.SmfParams()
    lib.zg_smf_default_params(C.byref(p))
    assert p.flux == 3 and p.limiter == 3 and p.CFL == 0.5 and p.accuracy == 1
    assert p.max_dt > 1e300 and p.gamma == 1.4 and p.eos_kind == 0


@pytest.mark.parametrize("name,kind", [
    ("MC", 3), ("mc", 3), ("van Albada", 5), ("vanAlbada1", 5), ("van-Albada 2", 6), ("van_albada_2", 6),
    ("minmod", 2), ("MinMod limiter", 2), ("none", 0), ("", 0), ("off", 0), ("unit", 1), ("van Leer", 4),
    ("CHARM", 7), ("HCUS", 8), ("HQUICK", 9), ("Koren", 10), ("smart", 11), ("superbee", 12), ("bogus", -1),
])
def test_limiter_names_follow_reference_parsing(name, kind):
    """limiter.cxx:163-252: lower-case, strip ' ', '-', '_', 'lim', 'limiter',
    then substring tests in the reference's order."""
    assert Z.load().zg_limiter_from_name(name.encode()) == kind


def test_kernel_names():
    lib = Z.load()
    assert [lib.zg_kernel_name(k).decode() for k in range(len(_lib.KERNEL_KINDS))] == _lib.KERNEL_KINDS


def test_null_arguments_are_rejected():
    lib = Z.load()
    assert lib.zg_create(None, 0) == -1
    assert lib.zg_destroy(None) == -1
    assert lib.zg_smf_update(None) == -1


def test_rectangle_sizes_follow_reference():
    """rectangle.cpp:105-133: ny = max(round(nx * H / W), 1)."""
    g = Z.Rectangle(0.0, 2.0, 0.0, 1.0)
    g.set_nx(48)
    assert (g.nx(), g.ny()) == (48, 24)
    g.set_nx(5)
    assert (g.nx(), g.ny()) == (5, 3)  # std::round(2.5) = 3 (half away from zero)
    g = Z.Rectangle(0.0, 1.0, 0.0, 3.0)
    g.set_ny(10)
    assert (g.nx(), g.ny()) == (3, 10)
    with pytest.raises(ValueError):
        g.set_nx(0)


def test_periodic_pairs():
    g = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
    g.set_boundaries(Z.Boundaries(Z.Boundary.PERIODIC, Z.Boundary.WALL, Z.Boundary.ZOE, Z.Boundary.ZOE))
    assert g.bounds.left == g.bounds.right == Z.Boundary.PERIODIC
    assert g.bounds.bottom == Z.Boundary.ZOE


def test_unimplemented_flux_is_refused():
    s = Z.SmFluid(Z.IdealGas(1.4))
    with pytest.raises(Z.ZgError):
        s.set_method(Z.Fluxes.CRP)  # the multi-material composite flux
    with pytest.raises(Z.ZgError):
        s.set_limiter("no-such-limiter")


@pytest.mark.parametrize("kind,name", [(1, "Water"), (0, "Air"), (1, "Air")])
def test_named_materials_match_the_oracle(kind, name):
    """zg_material_named (host only) against the oracle's restatement of
    IdealGas(name) / StiffenedGas(name) with the reference's literals."""
    from oracle import oracle as O
    m = _lib.Material()
    assert Z.load().zg_material_named(kind, name.encode(), C.byref(m)) == 0
    want = O.mm_material("stiffened" if kind == 1 else "ideal", name)
    got = [float(kind), m.gamma, m.P0, m.e0, m.Cv, m.T0, m.rho_ref]
    assert got == list(want)
    assert Z.load().zg_material_named(kind, b"Unobtainium", C.byref(m)) != 0
