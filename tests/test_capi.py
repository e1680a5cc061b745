"""The C-ABI library: builds, loads, exports every declared entry point, and
rejects bad input before touching a device (no compute calls here)."""
import ctypes as C
import os
import re

import pytest

from ns3d_wcns_b200 import _lib, build
from ns3d_wcns_b200.config import make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ns3d_b200.h")


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ns3d_[a-z0-9_]+)\s*\(", text)))


def test_header_lists_match_binding():
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), name


def test_defaults_and_status_strings(lib):
    p = _lib.Params()
    lib.ns3d_params_default(C.byref(p))
    assert p.gamma == 1.4 and p.sutherland_s == 110.4 / 288.15 and p.dt_fixed == -1.0
    assert list(p.bc) == [0] * 6 and p.precision == 0
    assert lib.ns3d_status_string(0) == b"ok"
    assert lib.ns3d_status_string(-5) == b"non-finite state"


def _create(lib, grid=(8, 8, 8, 0, 0, 0, 1, 1, 1), **kw):
    p = _lib.Params()
    lib.ns3d_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    g = _lib.Grid(*grid)
    h = C.c_void_p()
    return lib.ns3d_create(C.byref(p), C.byref(g), C.byref(h)), h


@pytest.mark.parametrize("grid,why", [
    ((2, 8, 8, 0, 0, 0, 1, 1, 1), b"at least 3"),          # narrower than the WCNS stencil's ghost layers
    ((8, 8, 0, 0, 0, 0, 1, 1, 1), b"at least 3"),          # empty
    ((-4, 8, 8, 0, 0, 0, 1, 1, 1), b"at least 3"),
    ((2048, 2048, 1024, 0, 0, 0, 1, 1, 1), b"too large"),  # beyond 2^31 cells
    ((8, 8, 8, 0, 0, 0, 1, 0, 1), b"positive"),            # zero domain length
])
def test_bad_grids_rejected_before_device(lib, grid, why):
    r, h = _create(lib, grid=grid)
    assert r == -2 and not h.value
    assert why in lib.ns3d_last_error(None)


@pytest.mark.parametrize("field,value", [("gamma", 1.0), ("Ma", 0.0), ("Re", -1.0), ("Pr", 0.0)])
def test_bad_physical_constants_rejected(lib, field, value):
    r, h = _create(lib, **{field: value})
    assert r == -2 and not h.value
    assert b"physical" in lib.ns3d_last_error(None)


def test_zero_interpolation_rejected_before_device(lib):
    r, h = _create(lib, interpolation=1)
    assert r == -2 and not h.value
    assert b"ZERO" in lib.ns3d_last_error(None)


def test_invalid_enums_rejected(lib):
    assert _create(lib, riemann_solver=9)[0] == -2
    assert _create(lib, precision=3)[0] == -2
    assert lib.ns3d_create(None, None, None) == -1


def test_null_handle_calls(lib):
    assert lib.ns3d_rk3_step(None, C.c_double(1e-3)) == -1
    assert lib.ns3d_destroy(None) == -1
    x = C.c_double()
    assert lib.ns3d_compute_timestep(None, C.byref(x)) == -1


def test_no_cpu_fallback(lib):
    from conftest import GPU
    if GPU:
        pytest.skip("device present")
    from ns3d_wcns_b200.solver import Solver
    P, G = make_params(n=(8, 8, 8))
    with pytest.raises(_lib.Ns3dError):
        Solver(P, G)
