"""CPU checks of the C ABI library: it loads, exports every entry point that
include/heracles_b200.h declares, reports errors without a device, and its
host-only setup plugins agree with the Python mirror."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "heracles_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(hcl_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from heraclespp_b200 import lib
    from heraclespp_b200._native import EXPORTS

    L = lib()
    declared = declared_functions()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(L, name), name
    # the Python binding covers the stage and fused entry points
    for name in EXPORTS:
        assert name in declared, name


def test_abi_version_and_errors_without_device():
    from heraclespp_b200 import lib
    from heraclespp_b200._native import Config

    L = lib()
    assert L.hcl_abi_version() == 4
    cfg = Config()
    L.hcl_config_default(C.byref(cfg))
    # reference defaults (utils/param.cpp): gamma 5/3, VanLeer, HLL, Nghost 2
    assert cfg.gamma == 5.0 / 3.0 and cfg.limiter == 1 and cfg.riemann == 0 and cfg.nghost == 2
    h = C.c_void_p()
    cfg.gamma = 1.0
    rc = L.hcl_create(C.byref(cfg), C.byref(h))
    assert rc == 2  # HCL_ERR_DOMAIN, perfect_gas.cpp:15-17
    assert b"Invalid gamma" in L.hcl_last_error()
    cfg.gamma = 1.4
    cfg.mmw = 0.0
    assert L.hcl_create(C.byref(cfg), C.byref(h)) == 2
    assert b"Invalid mmw" in L.hcl_last_error()


def _host_setup(name, ndim, nx, ini=None, xmax=(1.0, 1.0, 1.0)):
    from heraclespp_b200 import lib, setups
    from oracle import Oracle

    o = Oracle(ndim, nx, xmax=xmax)
    grid = setups.Grid.from_domain(o)
    n = o.n
    rho, u, P = np.zeros(o.shape3), np.zeros((ndim,) + o.shape3), np.zeros(o.shape3)
    xc = [np.ascontiguousarray(grid.xc[d]) for d in range(3)]
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    L = lib()
    L.hcl_setup_initial_prim.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int * 3, C.c_int] + [C.c_void_p] * 6
    rc = L.hcl_setup_initial_prim(name.encode(), ini.encode() if ini else None, ndim, (C.c_int * 3)(*n), 2,
                                  vp(xc[0]), vp(xc[1]), vp(xc[2]), vp(rho), vp(u), vp(P))
    assert rc == 0, L.hcl_last_error()
    return grid, (rho, u, P)


@pytest.mark.parametrize("name,ndim,nx,xmax", [
    ("kelvin_helmholtz", 2, [40, 24], (1.0, 1.0, 1.0)),
    ("rayleigh_taylor3d", 3, [8, 8, 16], (0.5, 0.5, 1.0)),
    ("gresho_vortex", 2, [32, 32], (1.0, 1.0, 1.0)),
    ("four_quadrant", 2, [20, 20], (1.0, 1.0, 1.0)),
    ("advection_sinus", 1, [50], (1.0, 1.0, 1.0)),
])
def test_cpp_setups_match_python(name, ndim, nx, xmax):
    from heraclespp_b200 import setups

    grid, (rho, u, P) = _host_setup(name, ndim, nx, xmax=xmax)
    kw = {"advection_sinus": {"u0": 1.0, "P0": 1.0}}.get(name, {})
    prho, pu, pP = setups.SETUPS[name](grid, **kw)
    np.testing.assert_allclose(rho, prho, rtol=1e-15, atol=0)
    np.testing.assert_allclose(P, pP, rtol=1e-14, atol=0)
    np.testing.assert_allclose(u, pu, rtol=1e-13, atol=1e-16)


def test_shock_tube_reads_ini(tmp_path):
    from heraclespp_b200 import setups

    ini = tmp_path / "st.ini"
    ini.write_text("[Initialisation]\nrho0 = 1\nrho1 = 0.125 ; inline comment\nu0 = 0\nu1 = 0\nP0 = 1\n"
                   "P1 = 0.1\nINTER = 0.5\n")
    grid, (rho, u, P) = _host_setup("shock_tube", 1, [64], ini=str(ini))
    prho, pu, pP = setups.shock_tube(grid)
    assert np.array_equal(rho, prho) and np.array_equal(P, pP) and np.array_equal(u, pu)


def test_unknown_setup_is_an_error():
    from heraclespp_b200 import lib

    L = lib()
    n = (C.c_int * 3)(8, 1, 1)
    z = np.zeros(8)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = L.hcl_setup_initial_prim(b"nope", None, 1, n, 2, vp(z), vp(z), vp(z), vp(z), vp(z), vp(z))
    assert rc == 1 and b"Setup not implemented" in L.hcl_last_error()
