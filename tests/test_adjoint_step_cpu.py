"""CPU check of the adjoint assembly: the loop-based reference of one step and
its adjoint (tests/adjoint_reference.py) against central finite differences
on a small smooth periodic 2-D state."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from adjoint_reference import NG, Ref

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("adjstep") / "libadjcheck.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "heraclespp_b200" / "csrc"),
                    str(ROOT / "tests" / "adjoint_cell_check.cpp"), "-o", str(out)], check=True)
    L = C.CDLL(str(out))
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.t_riemann_fwd.argtypes = [i, i, d, vp, vp, i, vp]
    L.t_riemann_rev.argtypes = [i, i, d, vp, vp, i, vp, vp, vp]
    L.t_flux_fwd.argtypes = [d, vp, i, vp]
    L.t_flux_rev.argtypes = [d, vp, i, vp, vp]
    L.t_p2c_fwd.argtypes = [d, vp, vp]
    L.t_p2c_rev.argtypes = [d, vp, vp, vp]
    L.t_c2p_fwd.argtypes = [d, vp, vp]
    L.t_c2p_rev.argtypes = [d, vp, vp, vp]
    L.t_limiter.argtypes = [i, d, d, C.POINTER(d), C.POINTER(d)]
    L.t_limiter.restype = d
    return L


def smooth_state(n, seed=0):
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    rho = 1 + 0.2 * np.sin(2 * np.pi * X + 0.3) * np.cos(2 * np.pi * Y + 0.7) + 0.05 * rng.uniform(-1, 1, (n, n))
    u = 0.3 * np.sin(2 * np.pi * Y + 0.1) + 0.05 * rng.uniform(-1, 1, (n, n))
    v = 0.2 * np.cos(2 * np.pi * X + 0.5) + 0.05 * rng.uniform(-1, 1, (n, n))
    P = 1 + 0.1 * np.cos(2 * np.pi * (X + Y)) + 0.05 * rng.uniform(-1, 1, (n, n))
    gamma = 1.4
    U = np.zeros((4, n + 2 * NG, n + 2 * NG))
    s = (slice(NG, NG + n), slice(NG, NG + n))
    U[0][s] = rho
    U[1][s] = rho * u
    U[2][s] = rho * v
    U[3][s] = P / (gamma - 1) + 0.5 * rho * (u * u + v * v)
    Ref.fill_periodic(U)
    return U


@pytest.mark.parametrize("lim,solver", [(1, 1), (2, 0), (3, 1)])
def test_one_step_adjoint_matches_fd(lib, lim, solver):
    n = 6
    ref = Ref(lib, lim=lim, solver=solver)
    U = smooth_state(n, seed=lim)
    dt, dx = 0.02, (1.0 / n, 1.0 / n)
    rng = np.random.default_rng(5)
    lam = np.zeros_like(U)
    lam[:, NG:NG + n, NG:NG + n] = rng.normal(size=(4, n, n))
    g = ref.step_adjoint(U, lam, dt, dx)

    def J(Ux):
        Ux = Ux.copy()
        Ref.fill_periodic(Ux)
        out = ref.step(Ux, dt, dx)
        return float(np.sum(lam[:, NG:NG + n, NG:NG + n] * out[:, NG:NG + n, NG:NG + n]))

    for _ in range(4):
        v = np.zeros_like(U)
        v[:, NG:NG + n, NG:NG + n] = rng.uniform(-1, 1, (4, n, n))
        eps = 1e-6
        fd = (J(U + eps * v) - J(U - eps * v)) / (2 * eps)
        ad = float(np.sum(g * v))
        assert ad == pytest.approx(fd, rel=1e-6, abs=1e-9)
