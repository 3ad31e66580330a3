"""CPU checks of the hand-written reverse-mode pieces of the discrete adjoint
(heraclespp_b200/csrc/adjoint_cell.cuh, compiled here as host C++): every
transpose-Jacobian product against central finite differences, away from the
branch switches (limiter sign test, wave-speed selection, HLLC star side)."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("adj") / "libadjcheck.so"
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
    L.t_sph_src.argtypes = [i, i, vp, vp, vp, vp]
    L.t_sph_src_rev.argtypes = [i, i, vp, vp, vp, vp, vp, vp]
    return L


def p(a):
    return a.ctypes.data_as(C.c_void_p)


def jac_fd(f, x, m, eps=1e-6):
    J = np.zeros((m, x.size))
    for k in range(x.size):
        h = eps * max(1.0, abs(x[k]))
        xp, xm = x.copy(), x.copy()
        xp[k] += h
        xm[k] -= h
        J[:, k] = (f(xp) - f(xm)) / (2 * h)
    return J


def cons_from(prim, gamma):
    nd = prim.size - 2
    U = np.zeros_like(prim)
    U[0] = prim[0]
    U[1:1 + nd] = prim[0] * prim[1:1 + nd]
    U[-1] = prim[-1] / (gamma - 1) + 0.5 * prim[0] * np.sum(prim[1:1 + nd] ** 2)
    return U


@pytest.mark.parametrize("nd", [1, 2, 3])
@pytest.mark.parametrize("solver", [0, 1, 2])
def test_riemann_reverse_matches_fd(lib, nd, solver):
    rng = np.random.default_rng(10 + nd + 3 * solver)
    gamma = 1.4
    checked = 0
    for trial in range(60):
        pl = np.concatenate([[rng.uniform(0.3, 2)], rng.uniform(-1.5, 1.5, nd), [rng.uniform(0.3, 3)]])
        pr = np.concatenate([[rng.uniform(0.3, 2)], rng.uniform(-1.5, 1.5, nd), [rng.uniform(0.3, 3)]])
        UL, UR = cons_from(pl, gamma), cons_from(pr, gamma)
        l = trial % nd
        x = np.concatenate([UL, UR])
        n = nd + 2

        def f(xx):
            out = np.zeros(n)
            a, b = np.ascontiguousarray(xx[:n]), np.ascontiguousarray(xx[n:])
            lib.t_riemann_fwd(nd, solver, gamma, p(a), p(b), l, p(out))
            return out

        J = jac_fd(f, x, n)
        # skip points next to a branch switch (FD straddles the kink)
        J2 = jac_fd(f, x, n, eps=3e-7)
        if np.max(np.abs(J - J2)) > 1e-4 * (1 + np.max(np.abs(J))):
            continue
        Fb = rng.normal(size=n)
        ULb, URb = np.zeros(n), np.zeros(n)
        lib.t_riemann_rev(nd, solver, gamma, p(UL), p(UR), l, p(Fb), p(ULb), p(URb))
        got = np.concatenate([ULb, URb])
        want = J.T @ Fb
        np.testing.assert_allclose(got, want, rtol=2e-6, atol=2e-6 * (1 + np.max(np.abs(want))))
        checked += 1
    assert checked > 40


def test_flux_and_conversions_reverse_match_fd(lib):
    rng = np.random.default_rng(3)
    gamma = 5.0 / 3.0
    for _ in range(30):
        W = np.array([rng.uniform(0.3, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.3, 3)])
        for l in (0, 1):
            def f(ww):
                out = np.zeros(4)
                lib.t_flux_fwd(gamma, p(np.ascontiguousarray(ww)), l, p(out))
                return out

            J = jac_fd(f, W, 4)
            b = rng.normal(size=4)
            got = np.zeros(4)
            lib.t_flux_rev(gamma, p(W), l, p(b), p(got))
            np.testing.assert_allclose(got, J.T @ b, rtol=1e-6, atol=1e-7)

        def g(ww):
            out = np.zeros(4)
            lib.t_p2c_fwd(gamma, p(np.ascontiguousarray(ww)), p(out))
            return out

        J = jac_fd(g, W, 4)
        b = rng.normal(size=4)
        got = np.zeros(4)
        lib.t_p2c_rev(gamma, p(W), p(b), p(got))
        np.testing.assert_allclose(got, J.T @ b, rtol=1e-6, atol=1e-7)

        U = cons_from(W, gamma)

        def h(uu):
            out = np.zeros(4)
            lib.t_c2p_fwd(gamma, p(np.ascontiguousarray(uu)), p(out))
            return out

        J = jac_fd(h, U, 4)
        got = np.zeros(4)
        lib.t_c2p_rev(gamma, p(U), p(b), p(got))
        np.testing.assert_allclose(got, J.T @ b, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("lim", [0, 1, 2, 3])
def test_limiter_partials_match_fd(lib, lim):
    rng = np.random.default_rng(lim)
    for _ in range(200):
        R, L = rng.normal(size=2)
        if abs(R) < 1e-3 or abs(L) < 1e-3 or abs(abs(R) - abs(L)) < 1e-3:
            continue
        gR, gL = C.c_double(), C.c_double()
        lib.t_limiter(lim, R, L, C.byref(gR), C.byref(gL))
        h = 1e-6
        d0, d1 = C.c_double(), C.c_double()
        fR = (lib.t_limiter(lim, R + h, L, C.byref(d0), C.byref(d1)) -
              lib.t_limiter(lim, R - h, L, C.byref(d0), C.byref(d1))) / (2 * h)
        fL = (lib.t_limiter(lim, R, L + h, C.byref(d0), C.byref(d1)) -
              lib.t_limiter(lim, R, L - h, C.byref(d0), C.byref(d1))) / (2 * h)
        assert gR.value == pytest.approx(fR, rel=1e-6, abs=1e-8)
        assert gL.value == pytest.approx(fL, rel=1e-6, abs=1e-8)


@pytest.mark.parametrize("nd", [1, 2, 3])
def test_riemann_forward_forms_equal_the_oracle(lib, nd):
    """The algebra the reverse sweep differentiates (perfect gas P = (gamma-1) e,
    one reciprocal per state) gives the oracle's fluxes up to rounding, for
    HLL, HLLC and the low-Mach splitting solver."""
    from oracle import Oracle

    gamma = 1.4
    o = Oracle(nd, [8] * nd, gamma=gamma)
    rng = np.random.default_rng(40 + nd)
    names = ["HLL", "HLLC", "Low Mach"]
    for trial in range(40):
        pl = np.concatenate([[rng.uniform(0.3, 2)], rng.uniform(-1.5, 1.5, nd), [rng.uniform(0.3, 3)]])
        pr = np.concatenate([[rng.uniform(0.3, 2)], rng.uniform(-1.5, 1.5, nd), [rng.uniform(0.3, 3)]])
        UL, UR = cons_from(pl, gamma), cons_from(pr, gamma)
        l = trial % nd
        for solver, name in enumerate(names):
            out = np.zeros(nd + 2)
            lib.t_riemann_fwd(nd, solver, gamma, p(UL), p(UR), l, p(out))
            ref = o.riemann(name, UL, UR, l)
            np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-12 * (1 + np.max(np.abs(ref))))


def sph_sources_ref(nd, d, geo, WL, WR):
    """The momentum sources of direction d as the step adds them, written from
    the source terms of hydro/source_terms.hpp:16-77 and their call sites in
    extrapolation_reconstruction.hpp:145-303 / godunov_scheme.hpp:165-256."""
    k, dS, dSp, rf, cot, sf = geo
    S = np.zeros(nd + 2)

    def grad_pres(PL, PR):
        return k * (PL + PR) / 2 * (dSp - dS)

    def grad_u_r(rL, rR, uL, uR):
        return k * ((rL * uL * uL) + (rR * uR * uR)) / 2 * (dSp - dS) / 2

    def grad_u_idir_r(rL, rR, uLr, uRr, uLo, uRo):
        return k * rf * ((rR * uRo * uRr * dSp) + (rL * uLo * uLr * dS))

    if d == 0:
        S[1] += grad_pres(WL[-1], WR[-1])
        for o in range(1, nd):
            S[1] += grad_u_r(WL[0], WR[0], WL[1 + o], WR[1 + o])
            S[1 + o] -= grad_u_idir_r(WL[0], WR[0], WL[1], WR[1], WL[1 + o], WR[1 + o])
    elif d == 1:
        S[2] += grad_pres(WL[-1], WR[-1])
        if nd == 3:
            S[2] += k * ((WL[0] * WL[3] * WL[3]) + (WR[0] * WR[3] * WR[3])) / 2 * cot * (dSp - dS) / 2
            S[3] -= k * sf * ((WR[0] * WR[3] * WR[2] * dSp) + (WL[0] * WL[3] * WL[2] * dS))
    return S


@pytest.mark.parametrize("nd", [1, 2, 3])
def test_spherical_sources_and_reverse(lib, nd):
    """Spherical source terms: the forward against the reference's formulas,
    the reverse against central differences of the forward."""
    rng = np.random.default_rng(40 + nd)
    nv = nd + 2
    for _ in range(40):
        geo = np.array([rng.uniform(0.01, 0.2), rng.uniform(0.5, 2), rng.uniform(0.5, 2), rng.uniform(0.01, 0.3),
                        rng.uniform(-2, 2), rng.uniform(-0.5, 0.5)])
        WL = np.concatenate([[rng.uniform(0.3, 2)], rng.uniform(-1, 1, nd), [rng.uniform(0.3, 3)]])
        WR = np.concatenate([[rng.uniform(0.3, 2)], rng.uniform(-1, 1, nd), [rng.uniform(0.3, 3)]])
        for d in range(nd):
            def f(x):
                out = np.zeros(nv)
                lib.t_sph_src(nd, d, p(geo), p(np.ascontiguousarray(x[:nv])), p(np.ascontiguousarray(x[nv:])),
                              p(out))
                return out

            x = np.concatenate([WL, WR])
            np.testing.assert_allclose(f(x), sph_sources_ref(nd, d, geo, WL, WR), rtol=1e-14, atol=1e-15)
            J = jac_fd(f, x, nv)
            b = rng.normal(size=nv)
            gL, gR = np.zeros(nv), np.zeros(nv)
            lib.t_sph_src_rev(nd, d, p(geo), p(WL), p(WR), p(b), p(gL), p(gR))
            np.testing.assert_allclose(np.concatenate([gL, gR]), J.T @ b, rtol=1e-6, atol=1e-8)
