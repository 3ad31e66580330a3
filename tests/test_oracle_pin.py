"""Pins the C oracle against the reference.

1. The reference's own unit-test known answers (tests/euler_equations.cpp,
   tests/riemann_solvers.cpp, tests/slopes.cpp, tests/thermodynamics.cpp,
   tests/conversions.cpp), restated as pytest checks on the oracle.
2. Bit-for-bit agreement of the oracle's per-cell physics with the
   reference's own per-cell headers compiled into oracle/_ref/
   (ref_cell_wrap.cpp), on seeded random states, for ndim = 1, 2, 3.
"""
import math

import numpy as np
import pytest

from oracle import Oracle, RefCell

LIMS = ["Constant", "VanLeer", "Minmod", "VanAlbada"]
SOLVERS = ["HLL", "HLLC", "Low Mach"]


def _o(ndim, gamma=1.4, mmw=1.0):
    return Oracle(ndim, [4] * ndim, gamma=gamma, mmw=mmw)


# ---------------------------------------------------------------------------
# Reference unit-test known answers
# ---------------------------------------------------------------------------
def test_kat_kinetic_energy(oracle_built):
    # tests/euler_equations.cpp:11-29 (1-D states)
    o = _o(1)
    assert o.ek_prim([2.0, 10.0, 0.0]) == 100.0
    assert o.ek_cons([2.0, 20.0, 100.0]) == 100.0


def test_kat_flux(oracle_built):
    # tests/euler_equations.cpp:31-63
    o = _o(1, 1.4, 1.0)
    f = o.flux_from_prim([2.0, 10.0, 0.0], 0)
    assert f[0] == pytest.approx(20.0, rel=4 * 2.2e-16)
    assert f[1] == pytest.approx(200.0, rel=4 * 2.2e-16)
    assert f[2] == pytest.approx(1000.0, rel=4 * 2.2e-16)
    f = o.flux_from_cons([2.0, 20.0, 100.0], 0)
    assert f[0] == pytest.approx(20.0, rel=4 * 2.2e-16)
    assert f[1] == pytest.approx(200.0, rel=4 * 2.2e-16)
    assert f[2] == pytest.approx(1000.0, rel=4 * 2.2e-16)


def test_kat_prim_cons_round_trip(oracle_built):
    # tests/euler_equations.cpp:65-79
    o = _o(1, 1.4, 1.0)
    prim = np.array([2.0, 10.0, 1.0])
    back = o.to_prim(o.to_cons(prim))
    np.testing.assert_allclose(back, prim, rtol=4 * 2.2e-16)


@pytest.mark.parametrize("solver", SOLVERS)
def test_kat_riemann_consistency(oracle_built, solver):
    # tests/riemann_solvers.cpp:41-57: F(U, U) = physical flux
    o = _o(1, 1.4, 1.0)
    cons = o.to_cons([2.0, 3.0, 10.0])
    num = o.riemann(solver, cons, cons, 0)
    phys = o.flux_from_cons(cons, 0)
    np.testing.assert_allclose(num, phys, rtol=4 * 2.2e-16)


@pytest.mark.parametrize("solver", SOLVERS)
def test_kat_riemann_mirror_symmetry(oracle_built, solver):
    # tests/riemann_solvers.cpp:59-83
    o = _o(1, 1.4, 1.0)
    L = o.to_cons([2.0, 3.0, 10.0])
    R = o.to_cons([3.0, -6.0, 5.5])
    f1 = o.riemann(solver, L, R, 0)
    L2, R2 = R.copy(), L.copy()
    L2[1] = -L2[1]
    R2[1] = -R2[1]
    f2 = o.riemann(solver, L2, R2, 0)
    assert f1[0] == pytest.approx(-f2[0], rel=4 * 2.2e-16)
    assert f1[1] == pytest.approx(f2[1], rel=4 * 2.2e-16)
    assert f1[2] == pytest.approx(-f2[2], rel=4 * 2.2e-16)


def test_kat_slopes(oracle_built):
    # tests/slopes.cpp:9-69
    o = _o(1)
    assert o.slope("Constant", 68.9, 37.65) == 0.0
    for lim in LIMS[1:]:
        assert o.slope(lim, 68.9, -37.65) == 0.0
        assert o.slope(lim, -68.9, 37.65) == 0.0
        assert o.slope(lim, 68.9, 68.9) == pytest.approx(68.9, rel=4 * 2.2e-16)
        assert o.slope(lim, -68.9, -68.9) == pytest.approx(-68.9, rel=4 * 2.2e-16)
        assert o.slope(lim, 2.0, 1.0) == pytest.approx(o.slope(lim, 1.0, 2.0), rel=4 * 2.2e-16)
        assert o.slope(lim, -2.0, -1.0) == pytest.approx(o.slope(lim, -1.0, -2.0), rel=4 * 2.2e-16)


def test_kat_eos_validity(oracle_built):
    # tests/thermodynamics.cpp:42-88 (PerfectGas)
    big = np.finfo(np.float64).max
    for gamma in (-math.inf, -1.0, 1.0, math.inf, math.nan):
        with pytest.raises(ValueError, match="Invalid gamma"):
            _o(1, gamma=gamma)
    for gamma in (np.nextafter(1.0, 2.0), big):
        _o(1, gamma=gamma)
    for mmw in (-math.inf, -1.0, 0.0, math.inf, math.nan):
        with pytest.raises(ValueError, match="Invalid mmw"):
            _o(1, mmw=mmw)
    for mmw in (5e-324, 1.0, big):
        _o(1, mmw=mmw)


def test_kat_eos_valid_state(oracle_built):
    # tests/thermodynamics.cpp:101-133
    o = _o(1)
    valid = [5e-324, np.finfo(np.float64).tiny, 1.0, np.finfo(np.float64).max]
    invalid = [-math.inf, -1.0, 0.0, math.inf, math.nan]
    for a in valid:
        for b in valid:
            assert o.eos_valid(a, b)
    for a in invalid:
        for b in invalid:
            assert not o.eos_valid(a, b)


@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_kat_array_conversions(oracle_built, ndim):
    # tests/conversions.cpp:17-103 on a 10^ndim uniform field with gamma = 2
    o = Oracle(ndim, [10] * ndim, ng=0, gamma=2.0, mmw=1.0)
    rho = np.full(o.shape3, 2.0)
    u = np.full((ndim,) + o.shape3, -1.0)
    P = np.full(o.shape3, 10.0)
    rhou, E = o.conv_prim_to_cons(0, rho, u, P)
    cons = o.to_cons(np.array([2.0] + [-1.0] * ndim + [10.0]))
    assert np.all(rhou == cons[1]) and np.all(E == cons[-1])
    rhou = np.full((ndim,) + o.shape3, -2.0)
    E = np.full(o.shape3, 10.0)
    u, P = o.conv_cons_to_prim(0, rho, rhou, E)
    prim = o.to_prim(np.array([2.0] + [-2.0] * ndim + [10.0]))
    assert np.all(u == prim[1]) and np.all(P == prim[-1])


# ---------------------------------------------------------------------------
# Bitwise agreement with the reference's own per-cell code
# ---------------------------------------------------------------------------
def _rand_states(rng, n, ndim):
    rho = rng.uniform(0.05, 5.0, n)
    u = rng.uniform(-3.0, 3.0, (n, ndim))
    P = rng.uniform(0.01, 10.0, n)
    return rho, u, P


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("gamma,mmw", [(1.4, 1.0), (5.0 / 3.0, 0.6)])
def test_bitwise_vs_reference_cell_physics(oracle_built, ref_cell_available, ndim, gamma, mmw):
    ref = RefCell(ndim)
    o = _o(ndim, gamma, mmw)
    rng = np.random.default_rng(1234 + ndim)
    rho, u, P = _rand_states(rng, 300, ndim)
    for n in range(rho.size):
        prim = np.concatenate([[rho[n]], u[n], [P[n]]])
        c_or = o.to_cons(prim)
        c_ref = ref.to_cons(gamma, mmw, prim)
        assert np.array_equal(c_or, c_ref)
        assert np.array_equal(o.to_prim(c_or), ref.to_prim(gamma, mmw, c_or))
        for l in range(ndim):
            assert np.array_equal(o.flux_from_prim(prim, l), ref.flux_from_prim(gamma, mmw, prim, l))
            assert np.array_equal(o.flux_from_cons(c_or, l), ref.flux_from_cons(gamma, mmw, c_or, l))


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("solver", SOLVERS)
def test_bitwise_vs_reference_riemann(oracle_built, ref_cell_available, ndim, solver):
    ref = RefCell(ndim)
    gamma, mmw = 1.4, 1.0
    o = _o(ndim, gamma, mmw)
    rng = np.random.default_rng(77 + ndim)
    rho, u, P = _rand_states(rng, 400, ndim)
    # include supersonic states so every HLLC branch is taken
    u[::7] *= 4.0
    for n in range(0, rho.size - 1):
        L = o.to_cons(np.concatenate([[rho[n]], u[n], [P[n]]]))
        R = o.to_cons(np.concatenate([[rho[n + 1]], u[n + 1], [P[n + 1]]]))
        for l in range(ndim):
            assert np.array_equal(o.riemann(solver, L, R, l), ref.riemann(solver, gamma, mmw, L, R, l))


@pytest.mark.parametrize("lim", LIMS)
def test_bitwise_vs_reference_limiters(oracle_built, ref_cell_available, lim):
    ref = RefCell(1)
    o = _o(1)
    rng = np.random.default_rng(5)
    vals = rng.normal(size=(2000, 2)) * 10.0 ** rng.integers(-6, 6, size=(2000, 2))
    vals[::11, 1] = 0.0
    for r, l in vals:
        assert o.slope(lim, r, l) == ref.slope(lim, r, l) or (
            math.isnan(o.slope(lim, r, l)) and math.isnan(ref.slope(lim, r, l)))
