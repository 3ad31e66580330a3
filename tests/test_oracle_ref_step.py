"""The oracle's array-level restatement against the reference's own array code.

oracle/_ref/libref_step_*.so is the reference's hydro/, mesh/, boundary*,
gravity/ and analysis/ sources (plus utils/param.cpp and vendor/inih) compiled
where they lie against the host Kokkos and single-rank MPI stand-ins of
oracle/ref_array (make -C oracle ref-step).  Each stage the oracle restates --
conversions, MUSCL-Hancock reconstruction with the Hancock predictor, the
Godunov update, the single-rank boundary sequence, the CFL time step, the
internal-energy check -- must give the same bits on seeded states, and so must
the time loop of main.cpp:354-531 over 20 steps, dt sequence included, on every
configuration of the parity case matrix that the wrapper covers (uniform and
point-mass gravity, Cartesian and spherical, 1-D to 3-D), with and without
passive scalars."""
import numpy as np
import pytest

from cases import CASES, oracle_kwargs

# internal-mass gravity is rebuilt from the density each step by main(); the
# wrapper drives the uniform and point-mass fields
NAMES = [n for n, c in CASES.items() if c[2].get("gravity") != "Internal_mass"]


@pytest.fixture(scope="session")
def ref_step_available():
    from oracle import build_oracle, ref_step_path

    if not ref_step_path(2).exists():
        import subprocess

        from conftest import ROOT

        build_oracle(ref=True)
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref-step"], check=True)
    if not ref_step_path(2).exists():
        pytest.skip("oracle/_ref reference step library not built (reference sources absent)")
    return True


def pair(name, nfx=0):
    from heraclespp_b200 import setups
    from oracle import Oracle, RefStep

    ndim, nx, kw, setup, skw = CASES[name]
    okw = oracle_kwargs(kw)
    o = Oracle(ndim, nx, nfx=nfx, **okw)
    r = RefStep(ndim, nx, nfx=nfx, **okw)
    prim = setups.SETUPS[setup](setups.Grid.from_domain(o), **skw)
    return o, r, prim


def perturbed_state(o, prim, seed):
    """The setup's conservative state with a seeded 1 % perturbation of every
    primitive (so limiters and Riemann branches see varied inputs), ghosts
    filled by the oracle's boundary sequence."""
    rng = np.random.default_rng(seed)
    rho0, u0, P0 = (np.array(a) for a in prim)
    rho0 *= 1 + 0.01 * rng.uniform(-1, 1, rho0.shape)
    P0 *= 1 + 0.01 * rng.uniform(-1, 1, P0.shape)
    u0 += 0.01 * rng.uniform(-1, 1, u0.shape)
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    if o.nfx:
        fx[:] = rng.uniform(0, 1, fx.shape)
        o.boundaries(rho, rhou, E, fx)
    return rho, rhou, E, fx


@pytest.mark.parametrize("name", NAMES)
def test_grid_arrays_equal(ref_step_available, name):
    o, r, _ = pair(name)
    go, gr = o.grid(), r.grid()
    for key in ("ds", "dv", "dx0", "dx1", "dx2", "x0c", "x1c", "x2c"):
        assert np.array_equal(go[key], gr[key]), key


@pytest.mark.parametrize("nfx", [0, 2])
@pytest.mark.parametrize("name", NAMES)
def test_stages_bitwise(ref_step_available, name, nfx):
    o, r, prim = pair(name, nfx)
    rho, rhou, E, fx = perturbed_state(o, prim, seed=sum(map(ord, name)) + nfx)
    ng = 2
    # conversions over all ghosts
    u_o, P_o = o.conv_cons_to_prim(ng, rho, rhou, E)
    u_r, P_r = r.conv_cons_to_prim(ng, rho, rhou, E)
    assert np.array_equal(u_o, u_r) and np.array_equal(P_o, P_r)
    m_o, E_o = o.conv_prim_to_cons(ng, rho, u_o, P_o)
    m_r, E_r = r.conv_prim_to_cons(ng, rho, u_o, P_o)
    assert np.array_equal(m_o, m_r) and np.array_equal(E_o, E_r)
    # CFL time step and the internal-energy check
    assert o.time_step(ng, rho, u_o, P_o) == r.time_step(ng, rho, u_o, P_o)
    assert o.min_internal_energy(rho, rhou, E) == r.min_internal_energy(rho, rhou, E)
    # reconstruction with the Hancock predictor (with_ghosts(1), dt/2)
    dt = 0.4 * o.time_step(ng, rho, u_o, P_o)  # time_step returns the dt at CFL 1
    rec_o = o.hydro_reconstruction(1, dt / 2, rho, u_o, P_o, fx)
    rec_r = r.hydro_reconstruction(1, dt / 2, rho, u_o, P_o, fx)
    for a, b, what in zip(rec_o, rec_r, ("rho_rec", "rhou_rec", "E_rec", "fx_rec")):
        if what == "fx_rec" and nfx == 0:
            continue
        assert np.array_equal(a, b), what
    # Godunov update (no_ghosts)
    new_o = o.godunov(0, dt, rho, rhou, E, *rec_o[:3], fx=fx, fx_rec=rec_o[3])
    new_r = r.godunov(0, dt, rho, rhou, E, *rec_o[:3], fx=fx, fx_rec=rec_o[3])
    for a, b, what in zip(new_o, new_r, ("rho_new", "rhou_new", "E_new", "fx_new")):
        if what == "fx_new" and nfx == 0:
            continue
        assert np.array_equal(a, b), what
    # boundary sequence on the new state
    bo = [x.copy() for x in new_o]
    br = [x.copy() for x in new_o]
    o.boundaries(*bo)
    r.boundaries(*br)
    for a, b in zip(bo, br):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("nfx", [0, 2])
@pytest.mark.parametrize("name", NAMES)
def test_time_loop_bitwise(ref_step_available, name, nfx):
    o, r, prim = pair(name, nfx)
    rho, rhou, E, fx = perturbed_state(o, prim, seed=7 + nfx)
    a = [x.copy() for x in (rho, rhou, E, fx)]
    t_o, it_o, st_o, dts_o = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=20, record_dts=True)
    t_r, it_r, st_r, dts_r = r.run(*a, cfl=0.4, max_iter=20, record_dts=True)
    assert (it_o, st_o) == (it_r, st_r) == (20, 0)
    assert t_o == t_r and np.array_equal(dts_o, dts_r)
    for x, y in zip((rho, rhou, E), a[:3]):
        assert np.array_equal(x, y)
    if nfx:
        assert np.array_equal(fx, a[3])


def test_sod_to_t_end_bitwise(ref_step_available):
    """Sod 1024 cells to t = 0.2: the dt clamp to t_end of main.cpp:374-378."""
    o, r, prim = pair("sod_1d")
    rho, rhou, E, fx = o.init_from_prim(*prim)
    a = [x.copy() for x in (rho, rhou, E, fx)]
    t_o, it_o, st_o, _ = o.run(rho, rhou, E, fx, cfl=0.4, t_end=0.2, max_iter=100000)
    t_r, it_r, st_r, _ = r.run(*a, cfl=0.4, t_end=0.2, max_iter=100000)
    assert st_o == st_r == 0 and it_o == it_r and t_o == t_r == 0.2
    for x, y in zip((rho, rhou, E), a[:3]):
        assert np.array_equal(x, y)
