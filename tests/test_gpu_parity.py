"""GPU parity: the product's CUDA kernels (through the C ABI) against the CPU
oracle on the same inputs.  FP64 is bit-exact: each stage entry point, the
fused step over many steps, and the dt sequence.  The FP32-mixed path is
checked by relative L1 error per variable."""
import numpy as np
import pytest

from cases import CASES, make_pair, rel_l1

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ALL = list(CASES)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("name", ALL)
def test_grid_bitwise(name):
    o, d, _ = make_pair(name)
    go, gd = o.grid(), d.grid()
    for k in go:
        assert np.array_equal(go[k], gd[k]), k


@pytest.mark.parametrize("name", ALL)
def test_initial_state_bitwise(name):
    o, d, (rho, u, P) = make_pair(name)
    r_o, m_o, E_o, _ = o.init_from_prim(rho, u, P)
    d.set_state_from_prim(rho, u, P)
    r_d, m_d, E_d = d.get_state()
    assert np.array_equal(r_o, r_d)
    assert np.array_equal(m_o, m_d)
    assert np.array_equal(E_o, E_d)


@pytest.mark.parametrize("name", ALL)
def test_stage_entry_points_bitwise(name):
    """One reference iteration (main.cpp:355-526) stage by stage."""
    o, d, (rho0, u0, P0) = make_pair(name)
    nd = o.ndim
    rho, rhou, E, _ = o.init_from_prim(rho0, u0, P0)
    ng = 2
    if CASES[name][2].get("gravity") == "Internal_mass":
        # make_internal_mass_gravity from this state: the radial table the
        # reconstruction and Godunov stages below use
        g_o = o.internal_mass_gravity(rho)
        t_g = torch.zeros(g_o.shape, dtype=torch.float64, device="cuda")
        d.internal_mass_gravity(_dev(rho), t_g)
        torch.cuda.synchronize()
        assert np.array_equal(_host(t_g), g_o)
    # cons -> prim on all_ghosts
    u_o, P_o = o.conv_cons_to_prim(ng, rho, rhou, E)
    t_rho, t_rhou, t_E = _dev(rho), _dev(rhou), _dev(E)
    t_u, t_P = torch.zeros_like(t_rhou), torch.zeros_like(t_rho)
    d.conv_cons_to_prim(ng, t_rho, t_rhou, t_E, t_u, t_P)
    torch.cuda.synchronize()
    assert np.array_equal(_host(t_u), u_o) and np.array_equal(_host(t_P), P_o)
    # prim -> cons
    m2, E2 = o.conv_prim_to_cons(ng, rho, u_o, P_o)
    t_m2, t_E2 = torch.zeros_like(t_rhou), torch.zeros_like(t_E)
    d.conv_prim_to_cons(ng, t_rho, t_u, t_P, t_m2, t_E2)
    torch.cuda.synchronize()
    assert np.array_equal(_host(t_m2), m2) and np.array_equal(_host(t_E2), E2)
    # time step
    inv_o = o.time_step(ng, rho, u_o, P_o)
    inv_d = d.time_step(ng, t_rho, t_u, t_P)
    assert inv_o == inv_d
    dt = 0.4 * inv_o
    # reconstruction (with_ghosts(1), dt/2)
    rr_o, mr_o, Er_o, _ = o.hydro_reconstruction(1, dt / 2, rho, u_o, P_o)
    shape3 = rho.shape
    t_rr = torch.zeros((nd, 2) + shape3, dtype=torch.float64, device="cuda")
    t_mr = torch.zeros((nd, nd, 2) + shape3, dtype=torch.float64, device="cuda")
    t_Er = torch.zeros((nd, 2) + shape3, dtype=torch.float64, device="cuda")
    d.hydro_reconstruction(1, dt / 2, t_rho, t_u, t_P, None, t_rr, t_mr, t_Er, None)
    torch.cuda.synchronize()
    assert np.array_equal(_host(t_rr), rr_o)
    assert np.array_equal(_host(t_mr), mr_o)
    assert np.array_equal(_host(t_Er), Er_o)
    # Godunov (no_ghosts, dt)
    rn_o, mn_o, En_o, _ = o.godunov(0, dt, rho, rhou, E, rr_o, mr_o, Er_o)
    t_rn, t_mn, t_En = torch.zeros_like(t_rho), torch.zeros_like(t_rhou), torch.zeros_like(t_E)
    d.godunov_scheme(0, dt, t_rho, t_rhou, t_E, None, t_rr, t_mr, t_Er, None, t_rn, t_mn, t_En, None)
    torch.cuda.synchronize()
    assert np.array_equal(_host(t_rn), rn_o)
    assert np.array_equal(_host(t_mn), mn_o)
    assert np.array_equal(_host(t_En), En_o)
    # boundaries on the new state (every ghost cell, corners included)
    o.boundaries(rn_o, mn_o, En_o)
    d.boundary_conditions(t_rn, t_mn, t_En)
    torch.cuda.synchronize()
    assert np.array_equal(_host(t_rn), rn_o)
    assert np.array_equal(_host(t_mn), mn_o)
    assert np.array_equal(_host(t_En), En_o)
    # health and conservation reductions
    assert d.minimum_internal_energy(t_rn, t_mn, t_En) == o.min_internal_energy(rn_o, mn_o, En_o)
    assert d.integrate(t_rn) == pytest.approx(o.integrate(rn_o), rel=1e-14, abs=0)


NSTEPS = {"sod_1d": 200, "sod_1d_odd": 60, "advection_1d": 100, "kh_2d": 60, "kh_2d_ragged": 40, "quad_2d": 40,
          "gresho_2d_lowmach": 30, "rt_3d": 12, "rt_3d_ragged": 10, "rt_3d_hllc": 10, "sph_1d_pointmass": 50,
          "sph_2d": 25, "sph_3d": 8, "sph_1d_internalmass": 50, "sph_2d_internalmass": 25}


@pytest.mark.parametrize("name", ALL)
def test_fused_fp64_bitwise(name):
    """The fused step (graph-replayed, device-resident dt) reproduces the
    oracle's main loop bit for bit, dt sequence included."""
    o, d, (rho0, u0, P0) = make_pair(name, "fp64")
    n = NSTEPS[name]
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    t_o, it_o, st_o, dts_o = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=n, record_dts=True)
    assert st_o == 0
    d.set_state_from_prim(rho0, u0, P0)
    r = d.run(cfl=0.4, max_iter=n, graph_chunk=12)
    assert r.iter == it_o == n
    assert r.t == t_o
    assert np.array_equal(d.dt_log()[:n], dts_o)
    r_d, m_d, E_d = d.get_state()
    assert np.array_equal(r_d, rho), np.max(np.abs(r_d - rho))
    assert np.array_equal(m_d, rhou)
    assert np.array_equal(E_d, E)


def test_sod_to_t_end_bitwise():
    """Sod 1024 cells to t=0.2 with the shipped output cadence (dt clamped at
    t=0.1, inputs/shock_tube.ini) -- device loop vs oracle."""
    o, d, (rho0, u0, P0) = make_pair("sod_1d", "fp64")
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    t_o, it_o, st_o, _ = o.run(rho, rhou, E, fx, cfl=0.4, t_end=0.2, max_iter=100000, time_frequency=0.1)
    d.set_state_from_prim(rho0, u0, P0)
    r = d.run(cfl=0.4, t_end=0.2, max_iter=100000, time_frequency=0.1)
    assert r.finished == 1
    assert r.t == t_o == 0.2
    assert r.iter == it_o
    r_d, m_d, E_d = d.get_state()
    assert np.array_equal(r_d, rho) and np.array_equal(m_d, rhou) and np.array_equal(E_d, E)


@pytest.mark.parametrize("name,tol", [("kh_2d", 1e-6), ("sod_1d", 2e-6), ("rt_3d", 1e-6), ("quad_2d", 1e-5),
                                      ("sph_2d", 1e-5), ("sph_1d_internalmass", 2e-6)])
def test_fused_mixed_l1(name, tol):
    """FP32-mixed against the FP64 oracle with the same dt sequence."""
    o, d, (rho0, u0, P0) = make_pair(name, "fp32_mixed")
    n = NSTEPS[name]
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    _, _, _, dts = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=n, record_dts=True)
    d.set_state_from_prim(rho0, u0, P0)
    d.run(nsteps=n, dts=dts)
    r_d, m_d, E_d = d.get_state()
    errs = [rel_l1(r_d, rho), rel_l1(E_d, E)] + [rel_l1(m_d[k], rhou[k]) for k in range(o.ndim)
                                                 if np.sum(np.abs(rhou[k])) > 1e-8]
    assert max(errs[:2]) < tol, errs


def test_conservation_sums_match_oracle():
    o, d, (rho0, u0, P0) = make_pair("kh_2d", "fp64")
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    d.set_state_from_prim(rho0, u0, P0)
    s = d.conservation_sums()
    assert s[0] == pytest.approx(o.integrate(rho), rel=1e-15)
    assert s[-1] == pytest.approx(o.integrate(E), rel=1e-15)
    d.run(cfl=0.4, max_iter=50)
    s2 = d.conservation_sums()
    # periodic box: mass and energy are conserved to round-off
    assert abs(s2[0] - s[0]) / s[0] < 1e-13
    assert abs(s2[-1] - s[-1]) / s[-1] < 1e-13


def test_invalid_state_reports_error_and_gpu_stays_usable():
    """main.cpp:397-425: a negative internal energy stops the loop with an
    error status (no trap); the next domain on the same GPU works."""
    from heraclespp_b200 import HclError

    o, d, (rho0, u0, P0) = make_pair("kh_2d", "fp64")
    P0 = P0.copy()
    P0[0, 2 + 10, 2 + 7] = -1.0  # host-side injected bad pressure
    d.set_state_from_prim(rho0, u0, P0)
    with pytest.raises(HclError, match="invalid"):
        d.run(cfl=0.4, max_iter=10)
    o2, d2, (r2, u2, p2) = make_pair("kh_2d", "fp64")
    d2.set_state_from_prim(r2, u2, p2)
    res = d2.run(cfl=0.4, max_iter=5)
    assert res.iter == 5
