"""Every schedule of the FP32-mixed fused kernel (shared-memory tiles and warp
strips) against the FP64 oracle with the same dt sequence, on periodic,
outflow/reflexive and gravity cases with ragged tile edges."""
import numpy as np
import pytest

from cases import make_pair, rel_l1

pytestmark = pytest.mark.gpu

CASES_2D = {
    # name in cases.CASES -> steps
    "kh_2d": 40,
    "kh_2d_ragged": 30,
    "quad_2d": 30,
}


@pytest.mark.parametrize("schedule", [0, 1, 2, 3, 4, 5, 6, 9, 10])
@pytest.mark.parametrize("name", list(CASES_2D))
def test_mixed_schedule_matches_oracle(name, schedule):
    o, d, (rho0, u0, P0) = make_pair(name, "fp32_mixed")
    assert d.set_schedule(schedule) == schedule
    n = CASES_2D[name]
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    _, _, _, dts = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=n, record_dts=True)
    d.set_state_from_prim(rho0, u0, P0)
    d.run(nsteps=n, dts=dts)
    r_d, m_d, E_d = d.get_state()
    # ghosts included: the in-kernel boundary fill must match too
    assert rel_l1(r_d, rho) < 2e-6
    assert rel_l1(E_d, E) < 2e-6
    for k in range(2):
        if np.sum(np.abs(rhou[k])) > 1e-3:
            assert rel_l1(m_d[k], rhou[k]) < 5e-5


@pytest.mark.parametrize("name", list(CASES_2D))
def test_in_step_strips_equal_independent_strips_bitwise(name):
    """Schedules 9 and 10 (16-warp CTAs marching in step, idle warps keeping
    the barrier sequence; rows staged by TMA in 9, by per-lane cp.async in 10)
    run the same per-cell arithmetic as schedule 6: equal states and dt
    sequences bit for bit."""
    out = []
    for schedule in (6, 9, 10):
        _, d, (rho0, u0, P0) = make_pair(name, "fp32_mixed")
        assert d.set_schedule(schedule) == schedule
        d.set_state_from_prim(rho0, u0, P0)
        r = d.run(cfl=0.4, nsteps=25)
        out.append((r.t, d.get_state()))
    (t6, s6) = out[0]
    for t, st in out[1:]:
        assert t == t6
        for a, b in zip(s6, st):
            assert np.array_equal(a, b)


def test_strip_with_gravity_and_reflexive_walls():
    """2-D Rayleigh-Taylor-like column: reflexive y walls, g along -y."""
    from heraclespp_b200 import Domain, setups
    from oracle import Oracle

    kw = dict(gamma=1.4, limiter="Minmod", riemann="HLL", bc=["Periodic", "Periodic", "Reflexive", "Reflexive"],
              g=(0.0, -0.1, 0.0), xmax=(0.5, 1.0, 1.0))
    o = Oracle(2, [40, 70], **kw)
    grid = setups.Grid.from_domain(o)
    rho0, u0, P0 = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    upper = np.broadcast_to(Y > 0.5, rho0[s3].shape)
    rho0[s3] = np.where(upper, 2.0, 1.0)
    P0[s3] = np.broadcast_to(2.5 + np.where(Y > 0.5, 2.0, 1.0) * -0.1 * (Y - 0.5), rho0[s3].shape)
    u0[1][s3] = np.broadcast_to(0.01 * np.cos(4 * np.pi * X) * np.exp(-((Y - 0.5) / 0.1) ** 2), rho0[s3].shape)
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    _, _, _, dts = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=40, record_dts=True)
    for schedule in (0, 4, 9, 10):
        d = Domain(2, [40, 70], precision="fp32_mixed", **kw)
        d.set_schedule(schedule)
        d.set_state_from_prim(rho0, u0, P0)
        d.run(nsteps=40, dts=dts)
        r_d, m_d, E_d = d.get_state()
        assert rel_l1(r_d, rho) < 2e-6, schedule
        assert rel_l1(E_d, E) < 2e-6, schedule
        assert rel_l1(m_d[1], rhou[1]) < 1e-4, schedule


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("name", ["rt_3d", "rt_3d_ragged", "rt_3d_hllc"])
def test_mixed_3d_schedule_matches_oracle(name, schedule):
    """3-D FP32-mixed schedules (shared-memory tiles, column march) against the
    FP64 oracle with the same dt sequence: gravity, reflecting and outflow
    walls, column blocks and plane ranges with ragged edges."""
    o, d, (rho0, u0, P0) = make_pair(name, "fp32_mixed")
    assert d.set_schedule(schedule) == schedule
    n = 20
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    _, _, _, dts = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=n, record_dts=True)
    d.set_state_from_prim(rho0, u0, P0)
    d.run(nsteps=n, dts=dts)
    r_d, m_d, E_d = d.get_state()
    assert rel_l1(r_d, rho) < 2e-6
    assert rel_l1(E_d, E) < 2e-6
    for k in range(3):
        if np.sum(np.abs(rhou[k])) > 1e-3 * np.sum(np.abs(rho)):
            assert rel_l1(m_d[k], rhou[k]) < 1e-4, k
