"""The RadGas EOS (gas plus radiation, thermodynamics/rad_gas.hpp) on the
GPU: the stage entry points and the fused FP64 loop against the oracle
(whose RadGas is pinned bit for bit to the reference's header) on a
radiation-dominated shock tube (T ~ 1e7 K).  The temperature comes from a
Newton iteration started at pow(., 1/4); CUDA's pow and the host libm's may
round differently, so the bar is the FP64 parity bar, 1e-12 relative L1 per
variable, not bit equality."""
import numpy as np
import pytest

from heraclespp_b200 import Domain, HclError, setups
from oracle import Oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-12


def rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / max(np.sum(np.abs(b)), 1e-300))


def radiative_tube(ndim, nx, riemann="HLLC", limiter="Minmod"):
    kw = dict(gamma=5.0 / 3.0, mmw=0.6, limiter=limiter, riemann=riemann, bc=["NullGradient"] * (2 * ndim))
    o = Oracle(ndim, nx, eos="RadGas", **kw)
    d = Domain(ndim, nx, eos="RadGas", **kw)
    prim = setups.shock_tube(setups.Grid.from_domain(o), rho0=1.0, rho1=0.125, P0=1e13, P1=1e11)
    return o, d, prim


@pytest.mark.parametrize("ndim,nx", [(1, [200]), (2, [48, 40])])
def test_stage_entry_points(ndim, nx):
    o, d, prim = radiative_tube(ndim, nx)
    rho, rhou, E, _ = o.init_from_prim(*prim)
    T = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    t_rho, t_rhou, t_E = T(rho), T(rhou), T(E)
    t_u, t_P = torch.zeros_like(t_rhou), torch.zeros_like(t_rho)
    d.conv_cons_to_prim(2, t_rho, t_rhou, t_E, t_u, t_P)
    u_o, P_o = o.conv_cons_to_prim(2, rho, rhou, E)
    torch.cuda.synchronize()
    assert rel_l1(t_P.cpu().numpy(), P_o) < TOL and rel_l1(t_u.cpu().numpy(), u_o) < TOL
    inv_o = o.time_step(2, rho, u_o, P_o)
    assert d.time_step(2, t_rho, T(u_o), T(P_o)) == pytest.approx(inv_o, rel=TOL)
    dt = 0.4 / inv_o
    rec = o.hydro_reconstruction(1, dt / 2, rho, u_o, P_o)[:3]
    new = o.godunov(0, dt, rho, rhou, E, *rec)[:3]
    t_rec = [torch.zeros_like(T(a)) for a in rec]
    d.hydro_reconstruction(1, dt / 2, t_rho, T(u_o), T(P_o), None, *t_rec, None)
    t_new = [torch.zeros_like(T(a)) for a in new]
    d.godunov_scheme(0, dt, t_rho, t_rhou, t_E, None, *t_rec, None, *t_new, None)
    torch.cuda.synchronize()
    for a, b in zip(t_rec, rec):
        assert rel_l1(a.cpu().numpy(), b) < TOL
    for a, b in zip(t_new, new):
        assert rel_l1(a.cpu().numpy(), b) < TOL


@pytest.mark.parametrize("ndim,nx,steps", [(1, [200], 80), (2, [48, 40], 30)])
def test_fused_loop(ndim, nx, steps):
    o, d, prim = radiative_tube(ndim, nx)
    rho, rhou, E, fx = o.init_from_prim(*prim)
    t_o, it_o, st_o, dts_o = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=steps, record_dts=True)
    assert st_o == 0 and it_o == steps
    d.set_state_from_prim(*prim)
    r = d.run(cfl=0.4, max_iter=steps)
    assert r.iter == steps and r.status == 0
    assert r.t == pytest.approx(t_o, rel=TOL)
    assert np.max(np.abs(d.dt_log()[:steps] - dts_o) / dts_o) < TOL
    for a, b in zip(d.get_state(), (rho, rhou, E)):
        assert rel_l1(a, b) < TOL


def test_radgas_needs_fp64():
    with pytest.raises(HclError):
        Domain(2, [32, 32], eos="RadGas", precision="fp32_mixed")
