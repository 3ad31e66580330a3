"""InternalMassGravity on the GPU: the radial gravity table from a density
(hcl_internal_mass_gravity) against the oracle's restatement of
gravity.cpp:59-128, and the stage-composed loop (passive scalar) with the
table rebuilt every step against the oracle's main loop, bit for bit.  The
fused loop with this gravity is in test_gpu_parity (sph_*_internalmass)."""
import numpy as np
import pytest

from heraclespp_b200 import Domain, setups
from oracle import Oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GEOMS = [
    (1, [80], ["Reflexive", "NullGradient"], (0.2, 0, 0), (1.2, 1, 1)),
    (2, [36, 20], ["Reflexive", "NullGradient", "Reflexive", "Reflexive"], (0.3, 0.5, 0), (1.0, 2.6, 1)),
    (3, [14, 10, 8], ["Reflexive", "NullGradient", "Reflexive", "Reflexive", "Periodic", "Periodic"],
     (0.3, 0.6, 0), (1.0, 2.5, 1.5)),
]


@pytest.mark.parametrize("ndim,nx,bc,xmin,xmax", GEOMS)
def test_table_from_random_density_bitwise(ndim, nx, bc, xmin, xmax):
    kw = dict(gamma=1.4, limiter="Minmod", riemann="HLLC", bc=bc, gravity="Internal_mass", central_mass=2e8,
              xmin=xmin, xmax=xmax)
    o = Oracle(ndim, nx, geom="Spherical", **kw)
    d = Domain(ndim, nx, geometry="Spherical", **kw)
    rng = np.random.default_rng(11 + ndim)
    for call in range(2):
        rho = rng.uniform(0.5, 2.0, o.zeros().shape)
        g_o = o.internal_mass_gravity(rho)
        t_g = torch.full(g_o.shape, np.nan, dtype=torch.float64, device="cuda")
        d.internal_mass_gravity(torch.tensor(rho, device="cuda"), t_g)
        torch.cuda.synchronize()
        assert np.array_equal(t_g.cpu().numpy(), g_o), call


def test_stage_loop_with_internal_mass_bitwise():
    """With a passive scalar (carried by the fused tile kernel) the table is
    still rebuilt from the density before every step (main.cpp:528) and the
    run equals the oracle's main loop."""
    kw = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Reflexive", "NullGradient"],
              gravity="Internal_mass", central_mass=1e8, xmin=(0.2, 0, 0), xmax=(1.2, 1, 1))
    o = Oracle(1, [96], nfx=1, geom="Spherical", **kw)
    d = Domain(1, [96], nfx=1, geometry="Spherical", **kw)
    prim = setups.shock_tube(setups.Grid.from_domain(o), inter=0.7)
    rho, rhou, E, fx = o.init_from_prim(*prim)
    grid = setups.Grid.from_domain(o)
    s3, (X, Y, Z), _ = grid.interior()
    fx[0][s3] = np.broadcast_to(np.where(X < 0.7, 1.0, 0.0), fx[0][s3].shape)
    o.boundaries(rho, rhou, E, fx)
    d.set_state(rho, rhou, E, fx=fx)
    t_o, it_o, st_o, dts_o = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=40, record_dts=True)
    assert st_o == 0 and it_o == 40
    r = d.run(cfl=0.4, max_iter=40)
    assert r.iter == it_o and r.t == t_o
    assert np.array_equal(d.dt_log(), dts_o)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    assert np.array_equal(r_d, rho) and np.array_equal(m_d, rhou) and np.array_equal(E_d, E)
    assert np.array_equal(fx_d, fx)
