"""Passive scalars in the fused tile kernels: hcl_run on handles with nfx > 0
(and no pressure fix) steps with k_fused_step, which carries the scalars'
face reconstruction, Hancock predictor (extrapolation_reconstruction.hpp:
315-337, :329-339) and upwind Godunov update (godunov_scheme.hpp:118-123,
:262-301).  The FP64 kernel equals the oracle's main loop bit for bit; the
FP32-mixed kernel stays within a small tolerance of it."""
import numpy as np
import pytest

import heraclespp_b200 as hb
from heraclespp_b200 import Domain, setups
from oracle import Oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def scalar_fields(o, fx, nfx):
    """Smooth fractions in [0, 1] with steps, different for each scalar."""
    grid = setups.Grid.from_domain(o)
    s3, (X, Y, Z), _ = grid.interior()
    for f in range(nfx):
        v = 0.5 + 0.5 * np.sin(2 * np.pi * (X + (f + 1) * Y + 0.5 * f * Z))
        v = np.where(X < 0.3 + 0.1 * f, 1.0, v)
        fx[f][s3] = np.broadcast_to(v, fx[f][s3].shape)


def shear_state(o, seed=11):
    """Sheared flow with density and pressure variations (all dimensions)."""
    rng = np.random.default_rng(seed)
    grid = setups.Grid.from_domain(o)
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    shape = rho[s3].shape
    rho[s3] = np.broadcast_to(1.0 + 0.5 * (np.abs(Y - 0.5) < 0.25) + 0.1 * np.sin(2 * np.pi * X), shape)
    u[0][s3] = np.broadcast_to(0.5 - 1.0 * (np.abs(Y - 0.5) < 0.25), shape)
    if o.ndim >= 2:
        u[1][s3] = np.broadcast_to(0.05 * np.sin(4 * np.pi * X), shape)
    if o.ndim == 3:
        u[2][s3] = np.broadcast_to(0.05 * np.cos(2 * np.pi * Y), shape)
    P[s3] = 2.5 * (1.0 + 0.01 * rng.uniform(-1, 1, shape))
    return rho, u, P


# (ndim, nx, nfx, bc, extra Domain/Oracle keywords, steps)
CASES = [
    (1, [160], 5, ["NullGradient", "Reflexive"], dict(limiter="Minmod"), 60),
    (2, [40, 36], 1, ["Periodic"] * 4, dict(limiter="VanLeer"), 40),
    (2, [36, 28], 3, ["NullGradient", "Periodic", "Reflexive", "Reflexive"], dict(limiter="VanAlbada", g=(0.0, -0.3, 0.0)),
     30),
    (3, [16, 12, 20], 2, ["Periodic", "Periodic", "NullGradient", "Reflexive", "Reflexive", "NullGradient"],
     dict(limiter="Minmod", riemann="HLL", g=(0.0, 0.0, -0.1)), 15),
]


def make_pair(ndim, nx, nfx, bc, extra, precision="fp64"):
    kw = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=bc)
    kw.update(extra)
    o = Oracle(ndim, nx, nfx=nfx, **kw)
    d = Domain(ndim, nx, nfx=nfx, precision=precision, **kw)
    rho, rhou, E, fx = o.init_from_prim(*shear_state(o))
    scalar_fields(o, fx, nfx)
    o.boundaries(rho, rhou, E, fx)
    return o, d, (rho, rhou, E, fx)


@pytest.mark.parametrize("ndim,nx,nfx,bc,extra,steps", CASES)
def test_fused_passive_scalars_match_oracle_bitwise(ndim, nx, nfx, bc, extra, steps):
    o, d, (rho, rhou, E, fx) = make_pair(ndim, nx, nfx, bc, extra)
    d.set_state(rho, rhou, E, fx=fx)
    t_o, it_o, st_o, dts_o = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=steps, record_dts=True)
    assert st_o == 0 and it_o == steps
    before = hb.kernel_launch_count()
    r = d.run(cfl=0.4, max_iter=steps)
    launches = hb.kernel_launch_count() - before
    # the fused loop replays chunks of 60 step launches (those after the last
    # step return at once); the stage-composed loop launches twelve or more
    # kernels per step
    assert launches < 6 * steps, launches
    assert r.iter == it_o and r.t == t_o
    assert np.array_equal(d.dt_log(), dts_o)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    assert np.array_equal(r_d, rho) and np.array_equal(m_d, rhou) and np.array_equal(E_d, E)
    assert np.array_equal(fx_d.view(np.uint64), fx.view(np.uint64))
    assert fx_d.min() >= 0.0 and fx_d.max() <= 1.0


def test_fused_passive_scalars_from_primitives():
    """hcl_set_state_from_prim fills the scalars' ghosts (main.cpp:305-311)."""
    kw = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["NullGradient", "Reflexive", "Periodic", "Periodic"])
    o = Oracle(2, [32, 24], nfx=2, **kw)
    d = Domain(2, [32, 24], nfx=2, **kw)
    prim = shear_state(o)
    fx = o.zeros(2)
    scalar_fields(o, fx, 2)  # interior only: the ghosts come from the boundaries
    rho, rhou, E, fxo = o.init_from_prim(*prim)
    fxo[...] = fx
    o.boundaries(rho, rhou, E, fxo)
    d.set_state_from_prim(*prim, fx=fx)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    assert np.array_equal(r_d, rho) and np.array_equal(m_d, rhou) and np.array_equal(E_d, E)
    assert np.array_equal(fx_d, fxo)
    o.run(rho, rhou, E, fxo, cfl=0.4, max_iter=20)
    d.run(cfl=0.4, max_iter=20)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    assert np.array_equal(r_d, rho) and np.array_equal(fx_d, fxo)


@pytest.mark.parametrize("ndim,nx,nfx,bc,extra,steps", CASES)
def test_fused_passive_scalars_mixed_close_to_fp64(ndim, nx, nfx, bc, extra, steps):
    """FP32-mixed kernels with passive scalars: the schedule is a tile, or
    for one or two scalars on a uniform Cartesian 2-D grid a 4-warp strip (for
    one scalar in 3-D the column march; the other strip schedules carry
    none), and the fields stay within a relative L1 of 1e-5 of the FP64
    oracle on the same dts."""
    o, d, (rho, rhou, E, fx) = make_pair(ndim, nx, nfx, bc, extra, precision="fp32_mixed")
    d.set_state(rho, rhou, E, fx=fx)
    r = d.run(cfl=0.4, max_iter=steps)
    assert r.iter == steps
    if ndim == 2:
        allowed = (0, 1, 2, 3, 4, 5, 6) if nfx in (1, 2) else (0, 1, 2)
    else:
        allowed = (0, 1) if (ndim == 3 and nfx == 1) else (0,)
    assert d.schedule() in allowed
    if ndim == 2:
        for sched in (9, 10):
            with pytest.raises(hb.HclError):
                d.set_schedule(sched)
    o.run(rho, rhou, E, fx, dts=d.dt_log(), max_iter=steps)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    ng = 2
    sl = tuple(slice(ng, -ng) if n > 1 else slice(None) for n in rho.shape)
    rel = lambda a, b: float(np.abs(a[sl] - b[sl]).sum() / np.abs(b[sl]).sum())  # noqa: E731
    assert rel(r_d, rho) < 1e-5
    for f in range(nfx):
        assert rel(fx_d[f], fx[f]) < 1e-5
    assert fx_d.min() >= 0.0 and fx_d.max() <= 1.0


def _other_physics_cases():
    from cases import CASES as PARITY_CASES
    out = []
    for name in ("sph_2d", "sph_3d", "sph_2d_internalmass"):
        ndim, nx, kw, setup, skw = PARITY_CASES[name]
        out.append((name, ndim, nx, kw, skw))
    rad = dict(gamma=5.0 / 3.0, mmw=0.6, limiter="Minmod", riemann="HLLC", eos="RadGas")
    out.append(("radgas_2d", 2, [40, 32], dict(rad, bc=["NullGradient"] * 4),
                dict(rho0=1.0, rho1=0.125, P0=1e13, P1=1e11)))
    return out


@pytest.mark.parametrize("name,ndim,nx,kw,skw", _other_physics_cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_fused_passive_scalars_other_physics_bitwise(name, ndim, nx, kw, skw):
    """Spherical geometry (with the geometric sources and the internal-mass
    gravity) and the RadGas EOS with two passive scalars: FP64 fused loop
    against the oracle's main loop, bit for bit."""
    from cases import oracle_kwargs
    nfx = 2
    o = Oracle(ndim, nx, nfx=nfx, **oracle_kwargs(kw))
    d = Domain(ndim, nx, nfx=nfx, **kw)
    rho, rhou, E, fx = o.init_from_prim(*setups.shock_tube(setups.Grid.from_domain(o), **skw))
    scalar_fields(o, fx, nfx)
    o.boundaries(rho, rhou, E, fx)
    d.set_state(rho, rhou, E, fx=fx)
    steps = 25
    t_o, it_o, st_o, dts_o = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=steps, record_dts=True)
    assert st_o == 0 and it_o == steps
    r = d.run(cfl=0.4, max_iter=steps)
    assert r.iter == it_o and r.t == t_o
    assert np.array_equal(d.dt_log(), dts_o)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    assert np.array_equal(r_d, rho) and np.array_equal(m_d, rhou) and np.array_equal(E_d, E)
    assert np.array_equal(fx_d, fx)


@pytest.mark.parametrize("nfx", [1, 2])
def test_strip_passive_scalar_schedules(nfx):
    """One or two passive scalars in the 4-warp strip kernel (schedules 3-6):
    every strip height gives the same bits, the result stays within 1e-6 of
    the FP32-mixed tile kernel and within 1e-5 of the FP64 oracle (relative
    L1, density and each scalar), and the scalars stay in [0, 1]."""
    kw = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic", "Periodic", "Reflexive", "NullGradient"],
              g=(0.0, -0.2, 0.0))
    nx = [150, 200]
    steps = 40
    o = Oracle(2, nx, nfx=nfx, **kw)
    rho, rhou, E, fx = o.init_from_prim(*shear_state(o))
    scalar_fields(o, fx, nfx)
    o.boundaries(rho, rhou, E, fx)
    ref = None
    dts = None
    out = {}
    for sched in (3, 4, 5, 6, 0):
        d = Domain(2, nx, nfx=nfx, precision="fp32_mixed", **kw)
        assert d.set_schedule(sched) == sched
        d.set_state(rho, rhou, E, fx=fx)
        if dts is None:
            r = d.run(cfl=0.4, max_iter=steps)
            assert r.iter == steps
            dts = d.dt_log()
        else:
            d.run(nsteps=steps, dts=dts)
        fx_d = np.zeros_like(fx)
        r_d, m_d, E_d = d.get_state(fx=fx_d)
        out[sched] = (r_d, fx_d)
        d.close()
    for sched in (4, 5, 6):
        assert np.array_equal(out[sched][0], out[3][0]) and np.array_equal(out[sched][1], out[3][1]), sched
    ng = 2
    sl = (slice(None), slice(ng, -ng), slice(ng, -ng))
    rel = lambda a, b: float(np.abs(a[sl] - b[sl]).sum() / np.abs(b[sl]).sum())  # noqa: E731
    assert rel(out[3][0], out[0][0]) < 1e-6
    o.run(rho, rhou, E, fx, dts=dts, max_iter=steps)
    assert rel(out[3][0], rho) < 1e-5
    for k in range(nfx):
        assert rel(out[3][1][k], out[0][1][k]) < 1e-6, k
        assert rel(out[3][1][k], fx[k]) < 1e-5, k
    assert out[3][1].min() >= 0.0 and out[3][1].max() <= 1.0


@pytest.mark.parametrize("limiter,riemann,nfx", [("Minmod", "HLL", 1), ("VanLeer", "HLLC", 1), ("VanAlbada", "Low Mach", 1),
                                                 ("Constant", "HLLC", 1), ("VanLeer", "HLLC", 2), ("Minmod", "HLL", 2)])
def test_column_march_passive_scalar(limiter, riemann, nfx):
    """One or two passive scalars in the 3-D column march (schedule 1), for
    several limiter x Riemann solver instantiations of the kernel: within 1e-6
    of the FP32-mixed tile kernel and within 1e-5 of the FP64 oracle (relative
    L1, density and every scalar), the scalars in [0, 1]."""
    kw = dict(gamma=1.4, limiter=limiter, riemann=riemann,
              bc=["Periodic", "Periodic", "NullGradient", "Reflexive", "Reflexive", "Reflexive"], g=(0.0, 0.0, -0.1))
    nx = [40, 30, 36]
    steps = 20
    o = Oracle(3, nx, nfx=nfx, **kw)
    rho, rhou, E, fx = o.init_from_prim(*shear_state(o))
    scalar_fields(o, fx, nfx)
    o.boundaries(rho, rhou, E, fx)
    out, dts = {}, None
    for sched in (1, 0):
        d = Domain(3, nx, nfx=nfx, precision="fp32_mixed", **kw)
        assert d.set_schedule(sched) == sched
        d.set_state(rho, rhou, E, fx=fx)
        if dts is None:
            r = d.run(cfl=0.4, max_iter=steps)
            assert r.iter == steps
            dts = d.dt_log()
        else:
            d.run(nsteps=steps, dts=dts)
        fx_d = np.zeros_like(fx)
        r_d, _, _ = d.get_state(fx=fx_d)
        out[sched] = (r_d, fx_d)
        d.close()
    ng = 2
    sl = (slice(ng, -ng),) * 3
    rel = lambda a, b: float(np.abs(a[sl] - b[sl]).sum() / np.abs(b[sl]).sum())  # noqa: E731
    assert rel(out[1][0], out[0][0]) < 1e-6
    o.run(rho, rhou, E, fx, dts=dts, max_iter=steps)
    assert rel(out[1][0], rho) < 1e-5
    for k in range(nfx):
        assert rel(out[1][1][k], out[0][1][k]) < 1e-6, k
        assert rel(out[1][1][k], fx[k]) < 1e-5, k
    assert out[1][1].min() >= 0.0 and out[1][1].max() <= 1.0
