"""GPU checks on grids of user-defined nodes (the reference's UserDefined grid
type, grid_type.cpp:151-186): the FP64, fast-FP64 and FP32-mixed fused steps
against the oracle, and the discrete adjoint against central differences.  On such grids the limited
slopes take the differences over the half spacings and the face values the
half width of each cell (limited_linear_reconstruction.hpp:46-64), and the
predictor and the update divide by each cell's own width (or volume).

The nodes follow x = lo + (hi - lo) (s + 0.35 sin(2 pi s) / (2 pi)) over a
uniform s, so cell widths vary smoothly by a factor of about 2 (and the ghost
widths of a periodic direction repeat the interior's)."""
import numpy as np
import pytest

from cases import oracle_kwargs
from heraclespp_b200 import Domain
from oracle import Oracle
from test_gpu_adjoint_scalars import gradient, interior, objective, smooth_state, split

pytestmark = pytest.mark.gpu
NG = 2

# name: (ndim, cells, nfx, domain kwargs, steps)
CASES = {
    "cart_2d": (2, [40, 24], 0, dict(gamma=1.4, limiter="VanLeer", riemann="HLLC",
                                     bc=["NullGradient", "Reflexive", "Reflexive", "Reflexive"],
                                     xmin=(0.0, 0.0, 0.0), xmax=(1.0, 0.6, 1.0)), 12),
    "cart_2d_scalar": (2, [36, 20], 1, dict(gamma=1.4, limiter="VanAlbada", riemann="HLL",
                                            bc=["Reflexive", "NullGradient", "Periodic", "Periodic"],
                                            xmin=(0.0, 0.0, 0.0), xmax=(1.0, 0.5, 1.0)), 12),
    "sph_1d": (1, [64], 0, dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                                bc=["Reflexive", "NullGradient"], xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), 16),
    "cart_3d": (3, [12, 10, 8], 0, dict(gamma=1.4, limiter="VanLeer", riemann="HLLC",
                                        bc=["Reflexive", "NullGradient", "Periodic", "Periodic", "Reflexive",
                                            "Reflexive"],
                                        xmin=(0.3, 0.6, 0.0), xmax=(1.0, 2.5, 1.5)), 10),
}


def stretched_nodes(ndim, nx, lo, hi):
    """Node coordinates (n_d + 1 values, ghosts included) of every direction."""
    out = []
    for d in range(3):
        n = (nx[d] if d < ndim else 1) + (2 * NG if d < ndim else 0)
        if d >= ndim:
            out.append(np.array([lo[d], hi[d]]))
            continue
        s = (np.arange(n + 1) - NG) / nx[d]
        out.append(lo[d] + (hi[d] - lo[d]) * (s + 0.35 * np.sin(2 * np.pi * s) / (2 * np.pi)))
    return out


def problem(name):
    ndim, nx, nfx, kw, nsteps = CASES[name]
    nodes = stretched_nodes(ndim, nx, kw["xmin"], kw["xmax"])
    o = Oracle(ndim, nx, nfx=nfx, nodes=nodes, **oracle_kwargs(kw))
    dx0 = np.diff(nodes[0])
    assert dx0.max() / dx0.min() > 1.8
    rho0, u0, P0, fx0 = smooth_state(o, ndim, nfx, kw)
    rho, rhou, E, _ = o.init_from_prim(rho0, u0, P0)
    o.boundaries(rho, rhou, E, fx0)
    U0 = np.concatenate([rho[None], rhou, E[None], fx0])
    d = Domain(ndim, nx, nfx=nfx, nodes=nodes, precision="fp64", **kw)
    d.set_state(rho, rhou, E, fx0)
    r = d.run(cfl=0.4, nsteps=nsteps)
    assert r.iter == nsteps
    dts = d.dt_log()[:nsteps]
    rng = np.random.default_rng(31)
    fxN = np.zeros_like(fx0)
    rhoN = d.get_state(fx=fxN)[0]
    targets = (rhoN * (1 + 0.01 * rng.uniform(-1, 1, rho.shape)), fxN + 0.01 * rng.uniform(-1, 1, fx0.shape))
    return o, d, U0, dts, targets


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_step_on_user_defined_nodes_matches_oracle(name):
    """The FP64 step on user-defined nodes against the oracle over the
    recorded dts: within 1e-12 relative L1 per field."""
    o, d, U0, dts, _ = problem(name)
    nd = d.ndim
    rho, rhou, E, fx = (a.copy() for a in split(U0, nd))
    o.run(rho, rhou, E, fx if fx.shape[0] else None, dts=dts, max_iter=len(dts))
    d.set_state(*split(U0, nd))
    d.run(nsteps=len(dts), dts=dts)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = d.get_state(fx=fx_d)
    s = interior(nd)
    rel = lambda a, b: float(np.abs(a[s] - b[s]).sum() / np.abs(b[s]).sum())  # noqa: E731
    assert rel(r_d, rho) <= 1e-12
    assert rel(E_d, E) <= 1e-12
    for k in range(nd):
        assert rel(m_d[k], rhou[k]) <= 1e-12, k
    for k in range(fx.shape[0]):
        assert rel(fx_d[k], fx[k]) <= 1e-12, k
    d.close()


@pytest.mark.parametrize("precision,bound", [("fp64_fast", 1e-12), ("fp32_mixed", 1e-5)])
@pytest.mark.parametrize("name", list(CASES))
def test_fast_and_mixed_steps_on_user_defined_nodes(name, precision, bound):
    """The fast-FP64 and FP32-mixed steps on user-defined nodes (the fused tile
    kernel's per-cell spacing path) against the oracle over the FP64 run's
    dts: relative L1 per field within the bounds those precisions are held
    to on regular grids."""
    o, d, U0, dts, _ = problem(name)
    d.close()
    ndim, nx, nfx, kw, _ = CASES[name]
    nd = ndim
    rho, rhou, E, fx = (a.copy() for a in split(U0, nd))
    o.run(rho, rhou, E, fx if fx.shape[0] else None, dts=dts, max_iter=len(dts))
    dp = Domain(ndim, nx, nfx=nfx, nodes=stretched_nodes(ndim, nx, kw["xmin"], kw["xmax"]), precision=precision, **kw)
    dp.set_state(*split(U0, nd))
    dp.run(nsteps=len(dts), dts=dts)
    fx_d = np.zeros_like(fx)
    r_d, m_d, E_d = dp.get_state(fx=fx_d)
    s = interior(nd)
    rel = lambda a, b: float(np.abs(a[s] - b[s]).sum() / np.abs(b[s]).sum())  # noqa: E731
    errs = [rel(r_d, rho), rel(E_d, E)] + [rel(m_d[k], rhou[k]) for k in range(nd)] + \
        [rel(fx_d[k], fx[k]) for k in range(nfx)]
    print(f"{name} {precision}: max rel L1 {max(errs):.2e}")
    assert max(errs) <= bound, errs
    dp.close()


@pytest.mark.parametrize("name", list(CASES))
def test_adjoint_on_user_defined_nodes_matches_finite_differences(name):
    o, d, U0, dts, targets = problem(name)
    nd = d.ndim
    g = gradient(d, U0, dts, targets, "fp64")
    s = (slice(None),) + interior(nd)
    rng = np.random.default_rng(77)
    eps = 1e-8
    errs = []
    for _ in range(10):
        v = np.zeros_like(U0)
        v[s] = rng.uniform(-1, 1, U0[s].shape) * np.abs(U0[s])
        fp = objective(d, o, U0 + eps * v, dts, targets)
        fm = objective(d, o, U0 - eps * v, dts, targets)
        fd = (fp - fm) / (2 * eps)
        errs.append(abs(fd - float(np.sum(g * v))) / max(abs(fd), 1e-300))
    errs = np.array(errs)
    print(f"{name}: FD rel err median {np.median(errs):.2e} max {errs.max():.2e}")
    assert np.median(errs) < 1e-5, errs
    assert np.max(errs) < 1e-3, errs
    mask = np.ones(U0.shape, bool)
    mask[s] = False
    assert np.all(g[mask] == 0)
    d.close()


def test_mixed_sweep_on_user_defined_nodes_close_to_fp64():
    """The FP32 sweep on a stretched 2-D grid against the FP64 sweep (the
    bound of the other mixed-sweep tests)."""
    o, d, U0, dts, targets = problem("cart_2d")
    g64 = gradient(d, U0, dts, targets, "fp64")
    g32 = gradient(d, U0, dts, targets, "fp32_mixed")
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print(f"cart_2d stretched: mixed vs fp64 adjoint rel L2 {rel:.2e}")
    assert rel < 1e-3, rel
    d.close()
