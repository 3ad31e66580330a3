"""GPU checks of the discrete adjoint with passive scalars (hcl_adjoint_* on a
handle with nfx > 0): the scalars' limited face values and the predictor's
mass-flux increment over the predicted face density
(extrapolation_reconstruction.hpp:87-88, :315-339), the upwind fluxes of the
update and the clamp of rho'x' / rho' (godunov_scheme.hpp:262-301), and their
coupling back into the density, the face states and the Riemann mass fluxes.

Smooth states whose fractions stay inside (0, 1) (the clamp is inactive and
differentiable there), dt recorded from a CFL run and held fixed;
J = 0.5 ||rho^N - rho_t||^2 + 0.5 sum_k ||x_k^N - x_t,k||^2 over the interior.
The FP64 gradient, including the scalars' planes, is checked against central
differences of the FP64 forward along seeded random directions, the FP32 sweep
against the FP64 one, and a 3-D FP64 sweep with more scalars than its tile's
shared memory holds is refused."""
import numpy as np
import pytest

from cases import oracle_kwargs
from heraclespp_b200 import Domain, HclError, setups
from oracle import Oracle

pytestmark = pytest.mark.gpu
NG = 2

# name: (ndim, cells, nfx, domain kwargs, steps)
CASES = {
    "cart_1d": (1, [64], 1, dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Reflexive", "NullGradient"],
                                 xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), 16),
    "cart_2d_two": (2, [40, 24], 2, dict(gamma=1.4, limiter="Minmod", riemann="HLL",
                                         bc=["Periodic", "Periodic", "Reflexive", "Reflexive"],
                                         xmin=(0.0, 0.0, 0.0), xmax=(1.0, 0.6, 1.0)), 12),
    "cart_2d_lowmach": (2, [36, 20], 1, dict(gamma=5.0 / 3.0, limiter="VanAlbada", riemann="Low Mach",
                                             bc=["NullGradient", "Reflexive", "Periodic", "Periodic"],
                                             gravity="Uniform", g=(0.0, -0.3, 0.0),
                                             xmin=(0.0, 0.0, 0.0), xmax=(1.0, 0.5, 1.0)), 12),
    "sph_2d": (2, [40, 24], 1, dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                                    bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive"],
                                    xmin=(0.2, 0.5, 0.0), xmax=(1.0, 2.6, 1.0)), 12),
    "cart_3d": (3, [12, 10, 8], 1, dict(gamma=1.4, limiter="VanLeer", riemann="HLLC",
                                        bc=["Reflexive", "NullGradient", "Periodic", "Periodic", "Reflexive",
                                            "Reflexive"],
                                        xmin=(0.3, 0.6, 0.0), xmax=(1.0, 2.5, 1.5)), 10),
}


def interior(ndim):
    return (slice(NG, -NG) if ndim == 3 else slice(None), slice(NG, -NG) if ndim >= 2 else slice(None),
            slice(NG, -NG))


def smooth_state(o, ndim, nfx, kw):
    """Smooth primitives that vary along every direction, with no extremum
    symmetric about a cell face and no field linear along a direction (where
    neighbours tie, or where |R| = |L| for Minmod, the limited slope sits on
    the limiter's kink and its branch is set by rounding), and fractions in
    [0.07, 0.93]."""
    grid = setups.Grid.from_domain(o)
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    shape = rho[s3].shape
    lo, hi = kw["xmin"], kw["xmax"]
    sr = (X - lo[0]) / (hi[0] - lo[0])
    st = (Y - lo[1]) / (hi[1] - lo[1]) if ndim >= 2 else 0.0 * X
    sp = (Z - lo[2]) / (hi[2] - lo[2]) if ndim == 3 else 0.0 * X
    rho[s3] = np.broadcast_to(1 + 0.2 * np.sin(2 * np.pi * sr + 0.3) * (1 + 0.3 * np.cos(np.pi * st + 0.2))
                              * (1 + 0.1 * np.sin(2 * np.pi * sp + 0.45)), shape)
    P[s3] = np.broadcast_to(1 + 0.1 * np.cos(2 * np.pi * sr + 0.5 * st + 0.37) + 0.05 * np.cos(2 * np.pi * sp + 0.4),
                            shape)
    u[0][s3] = np.broadcast_to(0.08 * np.sin(np.pi * sr) * (1 + 0.35 * sr) * (1 + 0.4 * np.cos(np.pi * st + 0.7))
                               * (1 + 0.2 * np.sin(2 * np.pi * sp + 0.6)), shape)
    if ndim >= 2:
        u[1][s3] = np.broadcast_to(0.06 * np.sin(np.pi * st) * (1 + 0.3 * st) * (1 + 0.5 * sr + 0.3 * sr * sr)
                                   * (1 + 0.3 * np.sin(2 * np.pi * sp + 0.1)), shape)
    if ndim == 3:
        u[2][s3] = np.broadcast_to((0.05 * np.sin(2 * np.pi * sp + 0.2) * (0.5 + sr) + 0.02)
                                   * (1 + 0.3 * np.cos(np.pi * st + 0.25)), shape)
    fx = np.zeros((nfx,) + rho.shape)
    for k in range(nfx):
        fx[k][s3] = np.broadcast_to(0.5 + 0.3 * np.sin(2 * np.pi * sr + 0.7 + 1.3 * k)
                                    * (1 + 0.25 * np.cos(np.pi * st + 0.4 + 0.5 * k))
                                    * (1 + 0.15 * np.sin(2 * np.pi * sp + 0.9)), shape)
    return rho, u, P, fx


def problem(name, precision="fp64"):
    ndim, nx, nfx, kw, nsteps = CASES[name]
    o = Oracle(ndim, nx, nfx=nfx, **oracle_kwargs(kw))
    rho0, u0, P0, fx0 = smooth_state(o, ndim, nfx, kw)
    rho, rhou, E, _ = o.init_from_prim(rho0, u0, P0)
    o.boundaries(rho, rhou, E, fx0)
    U0 = np.concatenate([rho[None], rhou, E[None], fx0])
    d = Domain(ndim, nx, nfx=nfx, precision=precision, **kw)
    d.set_state(rho, rhou, E, fx0)
    r = d.run(cfl=0.4, nsteps=nsteps)
    assert r.iter == nsteps
    dts = d.dt_log()[:nsteps]
    rng = np.random.default_rng(31)
    fxN = np.zeros_like(fx0)
    rhoN = d.get_state(fx=fxN)[0]
    targets = (rhoN * (1 + 0.01 * rng.uniform(-1, 1, rho.shape)), fxN + 0.01 * rng.uniform(-1, 1, fx0.shape))
    return o, d, U0, dts, targets


def split(U, nd):
    return U[0], U[1:1 + nd], U[1 + nd], U[2 + nd:]


def final_fields(d, o, U, dts):
    nd = d.ndim
    U = U.copy()
    rho, rhou, E, fx = split(U, nd)
    o.boundaries(rho, rhou, E, fx)
    d.set_state(rho, rhou, E, fx)
    d.run(nsteps=len(dts), dts=dts)
    fxN = np.zeros_like(fx)
    rN = d.get_state(fx=fxN)[0]
    s = interior(nd)
    return rN[s].copy(), fxN[(slice(None),) + s].copy()


def objective(d, o, U, dts, targets):
    nd = d.ndim
    s = interior(nd)
    rN, xN = final_fields(d, o, U, dts)
    return 0.5 * float(np.sum((rN - targets[0][s]) ** 2)) + 0.5 * float(
        np.sum((xN - targets[1][(slice(None),) + s]) ** 2))


def gradient(d, U0, dts, targets, precision, k=4):
    nd = d.ndim
    rho, rhou, E, fx = split(U0, nd)
    d.set_state(rho, rhou, E, fx)
    d.adjoint_forward(len(dts), dts=dts, precision=precision, checkpoint_every=k)
    fxN = np.zeros_like(fx)
    rN = d.get_state(fx=fxN)[0]
    lam = np.zeros_like(U0)
    s = interior(nd)
    lam[0][s] = (rN - targets[0])[s]
    lam[2 + nd:][(slice(None),) + s] = (fxN - targets[1])[(slice(None),) + s]
    return d.adjoint_backward(lam)


@pytest.mark.parametrize("name", list(CASES))
def test_scalar_adjoint_matches_finite_differences(name):
    o, d, U0, dts, targets = problem(name)
    nd = d.ndim
    g = gradient(d, U0, dts, targets, "fp64")
    s = (slice(None),) + interior(nd)
    rng = np.random.default_rng(77)
    eps = 1e-8
    errs = []
    # directions in every variable, then in the scalars' planes only (the
    # part of the gradient this change adds: the scalars' own adjoints)
    for trial in range(12):
        v = np.zeros_like(U0)
        v[s] = rng.uniform(-1, 1, U0[s].shape) * np.abs(U0[s])
        if trial >= 8:
            v[:2 + nd] = 0.0
        fp = objective(d, o, U0 + eps * v, dts, targets)
        fm = objective(d, o, U0 - eps * v, dts, targets)
        fd = (fp - fm) / (2 * eps)
        ad = float(np.sum(g * v))
        errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
    errs = np.array(errs)
    print(f"{name}: FD rel err median {np.median(errs):.2e} max {errs.max():.2e}")
    assert np.median(errs) < 1e-5, errs
    if CASES[name][3]["limiter"] == "Minmod":
        # Minmod is piecewise linear with a kink at |R| = |L|; over the steps
        # of the evolved state some cell's |R| and |L| come within ~1e-6 of
        # each other, and a central difference that straddles that kink
        # measures the kink, not the gradient: one direction may do so
        assert np.sort(errs)[-2] < 1e-3, errs
    else:
        assert np.max(errs) < 1e-3, errs
    # the gradient lives on the interior; ghost entries are zero
    mask = np.ones(U0.shape, bool)
    mask[s] = False
    assert np.all(g[mask] == 0)
    # the scalars' planes carry a gradient
    assert np.any(g[2 + nd:] != 0)
    d.close()


@pytest.mark.parametrize("name", ["cart_1d", "cart_2d_two", "sph_2d"])
def test_scalar_mixed_sweep_close_to_fp64(name):
    """The FP32 sweep (FP32-mixed forward and recomputation) against the FP64
    sweep on the FP64 forward: different branches at rounding-level ties and
    FP32 rounding bound the agreement (the bound of the other mixed-sweep
    tests)."""
    o, d, U0, dts, targets = problem(name)
    g64 = gradient(d, U0, dts, targets, "fp64")
    d.close()
    ndim, nx, nfx, kw, _ = CASES[name]
    dm = Domain(ndim, nx, nfx=nfx, precision="fp32_mixed", **kw)
    g32 = gradient(dm, U0, dts, targets, "fp32_mixed")
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    nd = ndim
    relx = np.linalg.norm(g32[2 + nd:] - g64[2 + nd:]) / np.linalg.norm(g64[2 + nd:])
    print(f"{name}: mixed vs fp64 adjoint rel L2 {rel:.2e}, scalars {relx:.2e}")
    assert rel < 1e-3, rel
    assert relx < 1e-3, relx
    dm.close()


def test_scalar_sweep_beyond_shared_memory_is_refused():
    """Two scalars in a 3-D FP64 sweep need more than the 227 KB of shared
    memory a B200 block may use: the forward pass refuses them up front, and
    the FP32 sweep of the same handle runs."""
    kw = CASES["cart_3d"][3]
    o = Oracle(3, [12, 10, 8], nfx=2, **oracle_kwargs(kw))
    rho0, u0, P0, fx0 = smooth_state(o, 3, 2, kw)
    rho, rhou, E, _ = o.init_from_prim(rho0, u0, P0)
    o.boundaries(rho, rhou, E, fx0)
    d = Domain(3, [12, 10, 8], nfx=2, precision="fp64", **kw)
    d.set_state(rho, rhou, E, fx0)
    with pytest.raises(HclError, match="shared memory"):
        d.adjoint_forward(2, precision="fp64", checkpoint_every=2)
    d.set_state(rho, rhou, E, fx0)
    d.adjoint_forward(2, precision="fp32_mixed", checkpoint_every=2)
    lam = np.zeros((3 + 2 + 2,) + rho.shape)
    lam[5][interior(3)] = 1.0
    g = d.adjoint_backward(lam)
    assert np.all(np.isfinite(g)) and np.any(g[5:] != 0)
    d.close()
