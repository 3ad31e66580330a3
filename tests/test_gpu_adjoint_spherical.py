"""GPU checks of the discrete adjoint on spherical grids (hcl_adjoint_* with
geometry "Spherical") and of the 1-D and 3-D reverse tiles: the face areas over the cell volumes in the flux
differences (extrapolation_reconstruction.hpp:130-142, godunov_scheme.hpp:
157-163) and the geometric source terms of the predictor and the update
(hydro/source_terms.hpp:16-77; extrapolation_reconstruction.hpp:145-303,
godunov_scheme.hpp:165-256), in 1-D, 2-D and 3-D.

Smooth states whose normal velocity vanishes at the reflecting walls, dt
recorded from a CFL run and held fixed; J = 0.5 ||rho^N - rho_target||^2 over
the interior.  The FP64 gradient is checked against central differences of the
FP64 forward along seeded random directions, and the FP32 sweep against the
FP64 one."""
import numpy as np
import pytest

from cases import oracle_kwargs
from heraclespp_b200 import Domain, setups
from oracle import Oracle

pytestmark = pytest.mark.gpu
NG = 2

# name: (ndim, cells, domain kwargs, steps); the Cartesian cases run the same
# states through the 1-D and 3-D reverse tiles without the geometric terms
CASES = {
    "sph_1d": (1, [64], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                             bc=["Reflexive", "NullGradient"], xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), 16),
    "sph_1d_pointmass": (1, [64], dict(gamma=1.4, limiter="VanAlbada", riemann="HLL", geometry="Spherical",
                                       bc=["Reflexive", "NullGradient"], gravity="Point_mass", central_mass=1e8,
                                       xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), 16),
    # internal-mass gravity (gravity.cpp:59-128): g_r = -G M(r) / r^2 rebuilt
    # from every step's input density, so the density also enters through the
    # enclosed mass of every shell outside it; rho and P carry RHO_SCALE so
    # that the gas's own mass (G M_gas ~ 0.05) is comparable to the central
    # mass's pull
    "sph_1d_internalmass": (1, [64], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                                          bc=["Reflexive", "NullGradient"], gravity="Internal_mass",
                                          central_mass=2e7, xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), 16),
    "sph_2d_internalmass": (2, [40, 24], dict(gamma=1.4, limiter="VanLeer", riemann="HLL", geometry="Spherical",
                                              bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive"],
                                              gravity="Internal_mass", central_mass=2e7,
                                              xmin=(0.2, 0.5, 0.0), xmax=(1.0, 2.6, 1.0)), 12),
    "sph_2d": (2, [40, 24], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                                 bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive"],
                                 xmin=(0.2, 0.5, 0.0), xmax=(1.0, 2.6, 1.0)), 12),
    "sph_3d": (3, [12, 10, 8], dict(gamma=1.4, limiter="VanLeer", riemann="HLL", geometry="Spherical",
                                    bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive", "Periodic", "Periodic"],
                                    xmin=(0.3, 0.6, 0.0), xmax=(1.0, 2.5, 1.5)), 10),
    "cart_1d": (1, [64], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Reflexive", "NullGradient"],
                              xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), 16),
    "cart_3d": (3, [12, 10, 8], dict(gamma=1.4, limiter="VanLeer", riemann="HLL",
                                     bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive", "Periodic", "Periodic"],
                                     xmin=(0.3, 0.6, 0.0), xmax=(1.0, 2.5, 1.5)), 10),
}


RHO_SCALE = {"sph_1d_internalmass": 1e8, "sph_2d_internalmass": 1e8}


def interior(ndim):
    return (slice(NG, -NG) if ndim == 3 else slice(None), slice(NG, -NG) if ndim >= 2 else slice(None),
            slice(NG, -NG))


def smooth_state(o, ndim, kw):
    """Smooth fields whose normal velocities vanish at the reflecting walls.
    Every primitive varies along every direction and no extremum is symmetric
    about a cell face: where two neighbours hold equal values (a field that
    does not depend on one coordinate, or a mirrored extremum) the limited
    slope sits on the limiter's kink (R L = 0) and its branch is set by
    rounding, which the adjoint follows and a central difference does not."""
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
        u[1][s3] = np.broadcast_to(0.06 * np.sin(np.pi * st) * (1 + 0.3 * st) * (1 + 0.5 * sr)
                                   * (1 + 0.3 * np.sin(2 * np.pi * sp + 0.1)), shape)
    if ndim == 3:
        u[2][s3] = np.broadcast_to((0.05 * np.sin(2 * np.pi * sp + 0.2) * (0.5 + sr) + 0.02)
                                   * (1 + 0.3 * np.cos(np.pi * st + 0.25)), shape)
    return rho, u, P


def problem(name):
    ndim, nx, kw, nsteps = CASES[name]
    o = Oracle(ndim, nx, **oracle_kwargs(kw))
    rho0, u0, P0 = smooth_state(o, ndim, kw)
    scale = RHO_SCALE.get(name, 1.0)
    rho, rhou, E, _ = o.init_from_prim(rho0 * scale, u0, P0 * scale)
    U0 = np.concatenate([rho[None], rhou, E[None]])
    d = Domain(ndim, nx, precision="fp64", **kw)
    d.set_state(rho, rhou, E)
    r = d.run(cfl=0.4, nsteps=nsteps)
    assert r.iter == nsteps
    dts = d.dt_log()[:nsteps]
    rng = np.random.default_rng(31)
    target = d.get_state()[0] * (1 + 0.01 * rng.uniform(-1, 1, rho.shape))
    return o, d, U0, dts, target


def final_rho(d, o, U, dts):
    nd = d.ndim
    U = U.copy()
    o.boundaries(U[0], U[1:1 + nd], U[1 + nd])
    d.set_state(U[0], U[1:1 + nd], U[1 + nd])
    d.run(nsteps=len(dts), dts=dts)
    return d.get_state()[0][interior(nd)].copy()


def gradient(d, U0, dts, target, precision, k=4):
    nd = d.ndim
    d.set_state(U0[0], U0[1:1 + nd], U0[1 + nd])
    d.adjoint_forward(len(dts), dts=dts, precision=precision, checkpoint_every=k)
    rN = d.get_state()[0]
    lam = np.zeros_like(U0)
    lam[0][interior(nd)] = (rN - target)[interior(nd)]
    return d.adjoint_backward(lam)


@pytest.mark.parametrize("name", list(CASES))
def test_spherical_adjoint_matches_finite_differences(name):
    o, d, U0, dts, target = problem(name)
    nd = d.ndim
    g = gradient(d, U0, dts, target, "fp64")
    s = (slice(None),) + interior(nd)
    t = target[interior(nd)]
    rng = np.random.default_rng(77)
    errs = []
    eps = 3e-9
    for _ in range(10):
        v = np.zeros_like(U0)
        v[s] = rng.uniform(-1, 1, U0[s].shape) * np.abs(U0[s])
        rp = final_rho(d, o, U0 + eps * v, dts)
        rm = final_rho(d, o, U0 - eps * v, dts)
        fd = float(np.sum((rp - rm) * (0.5 * (rp + rm) - t))) / (2 * eps)
        ad = float(np.sum(g * v))
        errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
    errs = np.array(errs)
    print(f"{name}: FD rel err median {np.median(errs):.2e} max {errs.max():.2e}")
    assert np.median(errs) < 1e-5, errs
    assert np.max(errs) < 1e-3, errs
    # the gradient lives on the interior; ghost entries are zero
    mask = np.ones(U0.shape, bool)
    mask[s] = False
    assert np.all(g[mask] == 0)
    d.close()


@pytest.mark.parametrize("name", ["sph_1d", "sph_2d", "sph_3d", "sph_1d_internalmass"])
def test_spherical_mixed_sweep_close_to_fp64(name):
    """The FP32 sweep decides the limiter and wave-speed branches on its own
    face states: where FP32 rounding moves an argument across a switch the two
    sweeps follow different branches of a piecewise-smooth map (the bound of
    the Cartesian mixed-sweep test)."""
    o, d, U0, dts, target = problem(name)
    g64 = gradient(d, U0, dts, target, "fp64")
    g32 = gradient(d, U0, dts, target, "fp32_mixed")
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print(f"{name}: mixed vs fp64 adjoint rel L2 {rel:.2e}")
    assert rel < 1e-3, rel
    d.close()
