"""Configurations shared by the parity tests: the same physics keys feed the
oracle (tests only) and the product's Domain."""
from __future__ import annotations

import numpy as np

from heraclespp_b200 import setups

# name -> (ndim, nx, physics kwargs, setup name, setup kwargs)
CASES = {
    "sod_1d": (1, [1024], dict(gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 2),
               "shock_tube", {}),
    "sod_1d_odd": (1, [100], dict(gamma=1.4, limiter="VanAlbada", riemann="HLL", bc=["NullGradient", "Reflexive"]),
                   "shock_tube", {}),
    "advection_1d": (1, [128], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 2),
                     "advection_sinus", {}),
    "kh_2d": (2, [64, 64], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4),
              "kelvin_helmholtz", {}),
    "kh_2d_ragged": (2, [37, 21], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4),
                     "kelvin_helmholtz", {}),
    "quad_2d": (2, [48, 40], dict(gamma=1.4, limiter="Minmod", riemann="HLLC",
                                  bc=["NullGradient", "Reflexive", "Reflexive", "NullGradient"]),
                "four_quadrant", {}),
    "gresho_2d_lowmach": (2, [32, 32], dict(gamma=5.0 / 3.0, limiter="Constant", riemann="Low Mach",
                                            bc=["Periodic"] * 4), "gresho_vortex", {}),
    "rt_3d": (3, [16, 16, 32], dict(gamma=1.4, limiter="Minmod", riemann="HLL",
                                    bc=["Periodic", "Periodic", "Periodic", "Periodic", "Reflexive", "Reflexive"],
                                    g=(0.0, 0.0, -0.1), xmax=(0.5, 0.5, 1.0)), "rayleigh_taylor3d", {}),
    "rt_3d_ragged": (3, [30, 14, 21], dict(gamma=1.4, limiter="Minmod", riemann="HLL",
                                           bc=["Periodic", "Periodic", "Periodic", "Periodic", "Reflexive",
                                               "Reflexive"], g=(0.0, 0.0, -0.1), xmax=(0.5, 0.5, 1.0)),
                     "rayleigh_taylor3d", {}),
    "rt_3d_hllc": (3, [29, 13, 16], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC",
                                         bc=["NullGradient", "NullGradient", "Periodic", "Periodic", "Reflexive",
                                             "Reflexive"], g=(0.02, 0.0, -0.1), xmax=(0.5, 0.5, 1.0)),
                   "rayleigh_taylor3d", {}),
    "sph_1d_pointmass": (1, [96], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                                       bc=["Reflexive", "NullGradient"], gravity="Point_mass", central_mass=1e8,
                                       xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)), "shock_tube", {"inter": 0.7}),
    "sph_1d_internalmass": (1, [96], dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", geometry="Spherical",
                                          bc=["Reflexive", "NullGradient"], gravity="Internal_mass",
                                          central_mass=1e8, xmin=(0.2, 0.0, 0.0), xmax=(1.2, 1.0, 1.0)),
                            "shock_tube", {"inter": 0.7}),
    "sph_2d_internalmass": (2, [40, 24], dict(gamma=1.4, limiter="Minmod", riemann="HLLC", geometry="Spherical",
                                              bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive"],
                                              gravity="Internal_mass", central_mass=3e7,
                                              xmin=(0.2, 0.5, 0.0), xmax=(1.0, 2.6, 1.0)),
                            "shock_tube", {"inter": 0.6}),
    "sph_2d": (2, [40, 24], dict(gamma=1.4, limiter="Minmod", riemann="HLLC", geometry="Spherical",
                                 bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive"],
                                 xmin=(0.2, 0.5, 0.0), xmax=(1.0, 2.6, 1.0)), "shock_tube", {"inter": 0.6}),
    "sph_3d": (3, [12, 10, 8], dict(gamma=1.4, limiter="VanLeer", riemann="HLL", geometry="Spherical",
                                    bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive", "Periodic",
                                        "Periodic"], xmin=(0.3, 0.6, 0.0), xmax=(1.0, 2.5, 1.5)),
               "shock_tube", {"inter": 0.65, "u0": 0.1}),
}


def oracle_kwargs(kw):
    out = dict(kw)
    if "geometry" in out:
        out["geom"] = out.pop("geometry")
    return out


def make_pair(name, precision="fp64"):
    """(oracle, domain, (rho, u, P) interior primitives)."""
    from oracle import Oracle
    from heraclespp_b200 import Domain

    ndim, nx, kw, setup, skw = CASES[name]
    o = Oracle(ndim, nx, **oracle_kwargs(kw))
    d = Domain(ndim, nx, precision=precision, **kw)
    grid = setups.Grid.from_domain(o)
    prim = setups.SETUPS[setup](grid, **skw)
    return o, d, prim


def rel_l1(a, b):
    den = np.sum(np.abs(b))
    return float(np.sum(np.abs(a - b)) / den) if den > 0 else float(np.sum(np.abs(a - b)))
