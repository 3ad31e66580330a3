"""The oracle's InternalMassGravity (gravity.cpp:59-128) against closed forms:
a uniform-density sphere around a central mass, and shell means of a density
that varies with the polar angle."""
import numpy as np

from oracle import Oracle

G = 6.6743015E-11


def _arrays(o):
    n0 = o.ctx.n[0]
    x = np.ctypeslib.as_array(o.ctx.x[0], shape=(n0 + 1,)).copy()
    xc = np.ctypeslib.as_array(o.ctx.xc[0], shape=(n0,)).copy()
    return x, xc


def test_uniform_sphere_closed_form():
    M0, rho0, ng = 1e9, 3.0, 2
    o = Oracle(1, [64], gamma=1.4, limiter="VanLeer", riemann="HLLC", geom="Spherical",
               bc=["Reflexive", "NullGradient"], gravity="Internal_mass", central_mass=M0,
               xmin=(0.2, 0, 0), xmax=(1.2, 1, 1))
    g = o.internal_mass_gravity(np.full(o.zeros().shape, rho0))
    x, xc = _arrays(o)
    # enclosed mass at the cell centres: the central mass plus the gas between
    # the inner face of the first interior cell and xc (the ghosts: M0 alone)
    M = np.where(np.arange(xc.size) < ng, M0, M0 + 4 * np.pi / 3 * rho0 * (xc ** 3 - x[ng] ** 3))
    assert np.max(np.abs(g - (-G * M / xc ** 2)) / (G * M / xc ** 2)) < 1e-13


def test_shell_means_over_the_polar_angle():
    """2-D spherical: the density of a shell is its volume-weighted mean over
    the interior polar cells; with rho depending on theta only, every shell
    has the same mean and M grows like the uniform sphere with that mean."""
    ng, M0 = 2, 5e8
    o = Oracle(2, [32, 16], gamma=1.4, limiter="Minmod", riemann="HLLC", geom="Spherical",
               bc=["Reflexive", "NullGradient", "Reflexive", "Reflexive"], gravity="Internal_mass",
               central_mass=M0, xmin=(0.3, 0.4, 0), xmax=(1.0, 2.7, 1))
    shape = o.zeros().shape  # (n2, n1, n0)
    th = np.ctypeslib.as_array(o.ctx.xc[1], shape=(o.ctx.n[1],)).copy()
    rho = np.ascontiguousarray(np.broadcast_to((1.0 + 0.5 * np.cos(th))[None, :, None], shape))
    dv = np.ctypeslib.as_array(o.ctx.dv, shape=rho.shape)
    s1 = slice(ng, ng + 16)
    w = dv[0, s1, ng]  # the volume weights of one shell (k = 0 plane, i = ng)
    mean = float(np.sum(rho[0, s1, ng] * w) / np.sum(w))
    g = o.internal_mass_gravity(rho)
    x, xc = _arrays(o)
    M = np.where(np.arange(xc.size) < ng, M0, M0 + 4 * np.pi / 3 * mean * (xc ** 3 - x[ng] ** 3))
    assert np.max(np.abs(g - (-G * M / xc ** 2)) / (G * M / xc ** 2)) < 1e-12
