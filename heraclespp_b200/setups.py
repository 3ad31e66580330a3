"""Setup plugins: initial primitive states on the interior cells.

Mirrors the reference's setup contract (src/initialization_interface.hpp:18-40,
src/setups/<name>/setup.hpp): ``ParamSetup`` values come from the .ini
``[Initialisation]`` section and ``execute(grid)`` returns rho, u, P on the
no_ghosts range (ghost entries stay zero; the boundaries fill them).

Seeded noise uses a counter-based hash of (seed, i, j, k) on the global
interior index, so a cell's perturbation does not depend on the grid split or
on the order of evaluation; the C++ host layer implements the same hash.
"""
from __future__ import annotations

import math

import numpy as np

M64 = (1 << 64) - 1


def _splitmix64(x):
    """splitmix64 finaliser on uint64 numpy arrays (wrapping arithmetic)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(M64)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(M64)
    return z ^ (z >> np.uint64(31))


def hash_uniform(seed, i, j, k):
    """Uniform double in [0, 1) from (seed, i, j, k) -- same as hcl_hash_uniform in C++."""
    with np.errstate(over="ignore"):
        h = _splitmix64(np.asarray(k, dtype=np.uint64))
        h = _splitmix64(h ^ np.asarray(j, dtype=np.uint64))
        h = _splitmix64(h ^ np.asarray(i, dtype=np.uint64))
        h = _splitmix64(h ^ np.uint64(seed))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class Grid:
    """The parts of Grid a setup reads: centres, extents, ghost count."""

    def __init__(self, ndim, n, ng, xc):
        self.ndim = ndim
        self.n = n
        self.ng = ng
        self.xc = xc  # list of 3 arrays of cell centres (with ghosts)

    @classmethod
    def from_domain(cls, dom_or_oracle, ng=2):
        g = dom_or_oracle.grid()
        return cls(dom_or_oracle.ndim, dom_or_oracle.n, ng, [g["x0c"], g["x1c"], g["x2c"]])

    def interior(self):
        """(slices, centres broadcast over the interior, interior index arrays)"""
        sl = []
        idx = []
        for d in range(3):
            if d < self.ndim:
                sl.append(slice(self.ng, self.n[d] - self.ng))
            else:
                sl.append(slice(0, 1))
        # numpy order is (k, j, i)
        s3 = (sl[2], sl[1], sl[0])
        X = self.xc[0][sl[0]][None, None, :]
        Y = self.xc[1][sl[1]][None, :, None]
        Z = self.xc[2][sl[2]][:, None, None]
        i = np.arange(sl[0].stop - sl[0].start)[None, None, :]
        j = np.arange(sl[1].stop - sl[1].start)[None, :, None]
        k = np.arange(sl[2].stop - sl[2].start)[:, None, None]
        return s3, (X, Y, Z), (i, j, k)

    def alloc(self):
        shape = (self.n[2], self.n[1], self.n[0])
        return np.zeros(shape), np.zeros((self.ndim,) + shape), np.zeros(shape)


def shock_tube(grid, rho0=1.0, rho1=0.125, u0=0.0, u1=0.0, P0=1.0, P1=0.1, inter=0.5):
    """setups/shock_tube/setup.hpp:74-91 (left state where x0 <= inter)."""
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    left = np.broadcast_to(X <= inter, rho[s3].shape)
    rho[s3] = np.where(left, rho0, rho1)
    P[s3] = np.where(left, P0, P1)
    for d in range(grid.ndim):
        u[d][s3] = np.where(left, u0, u1)
    return rho, u, P


def advection_sinus(grid, u0=1.0, P0=0.1):
    """setups/advection_sinus/setup.hpp:61-72."""
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    rho[s3] = np.broadcast_to(1.0 + 1e-1 * np.sin(2 * math.pi * X), rho[s3].shape)
    for d in range(grid.ndim):
        u[d][s3] = u0
    P[s3] = P0
    return rho, u, P


def kelvin_helmholtz(grid, seed=1234, noise=1e-3):
    """2-D shear layer on [0,1]^2: rho=2, vx=+0.5 where |y-0.5|<0.25, else rho=1,
    vx=-0.5; p=2.5; vy = 0.01 sin(4 pi x) + seeded U(-noise, noise)."""
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), (i, j, k) = grid.interior()
    shape = rho[s3].shape
    band = np.broadcast_to(np.abs(Y - 0.5) < 0.25, shape)
    rho[s3] = np.where(band, 2.0, 1.0)
    u[0][s3] = np.where(band, 0.5, -0.5)
    r = hash_uniform(seed, i, j, k)
    u[1][s3] = np.broadcast_to(0.01 * np.sin(4 * math.pi * X), shape) + noise * (2.0 * r - 1.0)
    P[s3] = 2.5
    return rho, u, P


def rayleigh_taylor_3d(grid, seed=4321, g=-0.1, noise=1e-4):
    """3-D RT on [0,0.5]^2 x [0,1]: rho=2 above z=0.5, 1 below; hydrostatic
    p with p=2.5 at the interface; vz seeded mode + U(-noise, noise)."""
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), (i, j, k) = grid.interior()
    shape = rho[s3].shape
    upper = np.broadcast_to(Z > 0.5, shape)
    rho[s3] = np.where(upper, 2.0, 1.0)
    P[s3] = np.broadcast_to(2.5 + np.where(Z > 0.5, 2.0, 1.0) * g * (Z - 0.5), shape)
    r = hash_uniform(seed, i, j, k)
    mode = 0.01 * (1 + np.cos(4 * math.pi * X)) * (1 + np.cos(4 * math.pi * Y)) * (1 + np.cos(3 * math.pi * Z)) / 8
    u[2][s3] = np.broadcast_to(mode, shape) + noise * (2.0 * r - 1.0)
    return rho, u, P


def gresho_vortex(grid, p0=5.0, rho0=1.0):
    """Gresho vortex centred at (0.5, 0.5): u_phi = 5r (r<0.2), 2-5r (r<0.4),
    0 beyond; pressure from radial balance with p0 (as in
    setups/gresho_vortex/setup.hpp:76-100, re-centred, p0 given)."""
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    shape = rho[s3].shape
    x = np.broadcast_to(X - 0.5, shape)
    y = np.broadcast_to(Y - 0.5, shape)
    r = np.sqrt(x * x + y * y)
    th = np.arctan2(y, x)
    uphi = np.where(r < 0.2, 5 * r, np.where(r < 0.4, 2 - 5 * r, 0.0))
    with np.errstate(divide="ignore"):
        p_mid = p0 + 12.5 * r * r + 4 - 20 * r + 4 * np.log(np.maximum(5 * r, 1e-300))
    pr = np.where(r < 0.2, p0 + 12.5 * r * r, np.where(r < 0.4, p_mid, p0 - 2 + 4 * math.log(2.0)))
    rho[s3] = rho0
    u[0][s3] = -uphi * np.sin(th)
    u[1][s3] = uphi * np.cos(th)
    P[s3] = pr
    return rho, u, P


def four_quadrant(grid, seed=7):
    """2-D four-quadrant Riemann problem with seeded states: rho, p in
    U[0.1, 2], velocities in U[-1, 1] per quadrant (split at x=y=0.5)."""
    h = lambda q, c: float(hash_uniform(seed, q, c, 1))  # noqa: E731
    states = [(0.1 + 1.9 * h(q, 0), -1.0 + 2.0 * h(q, 1), -1.0 + 2.0 * h(q, 2), 0.1 + 1.9 * h(q, 3)) for q in range(4)]
    rho, u, P = grid.alloc()
    s3, (X, Y, Z), _ = grid.interior()
    shape = rho[s3].shape
    q = (np.broadcast_to(X > 0.5, shape).astype(int) + 2 * np.broadcast_to(Y > 0.5, shape).astype(int))
    for qi, (r_, ux, uy, p_) in enumerate(states):
        m = q == qi
        rho[s3][m] = r_
        u[0][s3][m] = ux
        u[1][s3][m] = uy
        P[s3][m] = p_
    return rho, u, P


SETUPS = {
    "shock_tube": shock_tube,
    "advection_sinus": advection_sinus,
    "kelvin_helmholtz": kelvin_helmholtz,
    "rayleigh_taylor3d": rayleigh_taylor_3d,
    "gresho_vortex": gresho_vortex,
    "four_quadrant": four_quadrant,
}
