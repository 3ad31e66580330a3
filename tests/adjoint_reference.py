"""Loop-based reference of one fused step and of its discrete adjoint on a
small periodic 2-D grid, built from the per-cell functions of
heraclespp_b200/csrc/adjoint_cell.cuh (compiled for the host by the tests).

Test infrastructure: it restates the step's structure (primitives, limited
slopes, Hancock face states, one Riemann solve per face, Godunov update,
periodic ghosts) so the GPU adjoint kernel can be compared to it cell by cell.
Arrays are [var, j, i] with 2 ghost layers.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

NG = 2
KB = 1.380649e-23  # units.hpp: Boltzmann constant
MP = 1.672649e-27  # units.hpp: proton mass
ROOT = Path(__file__).resolve().parents[1]


def build_cell_lib(out):
    """Compiles tests/adjoint_cell_check.cpp (the per-cell forward and reverse
    functions of adjoint_cell.cuh as host code) into `out` and loads it."""
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "heraclespp_b200" / "csrc"),
                    str(ROOT / "tests" / "adjoint_cell_check.cpp"), "-o", str(out)], check=True)
    L = C.CDLL(str(out))
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.t_riemann_fwd.argtypes = [i, i, d, vp, vp, i, vp]
    L.t_riemann_rev.argtypes = [i, i, d, vp, vp, i, vp, vp, vp]
    L.t_flux_fwd.argtypes = [d, vp, i, vp]
    L.t_flux_rev.argtypes = [d, vp, i, vp, vp]
    L.t_p2c_fwd.argtypes = [d, vp, vp]
    L.t_p2c_rev.argtypes = [d, vp, vp, vp]
    L.t_c2p_fwd.argtypes = [d, vp, vp]
    L.t_c2p_rev.argtypes = [d, vp, vp, vp]
    L.t_limiter.argtypes = [i, d, d, C.POINTER(d), C.POINTER(d)]
    L.t_limiter.restype = d
    L.t_limiter_on.argtypes = [i, i, d, d, C.POINTER(d), C.POINTER(d)]
    L.t_limiter_on.restype = d
    return L


def p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.c_void_p)


def smooth_state(n, seed=0):
    """Smooth seeded periodic 2-D conserved state [4, n+4, n+4] (gamma 1.4)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    rho = 1 + 0.2 * np.sin(2 * np.pi * X + 0.3) * np.cos(2 * np.pi * Y + 0.7) + 0.05 * rng.uniform(-1, 1, (n, n))
    u = 0.3 * np.sin(2 * np.pi * Y + 0.1) + 0.05 * rng.uniform(-1, 1, (n, n))
    v = 0.2 * np.cos(2 * np.pi * X + 0.5) + 0.05 * rng.uniform(-1, 1, (n, n))
    P = 1 + 0.1 * np.cos(2 * np.pi * (X + Y)) + 0.05 * rng.uniform(-1, 1, (n, n))
    gamma = 1.4
    U = np.zeros((4, n + 2 * NG, n + 2 * NG))
    s = (slice(NG, NG + n), slice(NG, NG + n))
    U[0][s] = rho
    U[1][s] = rho * u
    U[2][s] = rho * v
    U[3][s] = P / (gamma - 1) + 0.5 * rho * (u * u + v * v)
    Ref.fill_periodic(U)
    return U


class Ref:
    def __init__(self, lib, gamma=1.4, lim=1, solver=1):
        self.L = lib
        self.g = gamma
        self.lim = lim
        self.solver = solver
        self.dx = (1.0, 1.0)  # cell spacing of the step being evaluated

    # ---- per-cell wrappers -----------------------------------------------
    def c2p(self, U):
        """Primitives rounded as the forward FP64 step rounds them (the
        perfect gas's temperature round trip, mmw = 1), which is where the
        FP64 sweep takes its branch decisions from."""
        rho, m0, m1, E = (float(x) for x in U)
        ek = (m0 * m0 + m1 * m1) / rho / 2
        T = (E - ek) * MP * (self.g - 1.0) / (rho * KB)
        return np.array([rho, m0 / rho, m1 / rho, rho * KB * T / MP])

    def c2p_rev(self, U, Wb):
        Ub = np.zeros(4)
        self.L.t_c2p_rev(self.g, p(U), p(Wb), Ub.ctypes.data_as(C.c_void_p))
        return Ub

    def p2c(self, W):
        U = np.zeros(4)
        self.L.t_p2c_fwd(self.g, p(W), U.ctypes.data_as(C.c_void_p))
        return U

    def p2c_rev(self, W, Ub):
        Wb = np.zeros(4)
        self.L.t_p2c_rev(self.g, p(W), p(Ub), Wb.ctypes.data_as(C.c_void_p))
        return Wb

    def flux(self, W, l):
        F = np.zeros(4)
        self.L.t_flux_fwd(self.g, p(W), l, F.ctypes.data_as(C.c_void_p))
        return F

    def flux_rev(self, W, l, Fb):
        Wb = np.zeros(4)
        self.L.t_flux_rev(self.g, p(W), l, p(Fb), Wb.ctypes.data_as(C.c_void_p))
        return Wb

    def riemann(self, UL, UR, l):
        F = np.zeros(4)
        self.L.t_riemann_fwd(2, self.solver, self.g, p(UL), p(UR), l, F.ctypes.data_as(C.c_void_p))
        return F

    def riemann_rev(self, UL, UR, l, Fb):
        a, b = np.zeros(4), np.zeros(4)
        self.L.t_riemann_rev(2, self.solver, self.g, p(UL), p(UR), l, p(Fb), a.ctypes.data_as(C.c_void_p),
                             b.ctypes.data_as(C.c_void_p))
        return a, b

    def limiter(self, R, L, dx=None):
        """phi(R, L) of raw differences and its partials.  With the cell
        spacing dx the branch is the forward step's: the sign of
        (R/dx)*(L/dx), as it forms the limiter's arguments (the raw product
        can underflow to 0 where that one does not)."""
        gR, gL = C.c_double(), C.c_double()
        if dx is None:
            phi = self.L.t_limiter(self.lim, float(R), float(L), C.byref(gR), C.byref(gL))
        else:
            prod = float(R) * float(L)
            active = prod > 0 if abs(prod) > 1e-270 * (dx * dx) else (float(L) / dx) * (float(R) / dx) > 0
            phi = self.L.t_limiter_on(self.lim, 1 if active else 0, float(R), float(L), C.byref(gR), C.byref(gL))
        return phi, gR.value, gL.value

    # ---- grid helpers ------------------------------------------------------
    @staticmethod
    def fill_periodic(U):
        n1, n0 = U.shape[1] - 2 * NG, U.shape[2] - 2 * NG
        U[:, :NG, :] = U[:, n1:n1 + NG, :]
        U[:, n1 + NG:, :] = U[:, NG:2 * NG, :]
        U[:, :, :NG] = U[:, :, n0:n0 + NG]
        U[:, :, n0 + NG:] = U[:, :, NG:2 * NG]

    @staticmethod
    def fold_periodic(lam):
        """Transpose of fill_periodic: ghost adjoints onto their sources."""
        n1, n0 = lam.shape[1] - 2 * NG, lam.shape[2] - 2 * NG
        lam[:, :, n0:n0 + NG] += lam[:, :, :NG]
        lam[:, :, NG:2 * NG] += lam[:, :, n0 + NG:]
        lam[:, :, :NG] = 0
        lam[:, :, n0 + NG:] = 0
        lam[:, n1:n1 + NG, :] += lam[:, :NG, :]
        lam[:, NG:2 * NG, :] += lam[:, n1 + NG:, :]
        lam[:, :NG, :] = 0
        lam[:, n1 + NG:, :] = 0

    # ---- forward -----------------------------------------------------------
    def faces(self, W, j, i, cth):
        """Hancock face states [xL, xR, yB, yT] of cell (j, i) and the intermediates."""
        wc = W[:, j, i]
        fp = {}
        for d, (dj, di) in enumerate(((0, 1), (1, 0))):
            fl = np.zeros(4)
            fr = np.zeros(4)
            for v in range(4):
                phi, _, _ = self.limiter(W[v, j + dj, i + di] - wc[v], wc[v] - W[v, j - dj, i - di], self.dx[d])
                fl[v] = wc[v] - 0.5 * phi
                fr[v] = wc[v] + 0.5 * phi
            fp[(0, d)] = fl
            fp[(1, d)] = fr
        inc = np.zeros(4)
        for d in range(2):
            inc += cth[d] * (self.flux(fp[(0, d)], d) - self.flux(fp[(1, d)], d))
        H = {}
        for key, w in fp.items():
            H[key] = self.p2c(w) + inc
        return H, fp

    def step(self, U, dt, dx):
        self.dx = dx
        n1, n0 = U.shape[1] - 2 * NG, U.shape[2] - 2 * NG
        cth = [0.5 * dt / dx[0], 0.5 * dt / dx[1]]
        W = np.zeros_like(U)
        for j in range(U.shape[1]):
            for i in range(U.shape[2]):
                W[:, j, i] = self.c2p(U[:, j, i])
        H = {}
        for j in range(NG - 1, NG + n1 + 1):
            for i in range(NG - 1, NG + n0 + 1):
                H[(j, i)], _ = self.faces(W, j, i, cth)
        out = U.copy()
        for j in range(NG, NG + n1):
            for i in range(NG, NG + n0):
                Fl = self.riemann(H[(j, i - 1)][(1, 0)], H[(j, i)][(0, 0)], 0)
                Fr = self.riemann(H[(j, i)][(1, 0)], H[(j, i + 1)][(0, 0)], 0)
                Gl = self.riemann(H[(j - 1, i)][(1, 1)], H[(j, i)][(0, 1)], 1)
                Gr = self.riemann(H[(j, i)][(1, 1)], H[(j + 1, i)][(0, 1)], 1)
                out[:, j, i] = U[:, j, i] + dt / dx[0] * (Fl - Fr) + dt / dx[1] * (Gl - Gr)
        self.fill_periodic(out)
        return out

    # ---- adjoint -----------------------------------------------------------
    def step_adjoint(self, U, lam_out, dt, dx):
        """lam_out: adjoint of the interior outputs (ghost entries ignored).
        Returns the adjoint of the full input U (ghost entries folded)."""
        self.dx = dx
        n1, n0 = U.shape[1] - 2 * NG, U.shape[2] - 2 * NG
        cth = [0.5 * dt / dx[0], 0.5 * dt / dx[1]]
        c = [dt / dx[0], dt / dx[1]]
        lo = np.zeros_like(U)
        lo[:, NG:NG + n1, NG:NG + n0] = lam_out[:, NG:NG + n1, NG:NG + n0]
        W = np.zeros_like(U)
        for j in range(U.shape[1]):
            for i in range(U.shape[2]):
                W[:, j, i] = self.c2p(U[:, j, i])
        H = {}
        for j in range(NG - 1, NG + n1 + 1):
            for i in range(NG - 1, NG + n0 + 1):
                H[(j, i)], _ = self.faces(W, j, i, cth)
        Hb = {key: {k: np.zeros(4) for k in ((0, 0), (1, 0), (0, 1), (1, 1))} for key in H}
        # every face used by an interior cell: x-faces i-1/2 for i in [NG, NG+n0], same for y
        for j in range(NG, NG + n1):
            for i in range(NG, NG + n0 + 1):
                Fb = c[0] * (lo[:, j, i] - lo[:, j, i - 1])
                a, b = self.riemann_rev(H[(j, i - 1)][(1, 0)], H[(j, i)][(0, 0)], 0, Fb)
                Hb[(j, i - 1)][(1, 0)] += a
                Hb[(j, i)][(0, 0)] += b
        for j in range(NG, NG + n1 + 1):
            for i in range(NG, NG + n0):
                Fb = c[1] * (lo[:, j, i] - lo[:, j - 1, i])
                a, b = self.riemann_rev(H[(j - 1, i)][(1, 1)], H[(j, i)][(0, 1)], 1, Fb)
                Hb[(j - 1, i)][(1, 1)] += a
                Hb[(j, i)][(0, 1)] += b
        Wb = np.zeros_like(U)
        for (j, i), hb in Hb.items():
            _, fp = self.faces(W, j, i, cth)
            fpb = {k: np.zeros(4) for k in fp}
            Sb = np.zeros(4)
            for key, b in hb.items():
                Sb += b
                fpb[key] += self.p2c_rev(fp[key], b)
            for d in range(2):
                fpb[(0, d)] += self.flux_rev(fp[(0, d)], d, cth[d] * Sb)
                fpb[(1, d)] += self.flux_rev(fp[(1, d)], d, -cth[d] * Sb)
            for d, (dj, di) in enumerate(((0, 1), (1, 0))):
                for v in range(4):
                    wc = W[v, j, i]
                    _, gR, gL = self.limiter(W[v, j + dj, i + di] - wc, wc - W[v, j - dj, i - di], self.dx[d])
                    phib = 0.5 * (fpb[(1, d)][v] - fpb[(0, d)][v])
                    Wb[v, j, i] += fpb[(0, d)][v] + fpb[(1, d)][v] - phib * gR + phib * gL
                    Wb[v, j + dj, i + di] += phib * gR
                    Wb[v, j - dj, i - di] -= phib * gL
        lam_in = np.zeros_like(U)
        lam_in[:, NG:NG + n1, NG:NG + n0] += lo[:, NG:NG + n1, NG:NG + n0]
        for j in range(U.shape[1]):
            for i in range(U.shape[2]):
                if np.any(Wb[:, j, i] != 0):
                    lam_in[:, j, i] += self.c2p_rev(U[:, j, i], Wb[:, j, i])
        self.fold_periodic(lam_in)
        return lam_in
