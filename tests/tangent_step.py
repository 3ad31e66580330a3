"""Test infrastructure: a torch FP64 restatement of the 2-D Cartesian periodic
MUSCL-Hancock step, used to form tangent-linear products J v by forward-mode
automatic differentiation (torch.func.jvp).

Together with the library's discrete adjoint (J^T lambda) it gives the
dot-product test <J v, lambda> = <v, J^T lambda>, which holds to rounding for
an exact adjoint and so separates adjoint error from the truncation and
rounding error of finite differences.

Scope: uniform Cartesian 2-D grid, periodic in both directions (neighbours by
torch.roll), no gravity, no passive scalars, PerfectGas with the reference's
temperature round trip, van Leer or minmod slopes, HLL or HLLC.  The arithmetic
follows the oracle's C restatement expression by expression so the forward
trajectory matches the FP64 GPU step:
  * perfect_gas.hpp:46-89 (EOS), euler_equations.hpp:41-134 (algebra),
  * slope_limiters.hpp:38-66, limited_linear_reconstruction.hpp:46-64,
  * hydro_reconstruction.hpp:99-126 and extrapolation_reconstruction.hpp:90-134
    (Hancock increments on every face),
  * riemann_solver.hpp:31-134 (HLL, HLLC), godunov_scheme.hpp:110-160.
Non-smooth points take the branch the discrete adjoint differentiates
(heraclespp_b200/csrc/adjoint_cell.cuh): a limited slope is zero unless
R*L > 0; min(a, b) is a when a < b, else b; max(a, b) is a when a > b, else b;
the HLLC star side is left when u* > 0; the supersonic flux when wsL*wsR > 0.

Arrays are interior-only [var, j, i] (var = rho, rho u_x, rho u_y, E); axis -1
is x (dimension 0) and axis -2 is y (dimension 1).
"""
import torch

KB = 1.380649e-23  # units.hpp: Boltzmann constant
MP = 1.672649e-27  # units.hpp: proton mass

LIMITERS = ("VanLeer", "Minmod")
SOLVERS = ("HLL", "HLLC")


def _nb(a, d, s):
    """Value of the neighbour at offset s along dimension d (periodic)."""
    return torch.roll(a, shifts=-s, dims=-1 - d)


def _div(a, c):
    """a / c for a Python float c as an element-wise division (torch turns a
    division by a scalar into a multiplication by its reciprocal, which
    rounds differently)."""
    return a / torch.full_like(a, c)


class _Sqrt(torch.autograd.Function):
    """Correctly rounded square root with its tangent t / (2 sqrt(x)).  On
    the CPU torch's vectorised sqrt is within about half an ulp but not
    always correctly rounded, so the value comes from numpy there; CUDA's
    FP64 sqrt is correctly rounded."""

    @staticmethod
    def forward(x):
        if x.device.type == "cpu":
            import numpy as np

            return torch.from_numpy(np.sqrt(x.detach().numpy()))
        return torch.sqrt(x)

    @staticmethod
    def setup_context(ctx, inputs, output):
        ctx.save_for_forward(output)

    @staticmethod
    def jvp(ctx, t):
        (s,) = ctx.saved_tensors
        return t / (2 * s)


class _Limited(torch.autograd.Function):
    """The reference's limited slope phi(R, L) (slope_limiters.hpp:38-66,
    value bit for bit) with the tangent of the branch it took, from the
    closed-form partials: van Leer 2RL/(R+L) has 2 (L/(R+L))^2 and
    2 (R/(R+L))^2, minmod takes R where R/L < 1 and L otherwise, and the
    slope is 0 (tangent 0) unless R*L > 0.  Differentiating the reference's
    ratio form instead overflows for tiny L ((R/L + 1)^2 = inf), which gives
    NaN tangents in nearly flat regions."""

    @staticmethod
    def forward(R, L, kind):
        cond = L * R > 0
        Ls = torch.where(cond, L, torch.ones_like(L))
        ratio = R / Ls
        if kind == 0:
            val = (1.0 / 2) * (R + L) * (4 * ratio) / ((ratio + 1) * (ratio + 1))
        else:
            # fmin(1, ratio) with ratio == 1 on the constant branch (slope L)
            val = 2 * torch.where(ratio < 1, ratio, torch.ones_like(ratio)) / (1 + ratio) * (L + R) / 2
        return torch.where(cond, val, torch.zeros_like(val))

    @staticmethod
    def setup_context(ctx, inputs, output):
        R, L, kind = inputs
        ctx.kind = kind
        ctx.save_for_forward(R, L)

    @staticmethod
    def jvp(ctx, Rt, Lt, _kind_t):
        R, L = ctx.saved_tensors
        cond = L * R > 0
        one = torch.ones_like(R)
        if ctx.kind == 0:
            s = torch.where(cond, R + L, one)
            a = L / s
            b = R / s
            t = 2 * a * a * Rt + 2 * b * b * Lt
        else:
            ratio = R / torch.where(cond, L, one)
            t = torch.where(ratio < 1, Rt, Lt)
        return torch.where(cond, t, torch.zeros_like(t))


def _min(a, b):
    return torch.where(a < b, a, b)


def _max(a, b):
    return torch.where(a > b, a, b)


class TangentStep:
    def __init__(self, gamma, dx, dy, dv, ds, limiter="VanLeer", riemann="HLLC", mmw=1.0):
        if limiter not in LIMITERS or riemann not in SOLVERS:
            raise ValueError(f"unsupported {limiter}/{riemann}")
        self.gamma = float(gamma)
        self.gm1 = float(gamma) - 1.0
        self.mmw = float(mmw)
        self.dl = (float(dx), float(dy))
        self.dv = float(dv)
        self.ds = (float(ds[0]), float(ds[1]))
        self.limiter = limiter
        self.riemann = riemann

    @classmethod
    def from_grid(cls, grid, gamma, limiter="VanLeer", riemann="HLLC", mmw=1.0):
        """From an oracle grid dict (dx0, dx1, dv, ds).  The restatement
        holds one dx, dv and ds per direction, so every cell must carry the
        same values bit for bit (power-of-two cell counts on [0, 1])."""
        import numpy as np

        vals = {}
        for key, a in (("dx0", grid["dx0"]), ("dx1", grid["dx1"]), ("dv", grid["dv"]), ("ds0", grid["ds"][0]),
                       ("ds1", grid["ds"][1])):
            u = np.unique(a)
            if u.size != 1:
                raise ValueError(f"{key} is not uniform bit for bit")
            vals[key] = float(u[0])
        return cls(gamma, vals["dx0"], vals["dx1"], vals["dv"], (vals["ds0"], vals["ds1"]), limiter, riemann, mmw)

    # ---- EOS (perfect_gas.hpp:46-78) ----------------------------------------
    def pres_from_evol(self, rho, evol):
        T = evol * self.mmw * MP * self.gm1 / (rho * KB)
        return _div(rho * KB * T, self.mmw * MP)

    def evol_from_pres(self, rho, P):
        T = P * self.mmw * MP / (rho * KB)
        return _div(rho * KB * T, self.mmw * MP * self.gm1)

    # ---- Euler algebra (euler_equations.hpp:41-134) -------------------------
    def to_prim(self, U):
        rho, m0, m1, E = U
        ek = (m0 * m0 + m1 * m1) / rho / 2
        return rho, m0 / rho, m1 / rho, self.pres_from_evol(rho, E - ek)

    def to_cons(self, W):
        rho, u0, u1, P = W
        ek = rho * (u0 * u0 + u1 * u1) / 2
        return rho, rho * u0, rho * u1, self.evol_from_pres(rho, P) + ek

    def flux_from_prim(self, W, l):
        rho, u0, u1, P = W
        ul = (u0, u1)[l]
        E = rho * (u0 * u0 + u1 * u1) / 2 + self.evol_from_pres(rho, P)
        f = [rho * ul, rho * ul * u0, rho * ul * u1, ul * (E + P)]
        f[1 + l] = f[1 + l] + P
        return f

    # ---- slopes (slope_limiters.hpp:38-66) ----------------------------------
    def slope(self, R, L):
        return _Limited.apply(R, L, 0 if self.limiter == "VanLeer" else 1)

    def faces(self, q, d):
        """(minus face, plus face) of q along d (limited_linear_reconstruction.hpp:46-64)."""
        dl = self.dl[d]
        h = (dl + dl) / 2
        s = self.slope(_div(_nb(q, d, 1) - q, h), _div(q - _nb(q, d, -1), h))
        return q - ((dl / 2) * s), q + ((dl / 2) * s)

    # ---- Riemann solvers (riemann_solver.hpp:31-134) ------------------------
    def riemann_flux(self, UL, UR, l):
        WL = self.to_prim(UL)
        WR = self.to_prim(UR)
        PL, PR = WL[3], WR[3]
        cL = _Sqrt.apply(self.gamma * PL / WL[0])
        cR = _Sqrt.apply(self.gamma * PR / WR[0])
        uL, uR = WL[1 + l], WR[1 + l]
        wsL = _min(uL - cL, uR - cR)
        wsR = _max(uL + cL, uR + cR)
        FL = self.flux_from_prim(WL, l)
        FR = self.flux_from_prim(WR, l)
        if self.riemann == "HLL":
            z = torch.zeros_like(wsL)
            sl = _min(wsL, z)
            sr = _max(wsR, z)
            return [((sr * FL[v]) - (sl * FR[v]) + (sl * sr * (UR[v] - UL[v]))) / (sr - sl) for v in range(4)]
        rcL = WL[0] * (wsL - uL)
        rcR = WR[0] * (wsR - uR)
        ustar = (PR - PL + (rcL * uL) - (rcR * uR)) / (rcL - rcR)
        pstar = 1.0 / 2 * (PL + PR + (rcL * (ustar - uL)) + (rcR * (ustar - uR)))
        left = ustar > 0
        S = torch.where(left, wsL, wsR)
        Uc = [torch.where(left, UL[v], UR[v]) for v in range(4)]
        Wc = [torch.where(left, WL[v], WR[v]) for v in range(4)]
        Fc = [torch.where(left, FL[v], FR[v]) for v in range(4)]
        un = Wc[1 + l]
        den = S - ustar
        rho_star = Uc[0] * (S - un) / den
        F = [None] * 4
        F[0] = Fc[0] + (S * (rho_star - Uc[0]))
        F[1] = rho_star * ustar * Wc[1]
        F[2] = rho_star * ustar * Wc[2]
        F[1 + l] = (rho_star * ustar * ustar) + pstar
        E_star = ((S - un) / den * Uc[3]) + ((ustar - un) / den * ((ustar * Uc[0] * (S - un)) + Wc[3]))
        F[3] = Fc[3] + (S * (E_star - Uc[3]))
        sup = wsL * wsR > 0
        return [torch.where(sup, Fc[v], F[v]) for v in range(4)]

    # ---- one step -------------------------------------------------------------
    def step(self, U, dt):
        """U [4, n1, n0] -> U after one step of size dt."""
        W = self.to_prim(U)
        # face primitives per dimension and side: rec[d][s] = (rho, u0, u1, P)
        rec = []
        for d in range(2):
            fm, fp = zip(*(self.faces(q, d) for q in W))
            rec.append((fm, fp))
        cons = [[list(self.to_cons(rec[d][s])) for s in range(2)] for d in range(2)]
        # Hancock predictor over half a step: every face of the cell gets the
        # increment of each direction in turn
        hdt = dt / 2
        dtodv = hdt / self.dv
        for idim in range(2):
            fL = self.flux_from_prim(rec[idim][0], idim)
            fR = self.flux_from_prim(rec[idim][1], idim)
            dsc = self.ds[idim]
            inc = [dtodv * ((fL[v] * dsc) - (fR[v] * dsc)) for v in range(4)]
            for ipos in range(2):
                for s in range(2):
                    for v in range(4):
                        cons[ipos][s][v] = cons[ipos][s][v] + inc[v]
        # Godunov update with one Riemann solve per face
        dtodv = dt / self.dv
        new = list(U)
        for idim in range(2):
            left = [_nb(cons[idim][1][v], idim, -1) for v in range(4)]
            FL = self.riemann_flux(left, cons[idim][0], idim)
            FR = [_nb(FL[v], idim, 1) for v in range(4)]
            dsc = self.ds[idim]
            for v in range(4):
                new[v] = new[v] + (dtodv * ((FL[v] * dsc) - (FR[v] * dsc)))
        return torch.stack(new)

    def run(self, U, dts):
        for dt in dts:
            U = self.step(U, float(dt))
        return U

    def jvp(self, U, V, dts):
        """(U^N, dU^N/dU0 . V) over the fixed dt sequence."""
        from torch.func import jvp

        return jvp(lambda x: self.run(x, dts), (U,), (V,))
