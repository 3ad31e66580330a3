"""ctypes binding of the C oracle (hcl_oracle.c) and of the reference's own
per-cell physics compiled into oracle/_ref/ (ref_cell_wrap.cpp).

TEST INFRASTRUCTURE ONLY: the checker, never the thing measured or shipped.
Arrays are numpy float64 in Kokkos LayoutLeft order, i.e. numpy arrays of
shape (n2, n1, n0) for a 3-D view (x0 fastest), (ncomp, n2, n1, n0) for a
4-D view, and so on; see hcl_oracle.h for the index maps.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

LIMITERS = {"Constant": 0, "VanLeer": 1, "Minmod": 2, "VanAlbada": 3}
RIEMANN = {"HLL": 0, "HLLC": 1, "Low Mach": 2}
BCS = {"NullGradient": 0, "Periodic": 1, "Reflexive": 2}
GEOMS = {"Cartesian": 0, "Spherical": 1}
GRAVITY = {"Uniform": 0, "Point_mass": 1, "Internal_mass": 2}
EOS = {"PerfectGas": 0, "RadGas": 1}

_dp = C.POINTER(C.c_double)


class _Ctx(C.Structure):
    _fields_ = [
        ("ndim", C.c_int),
        ("ng", C.c_int),
        ("nfx", C.c_int),
        ("nx", C.c_int * 3),
        ("n", C.c_int * 3),
        ("geom", C.c_int),
        ("gamma", C.c_double),
        ("gamma_m1", C.c_double),
        ("mmw", C.c_double),
        ("limiter", C.c_int),
        ("riemann", C.c_int),
        ("bc", C.c_int * 6),
        ("bc_order", C.c_int * 6),
        ("gravity", C.c_int),
        ("g", C.c_double * 3),
        ("central_mass", C.c_double),
        ("x", _dp * 3),
        ("dx", _dp * 3),
        ("xc", _dp * 3),
        ("ds", _dp),
        ("dv", _dp),
        ("g_r", _dp),
        ("eos", C.c_int),
    ]


class _RunParams(C.Structure):
    _fields_ = [
        ("cfl", C.c_double),
        ("t_ini", C.c_double),
        ("t_end", C.c_double),
        ("max_iter", C.c_int),
        ("iter_frequency", C.c_int),
        ("time_frequency", C.c_double),
        ("time_first_output", C.c_double),
        ("fixed_dt", C.c_int),
        ("dts", _dp),
        ("pressure_fix", C.c_int),
        ("eps_pf", C.c_double),
    ]


class _RunResult(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("iter", C.c_int),
        ("status", C.c_int),
        ("initial_mass", C.c_double),
        ("final_mass", C.c_double),
    ]


def oracle_lib_path() -> Path:
    return HERE / "liboracle.so"


def build_oracle(ref: bool = True) -> None:
    """Builds liboracle.so and, with ref, oracle/_ref (the recipe skips the
    reference build when the reference sources are absent)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


def reference_root() -> Path | None:
    """The reference checkout the oracle recipe reads (HCL_REF_SRC or the
    recipe's default), or None when it is absent."""
    out = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref-root"], check=True, capture_output=True,
                         text=True).stdout.strip()
    root = Path(out) if out else None
    return root if root is not None and (root / "src").is_dir() else None


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = oracle_lib_path()
        if not path.exists():
            build_oracle(ref=False)
        lib = C.CDLL(str(path))
        vp = C.c_void_p
        lib.or_ctx_init.argtypes = [C.POINTER(_Ctx), C.c_int, C.c_int * 3, C.c_int, C.c_int, C.c_int, C.c_double,
                                    C.c_double, C.c_int, C.c_int, C.c_int * 6, C.c_int, C.c_double * 3, C.c_double,
                                    C.c_double * 3, C.c_double * 3]
        lib.or_ctx_init_nodes.argtypes = [C.POINTER(_Ctx), C.c_int, C.c_int * 3, C.c_int, C.c_int, C.c_int,
                                          C.c_double, C.c_double, C.c_int, C.c_int, C.c_int * 6, C.c_int,
                                          C.c_double * 3, C.c_double, vp, vp, vp]
        lib.or_ctx_free.argtypes = [C.POINTER(_Ctx)]
        for name in ("or_to_prim", "or_to_cons"):
            getattr(lib, name).argtypes = [C.POINTER(_Ctx), vp, vp]
        for name in ("or_flux_from_prim", "or_flux_from_cons"):
            getattr(lib, name).argtypes = [C.POINTER(_Ctx), vp, C.c_int, vp]
        lib.or_ek_prim.argtypes = [C.POINTER(_Ctx), vp]
        lib.or_ek_prim.restype = C.c_double
        lib.or_ek_cons.argtypes = [C.POINTER(_Ctx), vp]
        lib.or_ek_cons.restype = C.c_double
        lib.or_slope.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.or_slope.restype = C.c_double
        lib.or_riemann.argtypes = [C.POINTER(_Ctx), C.c_int, vp, vp, C.c_int, vp]
        for name in ("or_speed_of_sound", "or_evol_from_pres", "or_pres_from_evol"):
            getattr(lib, name).argtypes = [C.POINTER(_Ctx), C.c_double, C.c_double]
            getattr(lib, name).restype = C.c_double
        lib.or_eos_valid.argtypes = [C.c_double, C.c_double]
        lib.or_eos_valid.restype = C.c_int
        lib.or_conv_prim_to_cons.argtypes = [C.POINTER(_Ctx), C.c_int, vp, vp, vp, vp, vp]
        lib.or_conv_cons_to_prim.argtypes = [C.POINTER(_Ctx), C.c_int, vp, vp, vp, vp, vp]
        lib.or_face_reconstruction.argtypes = [C.POINTER(_Ctx), C.c_int, vp, vp, C.c_long]
        lib.or_hydro_reconstruction.argtypes = [C.POINTER(_Ctx), C.c_int, C.c_double] + [vp] * 10
        lib.or_godunov.argtypes = [C.POINTER(_Ctx), C.c_int, C.c_double] + [vp] * 12
        lib.or_boundaries.argtypes = [C.POINTER(_Ctx), vp, vp, vp, vp]
        lib.or_pressure_fix.argtypes = [C.POINTER(_Ctx), C.c_double, C.c_double] + [vp] * 9
        lib.or_internal_mass_gravity.argtypes = [C.POINTER(_Ctx), vp]
        lib.or_set_eos.argtypes = [C.POINTER(_Ctx), C.c_int]
        lib.or_temperature.argtypes = [C.POINTER(_Ctx), C.c_double, C.c_double]
        lib.or_temperature.restype = C.c_double
        lib.or_time_step.argtypes = [C.POINTER(_Ctx), C.c_int, vp, vp, vp]
        lib.or_time_step.restype = C.c_double
        lib.or_min_internal_energy.argtypes = [C.POINTER(_Ctx), vp, vp, vp]
        lib.or_min_internal_energy.restype = C.c_double
        lib.or_integrate.argtypes = [C.POINTER(_Ctx), vp]
        lib.or_integrate.restype = C.c_double
        lib.or_run.argtypes = [C.POINTER(_Ctx), vp, vp, vp, vp, C.POINTER(_RunParams), C.POINTER(_RunResult), vp]
        lib.or_run.restype = C.c_int
        lib.or_init_from_prim.argtypes = [C.POINTER(_Ctx)] + [vp] * 7
        lib.or_set_threads.argtypes = [C.c_int]
        lib.or_get_threads.restype = C.c_int
        _LIB = lib
    return _LIB


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous float64"
    return a.ctypes.data_as(C.c_void_p)


def _id(mapping, key):
    if isinstance(key, (int, np.integer)):
        return int(key)
    return mapping[key]


class Oracle:
    """One grid + physics configuration of the CPU oracle."""

    def __init__(self, ndim, nx, *, ng=2, nfx=0, geom="Cartesian", gamma=1.4, mmw=1.0, limiter="VanLeer",
                 riemann="HLLC", bc=("Periodic",) * 6, gravity="Uniform", g=(0.0, 0.0, 0.0), central_mass=1.0,
                 xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), nodes=None, eos="PerfectGas"):
        self.lib = _lib()
        self.ctx = _Ctx()
        nx3 = (C.c_int * 3)(*[int(v) for v in (list(nx) + [1, 1, 1])[:3]])
        bc6 = (C.c_int * 6)(*[_id(BCS, b) for b in (list(bc) + ["Periodic"] * 6)[:6]])
        g3 = (C.c_double * 3)(*g)
        args = (C.byref(self.ctx), int(ndim), nx3, int(ng), int(nfx), _id(GEOMS, geom), float(gamma), float(mmw),
                _id(LIMITERS, limiter), _id(RIEMANN, riemann), bc6, _id(GRAVITY, gravity), g3, float(central_mass))
        if nodes is None:
            rc = self.lib.or_ctx_init(*args, (C.c_double * 3)(*xmin), (C.c_double * 3)(*xmax))
        else:
            self._nodes = [np.ascontiguousarray(x, dtype=np.float64) for x in nodes]
            rc = self.lib.or_ctx_init_nodes(*args, *[_p(x) for x in self._nodes])
        if rc != 0:
            raise ValueError("Invalid gamma" if rc == -1 else "Invalid mmw")
        self.lib.or_set_eos(C.byref(self.ctx), _id(EOS, eos))
        self.ndim = int(ndim)
        self.nfx = int(nfx)
        self.n = tuple(self.ctx.n)
        self.nx = tuple(self.ctx.nx)
        self.ncells = self.n[0] * self.n[1] * self.n[2]

    def __del__(self):
        try:
            self.lib.or_ctx_free(C.byref(self.ctx))
        except Exception:
            pass

    # ---- helpers -------------------------------------------------------
    @property
    def shape3(self):
        return (self.n[2], self.n[1], self.n[0])

    def zeros(self, ncomp=None):
        if ncomp is None:
            return np.zeros(self.shape3)
        return np.zeros((ncomp,) + self.shape3)

    def grid(self):
        """x nodes, dx, centres and ds/dv as numpy arrays (copies)."""
        out = {}
        for d in range(3):
            n = self.n[d]
            out[f"x{d}"] = np.ctypeslib.as_array(self.ctx.x[d], shape=(n + 1,)).copy()
            out[f"dx{d}"] = np.ctypeslib.as_array(self.ctx.dx[d], shape=(n,)).copy()
            out[f"x{d}c"] = np.ctypeslib.as_array(self.ctx.xc[d], shape=(n,)).copy()
        out["ds"] = np.ctypeslib.as_array(self.ctx.ds, shape=(3,) + self.shape3).copy()
        out["dv"] = np.ctypeslib.as_array(self.ctx.dv, shape=self.shape3).copy()
        return out

    # ---- per cell ------------------------------------------------------
    def to_prim(self, cons):
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        out = np.zeros(self.ndim + 2)
        self.lib.or_to_prim(C.byref(self.ctx), _p(cons), _p(out))
        return out

    def to_cons(self, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros(self.ndim + 2)
        self.lib.or_to_cons(C.byref(self.ctx), _p(prim), _p(out))
        return out

    def flux_from_prim(self, prim, locdim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros(self.ndim + 2)
        self.lib.or_flux_from_prim(C.byref(self.ctx), _p(prim), int(locdim), _p(out))
        return out

    def flux_from_cons(self, cons, locdim):
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        out = np.zeros(self.ndim + 2)
        self.lib.or_flux_from_cons(C.byref(self.ctx), _p(cons), int(locdim), _p(out))
        return out

    def ek_prim(self, prim):
        return self.lib.or_ek_prim(C.byref(self.ctx), _p(np.ascontiguousarray(prim, dtype=np.float64)))

    def ek_cons(self, cons):
        return self.lib.or_ek_cons(C.byref(self.ctx), _p(np.ascontiguousarray(cons, dtype=np.float64)))

    def riemann(self, solver, consL, consR, locdim):
        L = np.ascontiguousarray(consL, dtype=np.float64)
        R = np.ascontiguousarray(consR, dtype=np.float64)
        out = np.zeros(self.ndim + 2)
        self.lib.or_riemann(C.byref(self.ctx), _id(RIEMANN, solver), _p(L), _p(R), int(locdim), _p(out))
        return out

    def slope(self, limiter, diffR, diffL):
        return self.lib.or_slope(_id(LIMITERS, limiter), float(diffR), float(diffL))

    def speed_of_sound(self, rho, P):
        return self.lib.or_speed_of_sound(C.byref(self.ctx), rho, P)

    def evol_from_pres(self, rho, P):
        return self.lib.or_evol_from_pres(C.byref(self.ctx), rho, P)

    def pres_from_evol(self, rho, e):
        return self.lib.or_pres_from_evol(C.byref(self.ctx), rho, e)

    def eos_valid(self, rho, P):
        return bool(self.lib.or_eos_valid(rho, P))

    def temperature(self, rho, P):
        return self.lib.or_temperature(C.byref(self.ctx), rho, P)

    # ---- arrays --------------------------------------------------------
    def conv_prim_to_cons(self, ng_eff, rho, u, P):
        rhou = self.zeros(self.ndim)
        E = self.zeros()
        self.lib.or_conv_prim_to_cons(C.byref(self.ctx), ng_eff, _p(rho), _p(u), _p(P), _p(rhou), _p(E))
        return rhou, E

    def conv_cons_to_prim(self, ng_eff, rho, rhou, E):
        u = self.zeros(self.ndim)
        P = self.zeros()
        self.lib.or_conv_cons_to_prim(C.byref(self.ctx), ng_eff, _p(rho), _p(rhou), _p(E), _p(u), _p(P))
        return u, P

    def face_reconstruction(self, ng_eff, var):
        """Returns var_rec with numpy shape (ndim, 2, n2, n1, n0)."""
        out = np.zeros((self.ndim, 2) + self.shape3)
        self.lib.or_face_reconstruction(C.byref(self.ctx), ng_eff, _p(var), _p(out), 2 * self.ncells)
        return out

    def hydro_reconstruction(self, ng_eff, dt, rho, u, P, fx=None):
        nd, nfx = self.ndim, self.nfx
        rho_rec = np.zeros((nd, 2) + self.shape3)
        rhou_rec = np.zeros((nd, nd, 2) + self.shape3)
        E_rec = np.zeros((nd, 2) + self.shape3)
        fx_rec = np.zeros((max(nfx, 1), nd, 2) + self.shape3)
        u_rec = np.zeros((nd, nd, 2) + self.shape3)
        P_rec = np.zeros((nd, 2) + self.shape3)
        if fx is None:
            fx = self.zeros(max(nfx, 1))
        self.lib.or_hydro_reconstruction(C.byref(self.ctx), ng_eff, dt, _p(rho), _p(u), _p(P), _p(fx), _p(rho_rec),
                                         _p(rhou_rec), _p(E_rec), _p(fx_rec), _p(u_rec), _p(P_rec))
        return rho_rec, rhou_rec, E_rec, fx_rec

    def godunov(self, ng_eff, dt, rho, rhou, E, rho_rec, rhou_rec, E_rec, fx=None, fx_rec=None):
        nfx = max(self.nfx, 1)
        if fx is None:
            fx = self.zeros(nfx)
        if fx_rec is None:
            fx_rec = np.zeros((nfx, self.ndim, 2) + self.shape3)
        rho_new = self.zeros()
        rhou_new = self.zeros(self.ndim)
        E_new = self.zeros()
        fx_new = self.zeros(nfx)
        self.lib.or_godunov(C.byref(self.ctx), ng_eff, dt, _p(rho), _p(rhou), _p(E), _p(fx), _p(rho_rec),
                            _p(rhou_rec), _p(E_rec), _p(fx_rec), _p(rho_new), _p(rhou_new), _p(E_new), _p(fx_new))
        return rho_new, rhou_new, E_new, fx_new

    def pressure_fix(self, dt, eps, rho, rhou, E, rho_rec, rhou_rec, E_rec, rho_new, rhou_new, E_new):
        """Updates E_new in place (pressure_fix.hpp:19-172)."""
        self.lib.or_pressure_fix(C.byref(self.ctx), dt, eps, _p(rho), _p(rhou), _p(E), _p(rho_rec), _p(rhou_rec),
                                 _p(E_rec), _p(rho_new), _p(rhou_new), _p(E_new))
        return E_new

    def internal_mass_gravity(self, rho):
        """Recomputes the radial gravity table from rho (gravity.cpp:59-128) and
        returns a copy of it (g along dimension 0 per x0 index, ghosts included)."""
        self.lib.or_internal_mass_gravity(C.byref(self.ctx), _p(rho))
        return self.gravity_table()

    def gravity_table(self):
        """Copy of the radial gravity table g(i) (point-mass and internal-mass gravity)."""
        n0 = self.ctx.n[0]
        return np.ctypeslib.as_array(self.ctx.g_r, shape=(n0,)).copy()

    def boundaries(self, rho, rhou, E, fx=None):
        if fx is None:
            fx = self.zeros(max(self.nfx, 1))
        self.lib.or_boundaries(C.byref(self.ctx), _p(rho), _p(rhou), _p(E), _p(fx))

    def time_step(self, ng_eff, rho, u, P):
        return self.lib.or_time_step(C.byref(self.ctx), ng_eff, _p(rho), _p(u), _p(P))

    def min_internal_energy(self, rho, rhou, E):
        return self.lib.or_min_internal_energy(C.byref(self.ctx), _p(rho), _p(rhou), _p(E))

    def integrate(self, var):
        return self.lib.or_integrate(C.byref(self.ctx), _p(var))

    def init_from_prim(self, rho_prim, u, P):
        rho = self.zeros()
        rhou = self.zeros(self.ndim)
        E = self.zeros()
        fx = self.zeros(max(self.nfx, 1))
        self.lib.or_init_from_prim(C.byref(self.ctx), _p(np.ascontiguousarray(rho_prim)), _p(np.ascontiguousarray(u)),
                                   _p(np.ascontiguousarray(P)), _p(rho), _p(rhou), _p(E), _p(fx))
        return rho, rhou, E, fx

    def run(self, rho, rhou, E, fx=None, *, cfl=0.4, t_ini=0.0, t_end=1e30, max_iter=10000, iter_frequency=0,
            time_frequency=0.0, time_first_output=None, dts=None, record_dts=False, pressure_fix=False,
            eps_pf=1e-6):
        """Runs main.cpp's time loop in place.  Returns (t, iter, status, dts)."""
        if fx is None:
            fx = self.zeros(max(self.nfx, 1))
        p = _RunParams()
        p.cfl = cfl
        p.t_ini = t_ini
        p.t_end = t_end
        p.max_iter = max_iter
        p.iter_frequency = iter_frequency
        p.time_frequency = time_frequency
        p.time_first_output = t_ini + time_frequency if time_first_output is None else time_first_output
        p.pressure_fix = 1 if pressure_fix else 0
        p.eps_pf = eps_pf
        if dts is not None:
            dts_arr = np.ascontiguousarray(dts, dtype=np.float64)
            p.fixed_dt = 1
            p.dts = dts_arr.ctypes.data_as(_dp)
        r = _RunResult()
        rec = np.zeros(max_iter) if record_dts else None
        self.lib.or_run(C.byref(self.ctx), _p(rho), _p(rhou), _p(E), _p(fx), C.byref(p), C.byref(r), _p(rec))
        out_dts = rec[: r.iter] if record_dts else None
        return r.t, r.iter, r.status, out_dts

    @staticmethod
    def set_threads(n):
        _lib().or_set_threads(int(n))

    @staticmethod
    def get_threads():
        return _lib().or_get_threads()


class RefCell:
    """The reference's own per-cell physics (oracle/_ref), for pinning the oracle."""

    def __init__(self, ndim: int):
        path = HERE / "_ref" / f"libref_cell_{ndim}d.so"
        if not path.exists():
            raise FileNotFoundError(str(path))
        lib = C.CDLL(str(path))
        vp = C.c_void_p
        d = C.c_double
        lib.ref_ndim.restype = C.c_int
        lib.ref_perfect_gas_check.argtypes = [d, d]
        lib.ref_perfect_gas_check.restype = C.c_int
        lib.ref_eos_valid.argtypes = [d, d]
        lib.ref_eos_valid.restype = C.c_int
        for name in ("ref_evol_from_pres", "ref_pres_from_evol", "ref_speed_of_sound", "ref_rad_evol_from_pres",
                     "ref_rad_pres_from_evol", "ref_rad_speed_of_sound", "ref_rad_temp_from_pres"):
            getattr(lib, name).argtypes = [d, d, d, d]
            getattr(lib, name).restype = d
        lib.ref_rad_gas_check.argtypes = [d, d]
        lib.ref_rad_gas_check.restype = C.c_int
        lib.ref_rad_riemann.argtypes = [C.c_int, d, d, vp, vp, C.c_int, vp]
        lib.ref_to_prim.argtypes = [d, d, vp, vp]
        lib.ref_to_cons.argtypes = [d, d, vp, vp]
        lib.ref_flux_from_prim.argtypes = [d, d, vp, C.c_int, vp]
        lib.ref_flux_from_cons.argtypes = [d, d, vp, C.c_int, vp]
        lib.ref_ek_prim.argtypes = [vp]
        lib.ref_ek_prim.restype = d
        lib.ref_ek_cons.argtypes = [vp]
        lib.ref_ek_cons.restype = d
        lib.ref_riemann.argtypes = [C.c_int, d, d, vp, vp, C.c_int, vp]
        lib.ref_slope.argtypes = [C.c_int, d, d]
        lib.ref_slope.restype = d
        lib.ref_source_grad_pres.argtypes = [d] * 5
        lib.ref_source_grad_pres.restype = d
        lib.ref_source_grad_u_r.argtypes = [d] * 7
        lib.ref_source_grad_u_r.restype = d
        lib.ref_source_grad_u_idir_r.argtypes = [d] * 11
        lib.ref_source_grad_u_idir_r.restype = d
        lib.ref_source_grad_u_th.argtypes = [d] * 9
        lib.ref_source_grad_u_th.restype = d
        lib.ref_source_grad_u_phi.argtypes = [d] * 11
        lib.ref_source_grad_u_phi.restype = d
        self.lib = lib
        self.ndim = lib.ref_ndim()
        assert self.ndim == ndim

    def _vec(self):
        return np.zeros(self.ndim + 2)

    def to_prim(self, gamma, mmw, cons):
        out = self._vec()
        self.lib.ref_to_prim(gamma, mmw, _p(np.ascontiguousarray(cons, dtype=np.float64)), _p(out))
        return out

    def to_cons(self, gamma, mmw, prim):
        out = self._vec()
        self.lib.ref_to_cons(gamma, mmw, _p(np.ascontiguousarray(prim, dtype=np.float64)), _p(out))
        return out

    def flux_from_prim(self, gamma, mmw, prim, locdim):
        out = self._vec()
        self.lib.ref_flux_from_prim(gamma, mmw, _p(np.ascontiguousarray(prim, dtype=np.float64)), locdim, _p(out))
        return out

    def flux_from_cons(self, gamma, mmw, cons, locdim):
        out = self._vec()
        self.lib.ref_flux_from_cons(gamma, mmw, _p(np.ascontiguousarray(cons, dtype=np.float64)), locdim, _p(out))
        return out

    def riemann(self, solver, gamma, mmw, consL, consR, locdim, eos="PerfectGas"):
        out = self._vec()
        fn = self.lib.ref_rad_riemann if eos == "RadGas" else self.lib.ref_riemann
        fn(_id(RIEMANN, solver), gamma, mmw, _p(np.ascontiguousarray(consL, dtype=np.float64)),
           _p(np.ascontiguousarray(consR, dtype=np.float64)), locdim, _p(out))
        return out

    def slope(self, limiter, diffR, diffL):
        return self.lib.ref_slope(_id(LIMITERS, limiter), float(diffR), float(diffL))


# ---- the reference's own array code (oracle/_ref/libref_step_*.so) ----------------

class _RsConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int * 3),
        ("ng", C.c_int),
        ("nfx", C.c_int),
        ("xmin", C.c_double * 3),
        ("xmax", C.c_double * 3),
        ("gamma", C.c_double),
        ("mmw", C.c_double),
        ("limiter", C.c_char_p),
        ("riemann", C.c_char_p),
        ("bc", C.c_char_p * 6),
        ("bc_priority", C.c_char_p),
        ("gravity", C.c_int),
        ("g", C.c_double * 3),
        ("central_mass", C.c_double),
    ]


def ref_step_path(ndim: int, geom: str = "Cartesian") -> Path:
    tag = "sph" if geom == "Spherical" else "cart"
    return HERE / "_ref" / f"libref_step_{int(ndim)}d_{tag}.so"


_RS_LIBS: dict = {}


def _rs_lib(ndim, geom):
    key = (int(ndim), geom)
    if key in _RS_LIBS:
        return _RS_LIBS[key]
    path = ref_step_path(ndim, geom)
    if not path.exists():
        raise FileNotFoundError(f"{path} not built (make -C oracle ref-step where the reference sources are)")
    L = C.CDLL(str(path))
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.rs_create.argtypes = [C.POINTER(_RsConfig)]
    L.rs_create.restype = vp
    L.rs_destroy.argtypes = [vp]
    L.rs_set_threads.argtypes = [i]
    L.rs_get_threads.restype = i
    L.rs_grid.argtypes = [vp, vp, vp, vp, vp]
    L.rs_conv_prim_to_cons.argtypes = [vp, i, vp, vp, vp, vp, vp]
    L.rs_conv_cons_to_prim.argtypes = [vp, i, vp, vp, vp, vp, vp]
    L.rs_hydro_reconstruction.argtypes = [vp, i, d] + [vp] * 8
    L.rs_godunov.argtypes = [vp, i, d] + [vp] * 12
    L.rs_boundaries.argtypes = [vp, vp, vp, vp, vp]
    L.rs_time_step.argtypes = [vp, i, vp, vp, vp]
    L.rs_time_step.restype = d
    L.rs_min_internal_energy.argtypes = [vp, vp, vp, vp]
    L.rs_min_internal_energy.restype = d
    L.rs_run.argtypes = [vp, vp, vp, vp, vp, d, d, i, vp, C.POINTER(i), vp]
    L.rs_run.restype = i
    _RS_LIBS[key] = L
    return L


class RefStep:
    """The reference's own classes for one domain (MUSCLHancockHydroReconstruction,
    the Godunov scheme of its factory, DistributedBoundaryCondition on one rank,
    time_step, the conversions), run on the host through the Kokkos/MPI
    stand-ins of oracle/ref_array.  Same keyword arguments and array shapes as
    Oracle (uniform and point-mass gravity, perfect gas)."""

    def __init__(self, ndim, nx, *, ng=2, nfx=0, geom="Cartesian", gamma=1.4, mmw=1.0, limiter="VanLeer",
                 riemann="HLLC", bc=("Periodic",) * 6, gravity="Uniform", g=(0.0, 0.0, 0.0), central_mass=1.0,
                 xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), bc_priority=""):
        if gravity not in ("Uniform", "Point_mass"):
            raise ValueError("RefStep wraps the uniform and point-mass gravities")
        self.lib = _rs_lib(ndim, geom)
        cfg = _RsConfig()
        nx3 = (list(nx) + [1, 1, 1])[:3]
        for d in range(3):
            cfg.nx[d] = int(nx3[d])
            cfg.xmin[d] = float(xmin[d])
            cfg.xmax[d] = float(xmax[d])
            cfg.g[d] = float(g[d])
        cfg.ng, cfg.nfx, cfg.gamma, cfg.mmw = int(ng), int(nfx), float(gamma), float(mmw)
        self._keep = [s.encode() for s in [limiter, riemann, bc_priority] + (list(bc) + ["Periodic"] * 6)[:6]]
        cfg.limiter, cfg.riemann, cfg.bc_priority = self._keep[0], self._keep[1], self._keep[2]
        for f in range(6):
            cfg.bc[f] = self._keep[3 + f]
        cfg.gravity = 1 if gravity == "Point_mass" else 0
        cfg.central_mass = float(central_mass)
        self.h = self.lib.rs_create(C.byref(cfg))
        if not self.h:
            raise ValueError("the reference rejected this configuration (see stderr)")
        self.ndim, self.nfx = int(ndim), int(nfx)
        self.n = tuple(int(v) + (2 * ng if k < ndim else 0) for k, v in enumerate(nx3))
        self.ncells = self.n[0] * self.n[1] * self.n[2]

    def __del__(self):
        try:
            self.lib.rs_destroy(self.h)
        except Exception:
            pass

    @property
    def shape3(self):
        return (self.n[2], self.n[1], self.n[0])

    def zeros(self, ncomp=None):
        return np.zeros(self.shape3) if ncomp is None else np.zeros((ncomp,) + self.shape3)

    @staticmethod
    def set_threads(ndim, geom, n):
        _rs_lib(ndim, geom).rs_set_threads(int(n))

    def threads(self):
        return int(self.lib.rs_get_threads())

    def grid(self):
        dx = np.zeros(sum(self.n))
        xc = np.zeros(sum(self.n))
        ds = np.zeros((3,) + self.shape3)
        dv = np.zeros(self.shape3)
        self.lib.rs_grid(self.h, _p(dx), _p(xc), _p(ds), _p(dv))
        out = {"ds": ds, "dv": dv}
        off = 0
        for d in range(3):
            out[f"dx{d}"] = dx[off:off + self.n[d]]
            out[f"x{d}c"] = xc[off:off + self.n[d]]
            off += self.n[d]
        return out

    def conv_prim_to_cons(self, ng_eff, rho, u, P):
        rhou, E = self.zeros(self.ndim), self.zeros()
        self.lib.rs_conv_prim_to_cons(self.h, ng_eff, _p(rho), _p(u), _p(P), _p(rhou), _p(E))
        return rhou, E

    def conv_cons_to_prim(self, ng_eff, rho, rhou, E):
        u, P = self.zeros(self.ndim), self.zeros()
        self.lib.rs_conv_cons_to_prim(self.h, ng_eff, _p(rho), _p(rhou), _p(E), _p(u), _p(P))
        return u, P

    def hydro_reconstruction(self, ng_eff, dt, rho, u, P, fx=None):
        nd, nfx = self.ndim, self.nfx
        rho_rec = np.zeros((nd, 2) + self.shape3)
        rhou_rec = np.zeros((nd, nd, 2) + self.shape3)
        E_rec = np.zeros((nd, 2) + self.shape3)
        fx_rec = np.zeros((max(nfx, 1), nd, 2) + self.shape3)
        if fx is None:
            fx = self.zeros(max(nfx, 1))
        self.lib.rs_hydro_reconstruction(self.h, ng_eff, dt, _p(rho), _p(u), _p(P), _p(fx), _p(rho_rec), _p(rhou_rec),
                                         _p(E_rec), _p(fx_rec))
        return rho_rec, rhou_rec, E_rec, fx_rec

    def godunov(self, ng_eff, dt, rho, rhou, E, rho_rec, rhou_rec, E_rec, fx=None, fx_rec=None):
        nfx = max(self.nfx, 1)
        if fx is None:
            fx = self.zeros(nfx)
        if fx_rec is None:
            fx_rec = np.zeros((nfx, self.ndim, 2) + self.shape3)
        rho_new, rhou_new, E_new, fx_new = self.zeros(), self.zeros(self.ndim), self.zeros(), self.zeros(nfx)
        self.lib.rs_godunov(self.h, ng_eff, dt, _p(rho), _p(rhou), _p(E), _p(fx), _p(rho_rec), _p(rhou_rec),
                            _p(E_rec), _p(fx_rec), _p(rho_new), _p(rhou_new), _p(E_new), _p(fx_new))
        return rho_new, rhou_new, E_new, fx_new

    def boundaries(self, rho, rhou, E, fx=None):
        if fx is None:
            fx = self.zeros(max(self.nfx, 1))
        self.lib.rs_boundaries(self.h, _p(rho), _p(rhou), _p(E), _p(fx))

    def time_step(self, ng_eff, rho, u, P):
        return self.lib.rs_time_step(self.h, ng_eff, _p(rho), _p(u), _p(P))

    def min_internal_energy(self, rho, rhou, E):
        return self.lib.rs_min_internal_energy(self.h, _p(rho), _p(rhou), _p(E))

    def run(self, rho, rhou, E, fx=None, *, cfl=0.4, t_end=1e30, max_iter=10000, record_dts=False):
        """The reference's time loop (main.cpp:354-531 without outputs), in
        place.  Returns (t, iter, status, dts)."""
        if fx is None:
            fx = self.zeros(max(self.nfx, 1))
        t = C.c_double(0.0)
        it = C.c_int(0)
        rec = np.zeros(max_iter) if record_dts else None
        st = self.lib.rs_run(self.h, _p(rho), _p(rhou), _p(E), _p(fx), float(cfl), float(t_end), int(max_iter),
                             C.byref(t), C.byref(it), _p(rec))
        return t.value, it.value, st, (rec[: it.value] if record_dts else None)
