"""heraclespp_b200 -- B200-native MUSCL-Hancock step of HERACLES++.

Python view of the C ABI (include/heracles_b200.h).  ``Domain`` wraps one
handle: one grid on one GPU with the physics plugins chosen by the same
keys as the reference's factories (``Minmod``, ``HLLC``, ``NullGradient``,
...).  Host arrays are numpy float64 arrays in the reference's LayoutLeft
order, i.e. numpy shape (n2, n1, n0) for rho and (ndim, n2, n1, n0) for rhou.
Stage methods take torch CUDA tensors laid out the same way.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import (BCS, EOS, GEOMS, GRAVITY, LIMITERS, PRECISION, RIEMANN, Config, DomainError, HclError,
                      RunParams, RunResult, check, lib)

__all__ = ["Domain", "Ensemble", "make_config", "HclError", "DomainError", "lib", "kernel_launch_count"]


def kernel_launch_count() -> int:
    return int(lib().hcl_kernel_launch_count())


def _key(mapping, v, what):
    if isinstance(v, (int, np.integer)):
        return int(v)
    try:
        return mapping[v]
    except KeyError:
        raise HclError(1, f"Unknown {what}: {v}.") from None


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        assert t.dtype == np.float64 and t.flags["C_CONTIGUOUS"]
        return t.ctypes.data_as(C.c_void_p)
    return C.c_void_p(t.data_ptr())


def make_config(ndim, nx, *, nghost=2, nfx=0, geometry="Cartesian", gamma=5.0 / 3.0, mmw=1.0, limiter="VanLeer",
                riemann="HLL", bc=("Periodic",) * 6, gravity="Uniform", g=(0.0, 0.0, 0.0), central_mass=1.0,
                xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), nodes=None, precision="fp64", device=0,
                pressure_fix=False, eps_pf=1e-6, eos="PerfectGas"):
    """hcl_config from the reference's plugin keys; returns (config, node arrays kept alive)."""
    L = lib()
    cfg = Config()
    L.hcl_config_default(C.byref(cfg))
    cfg.ndim = int(ndim)
    nx = list(nx) + [1, 1, 1]
    for d in range(3):
        cfg.nx[d] = int(nx[d]) if d < ndim else 1
        cfg.g[d] = float(g[d])
        cfg.xmin[d] = float(xmin[d])
        cfg.xmax[d] = float(xmax[d])
    cfg.nghost = int(nghost)
    cfg.nfx = int(nfx)
    cfg.geometry = _key(GEOMS, geometry, "geometry")
    cfg.gamma = float(gamma)
    cfg.mmw = float(mmw)
    cfg.limiter = _key(LIMITERS, limiter, "face reconstruction algorithm")
    cfg.riemann = _key(RIEMANN, riemann, "riemann solver")
    bcs = list(bc) + ["Periodic"] * 6
    for f in range(6):
        cfg.bc[f] = _key(BCS, bcs[f], "boundary condition")
    cfg.gravity = _key(GRAVITY, gravity, "gravity")
    cfg.central_mass = float(central_mass)
    cfg.precision = _key(PRECISION, precision, "precision")
    cfg.device = int(device)
    cfg.pressure_fix = 1 if pressure_fix else 0
    cfg.eps_pf = float(eps_pf)
    cfg.eos = _key(EOS, eos, "eos")
    _nodes = None
    if nodes is not None:
        _nodes = [np.ascontiguousarray(x, dtype=np.float64) for x in nodes]
        for d in range(3):
            cfg.nodes[d] = _nodes[d].ctypes.data
    return cfg, _nodes


class Domain:
    """One domain on one GPU (hcl_create)."""

    def __init__(self, ndim, nx, *, nghost=2, nfx=0, geometry="Cartesian", gamma=5.0 / 3.0, mmw=1.0,
                 limiter="VanLeer", riemann="HLL", bc=("Periodic",) * 6, gravity="Uniform", g=(0.0, 0.0, 0.0),
                 central_mass=1.0, xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), nodes=None, precision="fp64",
                 device=0, pressure_fix=False, eps_pf=1e-6, eos="PerfectGas", stage_loop=False):
        cfg, self._nodes = make_config(ndim, nx, nghost=nghost, nfx=nfx, geometry=geometry, gamma=gamma, mmw=mmw,
                                       limiter=limiter, riemann=riemann, bc=bc, gravity=gravity, g=g,
                                       central_mass=central_mass, xmin=xmin, xmax=xmax, nodes=nodes,
                                       precision=precision, device=device, pressure_fix=pressure_fix,
                                       eps_pf=eps_pf, eos=eos)
        h = C.c_void_p()
        check(lib().hcl_create(C.byref(cfg), C.byref(h)))
        self._owned = True
        self._attach(h, cfg)
        if stage_loop:
            check(lib().hcl_set_stage_loop(h, 1))

    @classmethod
    def _view(cls, h, cfg):
        """Domain over a handle owned by someone else (an Ensemble)."""
        self = cls.__new__(cls)
        self._nodes = None
        self._owned = False
        self._attach(h, cfg)
        return self

    def _attach(self, h, cfg):
        self.cfg = cfg
        self.h = h
        self.ndim = int(cfg.ndim)
        self.nfx = int(cfg.nfx)
        n = (C.c_int * 3)()
        nc = C.c_int64()
        check(lib().hcl_get_extents(h, n, C.byref(nc)))
        self.n = tuple(n)
        self.ncells = int(nc.value)

    def close(self):
        if getattr(self, "h", None) and getattr(self, "_owned", False):
            lib().hcl_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape3(self):
        return (self.n[2], self.n[1], self.n[0])

    def zeros(self, ncomp=None):
        return np.zeros(self.shape3 if ncomp is None else (ncomp,) + self.shape3)

    # ---- grid --------------------------------------------------------
    def grid(self):
        x = [np.zeros(self.n[d] + 1) for d in range(3)]
        dx = [np.zeros(self.n[d]) for d in range(3)]
        xc = [np.zeros(self.n[d]) for d in range(3)]
        ds = np.zeros((3,) + self.shape3)
        dv = np.zeros(self.shape3)
        arr = lambda a: (C.c_void_p * 3)(*[v.ctypes.data for v in a])  # noqa: E731
        check(lib().hcl_get_grid(self.h, arr(x), arr(dx), arr(xc), _ptr(ds), _ptr(dv)))
        out = {"ds": ds, "dv": dv}
        for d in range(3):
            out[f"x{d}"] = x[d]
            out[f"dx{d}"] = dx[d]
            out[f"x{d}c"] = xc[d]
        return out

    # ---- stage entry points (device tensors) ---------------------------
    def conv_prim_to_cons(self, ng_eff, rho, u, P, rhou, E, stream=None):
        check(lib().hcl_conv_prim_to_cons(self.h, ng_eff, _ptr(rho), _ptr(u), _ptr(P), _ptr(rhou), _ptr(E), stream))

    def conv_cons_to_prim(self, ng_eff, rho, rhou, E, u, P, stream=None):
        check(lib().hcl_conv_cons_to_prim(self.h, ng_eff, _ptr(rho), _ptr(rhou), _ptr(E), _ptr(u), _ptr(P), stream))

    def face_reconstruction(self, ng_eff, var, var_rec, stream=None):
        check(lib().hcl_face_reconstruction(self.h, ng_eff, _ptr(var), _ptr(var_rec), stream))

    def hydro_reconstruction(self, ng_eff, dt, rho, u, P, fx, rho_rec, rhou_rec, E_rec, fx_rec, u_rec=None,
                             P_rec=None, stream=None):
        check(lib().hcl_hydro_reconstruction(self.h, ng_eff, float(dt), _ptr(rho), _ptr(u), _ptr(P), _ptr(fx),
                                             _ptr(rho_rec), _ptr(rhou_rec), _ptr(E_rec), _ptr(fx_rec), _ptr(u_rec),
                                             _ptr(P_rec), stream))

    def godunov_scheme(self, ng_eff, dt, rho, rhou, E, fx, rho_rec, rhou_rec, E_rec, fx_rec, rho_new, rhou_new,
                       E_new, fx_new, stream=None):
        check(lib().hcl_godunov_scheme(self.h, ng_eff, float(dt), _ptr(rho), _ptr(rhou), _ptr(E), _ptr(fx),
                                       _ptr(rho_rec), _ptr(rhou_rec), _ptr(E_rec), _ptr(fx_rec), _ptr(rho_new),
                                       _ptr(rhou_new), _ptr(E_new), _ptr(fx_new), stream))

    def pressure_fix(self, dt, eps, rho, rhou, E, rho_rec, rhou_rec, E_rec, rho_new, rhou_new, E_new, stream=None):
        check(lib().hcl_pressure_fix(self.h, float(dt), float(eps), _ptr(rho), _ptr(rhou), _ptr(E), _ptr(rho_rec),
                                     _ptr(rhou_rec), _ptr(E_rec), _ptr(rho_new), _ptr(rhou_new), _ptr(E_new),
                                     stream))

    def internal_mass_gravity(self, rho, g_out=None, stream=None):
        """make_internal_mass_gravity: the radial gravity table from the device
        density rho; g_out (device, n0 doubles) receives a copy of it."""
        check(lib().hcl_internal_mass_gravity(self.h, _ptr(rho), _ptr(g_out), stream))

    def boundary_conditions(self, rho, rhou, E, fx=None, stream=None):
        check(lib().hcl_boundary_conditions(self.h, _ptr(rho), _ptr(rhou), _ptr(E), _ptr(fx), stream))

    def time_step(self, ng_eff, rho, u, P, stream=None):
        out = C.c_double()
        check(lib().hcl_time_step(self.h, ng_eff, _ptr(rho), _ptr(u), _ptr(P), C.byref(out), stream))
        return out.value

    def minimum_internal_energy(self, rho, rhou, E, stream=None):
        out = C.c_double()
        check(lib().hcl_minimum_internal_energy(self.h, _ptr(rho), _ptr(rhou), _ptr(E), C.byref(out), stream))
        return out.value

    def integrate(self, var, stream=None):
        out = C.c_double()
        check(lib().hcl_integrate(self.h, _ptr(var), C.byref(out), stream))
        return out.value

    # ---- handle-owned state -------------------------------------------
    def set_state(self, rho, rhou, E, fx=None, device=False):
        if not device:
            rho, rhou, E = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, rhou, E))
            if fx is not None:
                fx = np.ascontiguousarray(fx, dtype=np.float64)
        check(lib().hcl_set_state(self.h, _ptr(rho), _ptr(rhou), _ptr(E), _ptr(fx), 1 if device else 0))

    def get_state(self, out=None, device=False, fx=None):
        """(rho, rhou, E); with nfx > 0, fx (an array of nfx planes) is filled too."""
        if out is None:
            out = (self.zeros(), self.zeros(self.ndim), self.zeros())
        rho, rhou, E = out
        check(lib().hcl_get_state(self.h, _ptr(rho), _ptr(rhou), _ptr(E), _ptr(fx), 1 if device else 0))
        return out

    def set_state_from_prim(self, rho, u, P, fx=None):
        rho, u, P = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, P))
        if fx is not None:
            fx = np.ascontiguousarray(fx, dtype=np.float64)
        check(lib().hcl_set_state_from_prim(self.h, _ptr(rho), _ptr(u), _ptr(P), _ptr(fx)))

    def reset_clock(self, t_ini=0.0):
        check(lib().hcl_reset_clock(self.h, float(t_ini)))

    def run(self, *, cfl=0.4, t_end=1e300, max_iter=2 ** 31 - 1, iter_frequency=0, time_frequency=0.0,
            time_first_output=None, nsteps=0, graph_chunk=0, dts=None, check_status=True):
        p = RunParams()
        p.cfl = cfl
        p.t_end = t_end
        p.max_iter = int(max_iter)
        p.iter_frequency = int(iter_frequency)
        p.time_frequency = float(time_frequency)
        p.time_first_output = float(time_frequency if time_first_output is None else time_first_output)
        p.nsteps = int(nsteps)
        p.graph_chunk = int(graph_chunk)
        keep = None
        if dts is not None:
            keep = np.ascontiguousarray(dts, dtype=np.float64)
            p.fixed_dt = 1
            p.dts = keep.ctypes.data_as(C.POINTER(C.c_double))
        r = RunResult()
        rc = lib().hcl_run(self.h, C.byref(p), C.byref(r))
        if check_status:
            check(rc)
        return r

    def step_fixed_dt(self, dt, stream=None):
        check(lib().hcl_step_fixed_dt(self.h, float(dt), stream))

    def dt_log(self, max_count=1 << 20):
        buf = np.zeros(max_count)
        cnt = C.c_int()
        check(lib().hcl_get_dt_log(self.h, _ptr(buf), max_count, C.byref(cnt)))
        return buf[: cnt.value].copy()

    # ---- discrete adjoint ----------------------------------------------
    def adjoint_forward(self, nsteps, *, dts=None, cfl=0.4, checkpoint_every=32, precision="fp64"):
        """Runs nsteps steps from the current state, checkpointing; returns the dts used."""
        from ._native import AdjointParams

        p = AdjointParams()
        p.nsteps = int(nsteps)
        keep = None
        if dts is not None:
            keep = np.ascontiguousarray(dts, dtype=np.float64)
            p.dts = keep.ctypes.data_as(C.POINTER(C.c_double))
        p.cfl = float(cfl)
        p.checkpoint_every = int(checkpoint_every)
        p.precision = _key(PRECISION, precision, "precision")
        check(lib().hcl_adjoint_forward(self.h, C.byref(p)))
        out = np.zeros(int(nsteps))
        cnt = C.c_int()
        check(lib().hcl_adjoint_dts(self.h, _ptr(out), int(nsteps), C.byref(cnt)))
        return out[: cnt.value]

    def adjoint_backward(self, lam_final, grad=None, device=False):
        """lam_final, grad: one contiguous buffer of (ndim+2+nfx)*N doubles
        (rho, rhou, E, then the passive scalars' fractions)."""
        if grad is None:
            grad = np.zeros(((self.ndim + 2 + self.nfx),) + self.shape3)
        if not device:
            lam_final = np.ascontiguousarray(lam_final, dtype=np.float64)
        check(lib().hcl_adjoint_backward(self.h, _ptr(lam_final), _ptr(grad), 1 if device else 0))
        return grad

    def get_prim(self, with_temperature=True, fx=None):
        """(rho, u, P, T) over all cells (reference layout), as main() holds
        them when it writes an output; fx (nfx, ...) is filled when given."""
        rho = self.zeros()
        u = self.zeros(self.ndim)
        P = self.zeros()
        T = self.zeros() if with_temperature else None
        check(lib().hcl_get_prim(self.h, _ptr(rho), _ptr(u), _ptr(P), _ptr(T), _ptr(fx), 0))
        return rho, u, P, T

    def set_clock(self, t, iteration):
        check(lib().hcl_set_clock(self.h, float(t), int(iteration)))

    def write_output(self, directory, prefix, output_id, *, iter_output_id=-1, time_output_id=-1, iteration=0,
                     t=0.0):
        """One output with the reference's dataset set (hcl_write_output):
        <directory>/<prefix>_<output_id:08d>.hclraw and <prefix>.xmf."""
        check(lib().hcl_write_output(self.h, str(directory).encode(), str(prefix).encode(), int(output_id),
                                     int(iter_output_id), int(time_output_id), int(iteration), float(t)))

    def read_restart(self, path):
        """Restart from an output file of the same grid (hcl_read_restart):
        sets the state and the clock; returns the file's counters."""
        out = [C.c_int(-1) for _ in range(4)]
        t = C.c_double(0.0)
        check(lib().hcl_read_restart(self.h, str(path).encode(), *[C.byref(o) for o in out], C.byref(t)))
        return {"output_id": out[0].value, "iter_output_id": out[1].value, "time_output_id": out[2].value,
                "iter": out[3].value, "current_time": t.value}

    def set_schedule(self, schedule):
        """Forces a schedule of the mixed kernel (-1: autotune); returns the one in use."""
        used = C.c_int()
        check(lib().hcl_set_schedule(self.h, int(schedule), C.byref(used)))
        return used.value

    def schedule(self):
        """Schedule of the mixed kernel in use (-1 until the autotuner has run)."""
        return self.set_schedule(-2)

    def interior(self):
        nx = (C.c_int * 3)()
        ng = C.c_int()
        check(lib().hcl_get_interior(self.h, nx, C.byref(ng)))
        return tuple(nx), ng.value

    def stream_handle(self) -> int:
        """cudaStream_t of the handle (for timing events on the launching stream)."""
        s = C.c_void_p()
        check(lib().hcl_get_stream(self.h, C.byref(s)))
        return int(s.value or 0)

    def conservation_sums(self):
        out = np.zeros(self.ndim + 2)
        check(lib().hcl_conservation_sums(self.h, _ptr(out)))
        return out


class Ensemble:
    """A batch of independent 2-D FP32-mixed problems stepped by one persistent
    cooperative launch (hcl_ensemble_*).  ``configs`` is a list of keyword
    dicts for :func:`make_config`; ``domains[p]`` is a :class:`Domain` view of
    problem p's handle (set its state, read its results)."""

    def __init__(self, configs):
        from ._native import EnsembleParams  # noqa: F401  (checks the binding)

        cfgs = (Config * len(configs))()
        self._nodes = []
        for p, kw in enumerate(configs):
            kw = dict(kw)
            kw.setdefault("precision", "fp32_mixed")
            cfg, nodes = make_config(2, kw.pop("nx"), **kw)
            cfgs[p] = cfg
            self._nodes.append(nodes)
        e = C.c_void_p()
        check(lib().hcl_ensemble_create(cfgs, len(configs), C.byref(e)))
        self.e = e
        self.domains = []
        for p in range(len(configs)):
            h = C.c_void_p()
            check(lib().hcl_ensemble_handle(e, p, C.byref(h)))
            self.domains.append(Domain._view(h, cfgs[p]))
        self.result = None

    def close(self):
        if getattr(self, "e", None):
            for d in self.domains:
                d.h = None
            lib().hcl_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.domains)

    def stream_handle(self) -> int:
        s = C.c_void_p()
        check(lib().hcl_ensemble_stream(self.e, C.byref(s)))
        return int(s.value or 0)

    def run(self, nsteps, *, cfl=0.4, checkpoint_every=0, strip_rows=0, blocks_per_sm=0, use_graph=True,
            adjoint_precision="fp64", check_status=True, warps_per_cta=0, barrier_spin_limit=0,
            barrier_extra_arrivals=0):
        from ._native import EnsembleParams, EnsembleResult

        p = EnsembleParams()
        p.nsteps = int(nsteps)
        p.cfl = float(cfl)
        p.checkpoint_every = int(checkpoint_every)
        p.strip_rows = int(strip_rows)
        p.blocks_per_sm = int(blocks_per_sm)
        p.use_graph = 1 if use_graph else 0
        p.adjoint_precision = _key(PRECISION, adjoint_precision, "precision")
        p.warps_per_cta = int(warps_per_cta)
        p.barrier_spin_limit = int(barrier_spin_limit)
        p.barrier_extra_arrivals = int(barrier_extra_arrivals)
        r = EnsembleResult()
        rc = lib().hcl_ensemble_run(self.e, C.byref(p), C.byref(r))
        if check_status:
            check(rc)
        self.result = r
        return r

    def adjoint(self, lam_finals, grads, device=True):
        """Reverse pass of the last run (checkpoint_every > 0); per problem one
        contiguous (ndim+2)*N buffer for lam_final and for the gradient."""
        n = len(self.domains)
        lam = (C.c_void_p * n)(*[_ptr(t).value for t in lam_finals])
        out = (C.c_void_p * n)(*[_ptr(t).value for t in grads])
        check(lib().hcl_ensemble_adjoint(self.e, lam, out, 1 if device else 0))
        return grads
