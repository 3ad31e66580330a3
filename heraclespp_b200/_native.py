"""ctypes binding of libheracles_b200.so (include/heracles_b200.h).

The library is built in-tree (``make -C heraclespp_b200``).  There is no
fallback: if the shared library is missing or a device call fails, the error
surfaces as an exception.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libheracles_b200.so"

HCL_OK = 0
STATUS_NAMES = {
    1: "HCL_ERR_CONFIG", 2: "HCL_ERR_DOMAIN", 3: "HCL_ERR_CUDA", 4: "HCL_ERR_INVALID_STATE",
    5: "HCL_ERR_NEGATIVE_DT", 6: "HCL_ERR_TIMEOUT", 7: "HCL_ERR_NO_DEVICE", 8: "HCL_ERR_ARGUMENT",
}

LIMITERS = {"Constant": 0, "VanLeer": 1, "Minmod": 2, "VanAlbada": 3}
RIEMANN = {"HLL": 0, "HLLC": 1, "Low Mach": 2}
BCS = {"NullGradient": 0, "Periodic": 1, "Reflexive": 2}
GEOMS = {"Cartesian": 0, "Spherical": 1}
GRAVITY = {"Uniform": 0, "Point_mass": 1, "Internal_mass": 2}
EOS = {"PerfectGas": 0, "RadGas": 1}
PRECISION = {"fp64": 0, "fp32_mixed": 1, "fp64_fast": 2}

# Every entry point declared in include/heracles_b200.h.
EXPORTS = [
    "hcl_config_default", "hcl_create", "hcl_destroy", "hcl_last_error", "hcl_abi_version", "hcl_get_extents",
    "hcl_get_grid", "hcl_get_grid_device", "hcl_conv_prim_to_cons", "hcl_conv_cons_to_prim",
    "hcl_face_reconstruction", "hcl_hydro_reconstruction", "hcl_godunov_scheme", "hcl_boundary_conditions",
    "hcl_time_step", "hcl_minimum_internal_energy", "hcl_integrate", "hcl_set_state", "hcl_get_state",
    "hcl_set_state_from_prim", "hcl_run", "hcl_step_fixed_dt", "hcl_reset_clock", "hcl_get_dt_log",
    "hcl_conservation_sums", "hcl_kernel_launch_count", "hcl_get_stream", "hcl_get_interior",
    "hcl_adjoint_forward", "hcl_adjoint_backward", "hcl_adjoint_dts", "hcl_set_schedule",
    "hcl_ensemble_create", "hcl_ensemble_destroy", "hcl_ensemble_handle", "hcl_ensemble_stream",
    "hcl_ensemble_run", "hcl_ensemble_adjoint", "hcl_pressure_fix", "hcl_internal_mass_gravity",
    "hcl_set_stage_loop", "hcl_temperature", "hcl_get_prim", "hcl_set_clock", "hcl_get_config",
    "hcl_write_output", "hcl_read_restart",
]


class HclError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class DomainError(HclError, ValueError):
    """Invalid EOS parameter (the reference throws std::domain_error)."""


class Config(C.Structure):
    _fields_ = [
        ("ndim", C.c_int),
        ("nx", C.c_int * 3),
        ("nghost", C.c_int),
        ("nfx", C.c_int),
        ("geometry", C.c_int),
        ("gamma", C.c_double),
        ("mmw", C.c_double),
        ("limiter", C.c_int),
        ("riemann", C.c_int),
        ("bc", C.c_int * 6),
        ("gravity", C.c_int),
        ("g", C.c_double * 3),
        ("central_mass", C.c_double),
        ("xmin", C.c_double * 3),
        ("xmax", C.c_double * 3),
        ("nodes", C.c_void_p * 3),
        ("precision", C.c_int),
        ("device", C.c_int),
        ("pressure_fix", C.c_int),
        ("eps_pf", C.c_double),
        ("eos", C.c_int),
    ]


class RunParams(C.Structure):
    _fields_ = [
        ("cfl", C.c_double),
        ("t_end", C.c_double),
        ("max_iter", C.c_int),
        ("iter_frequency", C.c_int),
        ("time_frequency", C.c_double),
        ("time_first_output", C.c_double),
        ("nsteps", C.c_int),
        ("graph_chunk", C.c_int),
        ("fixed_dt", C.c_int),
        ("dts", C.POINTER(C.c_double)),
    ]


class AdjointParams(C.Structure):
    _fields_ = [
        ("nsteps", C.c_int),
        ("dts", C.POINTER(C.c_double)),
        ("cfl", C.c_double),
        ("checkpoint_every", C.c_int),
        ("precision", C.c_int),
    ]


class EnsembleParams(C.Structure):
    _fields_ = [
        ("nsteps", C.c_int),
        ("cfl", C.c_double),
        ("checkpoint_every", C.c_int),
        ("strip_rows", C.c_int),
        ("blocks_per_sm", C.c_int),
        ("use_graph", C.c_int),
        ("adjoint_precision", C.c_int),
        ("warps_per_cta", C.c_int),
        ("barrier_spin_limit", C.c_longlong),
        ("barrier_extra_arrivals", C.c_int),
    ]


class EnsembleResult(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("strip_rows", C.c_int),
        ("blocks_per_sm", C.c_int),
        ("grid", C.c_int),
        ("launches", C.c_int),
        ("graph", C.c_int),
        ("cells", C.c_int64),
        ("warps_per_cta", C.c_int),
    ]


class RunResult(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("iter", C.c_int),
        ("status", C.c_int),
        ("bad_cell", C.c_int64),
        ("finished", C.c_int),
        ("last_dt", C.c_double),
    ]


_LIB = None


def lib():
    """Loads the in-tree shared library (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("HCL_LIB", str(LIB_PATH)))
    if not path.exists():
        raise FileNotFoundError(
            f"{path} not found: build it with `make -C heraclespp_b200` (or __graft_entry__.build()); "
            "there is no CPU fallback")
    L = C.CDLL(str(path))
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    H = C.c_void_p
    L.hcl_config_default.argtypes = [C.POINTER(Config)]
    L.hcl_config_default.restype = None
    L.hcl_create.argtypes = [C.POINTER(Config), C.POINTER(H)]
    L.hcl_destroy.argtypes = [H]
    L.hcl_last_error.restype = C.c_char_p
    L.hcl_abi_version.restype = i
    L.hcl_get_extents.argtypes = [H, C.c_int * 3, C.POINTER(C.c_int64)]
    L.hcl_get_grid.argtypes = [H, vp * 3, vp * 3, vp * 3, vp, vp]
    L.hcl_get_grid_device.argtypes = [H, vp * 3, C.POINTER(vp), C.POINTER(vp)]
    L.hcl_conv_prim_to_cons.argtypes = [H, i, vp, vp, vp, vp, vp, vp]
    L.hcl_conv_cons_to_prim.argtypes = [H, i, vp, vp, vp, vp, vp, vp]
    L.hcl_face_reconstruction.argtypes = [H, i, vp, vp, vp]
    L.hcl_hydro_reconstruction.argtypes = [H, i, d] + [vp] * 11
    L.hcl_godunov_scheme.argtypes = [H, i, d] + [vp] * 13
    L.hcl_boundary_conditions.argtypes = [H, vp, vp, vp, vp, vp]
    L.hcl_pressure_fix.argtypes = [H, d, d] + [vp] * 10
    L.hcl_internal_mass_gravity.argtypes = [H, vp, vp, vp]
    L.hcl_time_step.argtypes = [H, i, vp, vp, vp, C.POINTER(d), vp]
    L.hcl_minimum_internal_energy.argtypes = [H, vp, vp, vp, C.POINTER(d), vp]
    L.hcl_integrate.argtypes = [H, vp, C.POINTER(d), vp]
    L.hcl_set_state.argtypes = [H, vp, vp, vp, vp, i]
    L.hcl_get_state.argtypes = [H, vp, vp, vp, vp, i]
    L.hcl_set_state_from_prim.argtypes = [H, vp, vp, vp, vp]
    L.hcl_run.argtypes = [H, C.POINTER(RunParams), C.POINTER(RunResult)]
    L.hcl_step_fixed_dt.argtypes = [H, d, vp]
    L.hcl_reset_clock.argtypes = [H, d]
    L.hcl_get_dt_log.argtypes = [H, vp, i, C.POINTER(i)]
    L.hcl_conservation_sums.argtypes = [H, vp]
    L.hcl_kernel_launch_count.restype = C.c_int64
    L.hcl_get_stream.argtypes = [H, C.POINTER(vp)]
    L.hcl_get_interior.argtypes = [H, C.c_int * 3, C.POINTER(i)]
    L.hcl_adjoint_forward.argtypes = [H, C.POINTER(AdjointParams)]
    L.hcl_adjoint_backward.argtypes = [H, vp, vp, i]
    L.hcl_adjoint_dts.argtypes = [H, vp, i, C.POINTER(i)]
    L.hcl_set_schedule.argtypes = [H, i, C.POINTER(i)]
    L.hcl_set_stage_loop.argtypes = [H, i]
    L.hcl_temperature.argtypes = [H, i, vp, vp, vp, vp]
    L.hcl_get_prim.argtypes = [H, vp, vp, vp, vp, vp, i]
    L.hcl_set_clock.argtypes = [H, d, i]
    L.hcl_get_config.argtypes = [H, C.POINTER(Config)]
    L.hcl_write_output.argtypes = [H, C.c_char_p, C.c_char_p, i, i, i, i, d]
    L.hcl_read_restart.argtypes = [H, C.c_char_p, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i),
                                   C.POINTER(d)]
    L.hcl_ensemble_create.argtypes = [C.POINTER(Config), i, C.POINTER(vp)]
    L.hcl_ensemble_destroy.argtypes = [vp]
    L.hcl_ensemble_handle.argtypes = [vp, i, C.POINTER(H)]
    L.hcl_ensemble_stream.argtypes = [vp, C.POINTER(vp)]
    L.hcl_ensemble_run.argtypes = [vp, C.POINTER(EnsembleParams), C.POINTER(EnsembleResult)]
    L.hcl_ensemble_adjoint.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), i]
    _LIB = L
    return L


def check(rc: int):
    if rc != HCL_OK:
        msg = lib().hcl_last_error().decode(errors="replace")
        if rc == 2:
            raise DomainError(rc, msg)
        raise HclError(rc, msg)
