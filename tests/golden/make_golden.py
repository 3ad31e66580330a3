"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run where the reference tree is present (the checkout the oracle recipe
reads: HCL_REF_SRC=<checkout>/src or the recipe's default) after
``make -C oracle ref``:

    python tests/golden/make_golden.py

Outputs (small, committed):
  sod_exact.npz        -- exact Riemann solution of the Sod tube at t=0.2 on
                          the 1024 cell centres of [0, 1], from the
                          reference's test/exact_shock_tube.py (Toro).
  ref_cell_vectors.npz -- outputs of the reference's own per-cell physics
                          (oracle/_ref, built from hydro/*.hpp and
                          thermodynamics/perfect_gas.*) on seeded states.
"""
import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
from oracle import reference_root  # noqa: E402

REF_ROOT = reference_root()
if REF_ROOT is None:
    raise SystemExit("reference checkout not found: set HCL_REF_SRC to its src/ directory")

SOLVERS = ["HLL", "HLLC", "Low Mach"]
LIMS = ["Constant", "VanLeer", "Minmod", "VanAlbada"]


def sod_exact():
    spec = importlib.util.spec_from_file_location("exact_shock_tube", REF_ROOT / "test" / "exact_shock_tube.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    gamma = 1.4
    nx = 1024
    x = (np.arange(nx) + 0.5) / nx
    rhoL, uL, PL = 1.0, 0.0, 1.0
    rhoR, uR, PR = 0.125, 0.0, 0.1
    cL = np.sqrt(gamma * PL / rhoL)
    cR = np.sqrt(gamma * PR / rhoR)
    rho, u, P, e = mod.ExactShockTube(x, 0.5, [rhoL, uL, PL, cL], [rhoR, uR, PR, cR], 0.2, gamma)
    np.savez_compressed(HERE / "sod_exact.npz", x=x, rho=rho, u=u, P=P, e=e, t=0.2, gamma=gamma)


def ref_cell_vectors():
    from oracle import RefCell

    out = {}
    for ndim in (1, 2, 3):
        ref = RefCell(ndim)
        rng = np.random.default_rng(2024 + ndim)
        n = 64
        prim = np.concatenate([rng.uniform(0.05, 5.0, (n, 1)), rng.uniform(-3, 3, (n, ndim)),
                               rng.uniform(0.01, 10.0, (n, 1))], axis=1)
        prim[::5, 1:1 + ndim] *= 4.0
        for gi, (gamma, mmw) in enumerate([(1.4, 1.0), (5.0 / 3.0, 0.6)]):
            key = f"d{ndim}_g{gi}"
            cons = np.array([ref.to_cons(gamma, mmw, p) for p in prim])
            out[key + "_gamma_mmw"] = np.array([gamma, mmw])
            out[key + "_prim"] = prim
            out[key + "_to_cons"] = cons
            out[key + "_to_prim"] = np.array([ref.to_prim(gamma, mmw, c) for c in cons])
            out[key + "_flux_prim"] = np.array([[ref.flux_from_prim(gamma, mmw, p, l) for l in range(ndim)]
                                               for p in prim])
            for s in SOLVERS:
                out[key + f"_riemann_{s.replace(' ', '_')}"] = np.array(
                    [[ref.riemann(s, gamma, mmw, cons[i], cons[i + 1], l) for l in range(ndim)]
                     for i in range(n - 1)])
    ref = RefCell(1)
    rng = np.random.default_rng(99)
    diffs = rng.normal(size=(500, 2)) * 10.0 ** rng.integers(-4, 4, size=(500, 2))
    out["slope_diffs"] = diffs
    for lim in LIMS:
        out[f"slope_{lim}"] = np.array([ref.slope(lim, r, l) for r, l in diffs])
    np.savez_compressed(HERE / "ref_cell_vectors.npz", **out)


if __name__ == "__main__":
    sod_exact()
    ref_cell_vectors()
    print("golden fixtures written to", HERE)
