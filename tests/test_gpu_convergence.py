"""Second-order convergence of the FP32-mixed step on the reference's
advection_sinus problem (test/convergence_advection_sinus/
check_convergence_advection_sinus.py:52-80: L1 density error after one
period, slope within 5 % of 2 for the FP64 method): the 1-D fused kernel and,
in 2-D, the warp-strip schedules (the profile varies along x only)."""
import numpy as np
import pytest

from heraclespp_b200 import Domain, setups

pytestmark = pytest.mark.gpu


def advection_error(ndim, nx, schedule=None):
    # 2-D: 16 rows of square cells, so that dt scales with dx as in 1-D
    n = [nx] if ndim == 1 else [nx, 16]
    d = Domain(ndim, n, gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * (2 * ndim),
               precision="fp32_mixed", xmax=(1.0, 16.0 / nx, 1.0))
    if schedule is not None:
        assert d.set_schedule(schedule) == schedule
    grid = setups.Grid.from_domain(d)
    d.set_state_from_prim(*setups.advection_sinus(grid))
    r = d.run(cfl=0.4, t_end=1.0, max_iter=10 ** 7, time_frequency=1.0)
    assert r.status == 0 and r.t == 1.0
    rho = d.get_state()[0]
    x = d.grid()["x0"][2:-2]
    exact = 1 + 0.1 * np.sin(2 * np.pi * (x[1:] + x[:-1]) / 2)
    row = rho[0, 2 if ndim == 2 else 0, 2:-2]
    return float(np.sum(np.abs(exact - row) * np.diff(x)))


@pytest.mark.parametrize("ndim,schedule", [(1, None), (2, 6), (2, 9)])
def test_mixed_second_order(ndim, schedule):
    nxs = [32 * 2 ** i for i in range(4)]
    errs = np.array([advection_error(ndim, n, schedule) for n in nxs])
    slope = np.polyfit(np.log10(nxs[0] / np.array(nxs)), np.log10(errs), 1)[0]
    assert abs(slope - 2) / 2 < 0.05, (slope, errs)
