"""Failure path of the ensemble's bounded grid barrier.

The persistent ensemble kernel separates time steps with a grid barrier whose
thread-0 poll loop gives up after a limit and records HCL_ERR_TIMEOUT, after
which every CTA returns.  Here the barrier is told to wait for one arrival
more than the CTAs it has (an arrival that never comes) with a short poll
limit: the run must come back with HCL_ERR_TIMEOUT instead of hanging, and
the same process and GPU must then run the same batch normally, bit for bit
equal to the single-problem kernel.  No GPU fault is involved: the wait simply
runs out and the host reads the status."""
import numpy as np
import pytest

from test_gpu_ensemble import SIDES, initial, make_ensemble, single

pytestmark = pytest.mark.gpu

HCL_ERR_TIMEOUT = 6


@pytest.mark.parametrize("use_graph,nw", [(False, 4), (True, 16)])
def test_barrier_timeout_then_normal_run(use_graph, nw):
    from heraclespp_b200._native import lib

    ens = make_ensemble()
    r = ens.run(6, strip_rows=64, warps_per_cta=nw, use_graph=use_graph, barrier_spin_limit=2000,
                barrier_extra_arrivals=1, check_status=False)
    assert r.status == HCL_ERR_TIMEOUT
    assert "timed out" in lib().hcl_last_error().decode()
    # the context is intact: the same batch, reset, runs to completion
    for p, d in enumerate(ens.domains):
        d.set_state_from_prim(*initial(d, p))
    n = 12
    r = ens.run(n, strip_rows=64, warps_per_cta=nw, use_graph=use_graph)
    assert r.status == 0
    for p, (nx, d_e) in enumerate(zip(SIDES, ens.domains)):
        d = single(p, list(nx), 64)
        d.run(nsteps=n)
        for a, b in zip(d_e.get_state(), d.get_state()):
            assert np.array_equal(a, b), f"problem {p}"
        d.close()
    ens.close()
