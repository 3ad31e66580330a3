"""Parity at the sizes the benchmark runs.

The schedule tests compare every kernel with the oracle on small grids, where a
strip kernel gets a handful of strips and most of its warps idle.  These tests
run the kernels on the benchmark's own grids and work distribution:

* Kelvin-Helmholtz 2048^2 (periodic, van Leer, HLLC, CFL 0.4): the plain FP64
  fused step for 10 steps bit for bit against the oracle (every field, ghost
  cells included, and the CFL dt sequence); fast FP64 for 10 steps within
  1e-12 relative L1 per field; the FP32-mixed step on schedule 9
  (one 16-warp CTA per SM, 2368 strips of 64 rows) for 20 steps with the
  oracle's dts, relative L1 and L-infinity per field; its rows staged by TMA
  (schedule 9) or by per-lane cp.async (schedule 10) give the same bits.
* Rayleigh-Taylor 256x256x512 (reflecting z walls, g_z = -0.1, Minmod, HLL):
  the FP64 fused step (8x8x4 tiles) for 3 steps bit for bit, the FP32-mixed
  column march (440 CTAs x 256 planes) for 3 steps with the oracle's dts.

The oracle steps these grids with OpenMP on the host cores (KH: about 0.15 s
per step on 8 cores; RT: about 1.3 s per step and 22 GB of host memory).
"""
import numpy as np
import pytest

from cases import rel_l1

pytestmark = pytest.mark.gpu

KH_NX = [2048, 2048]
KH_KW = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
RT_NX = [256, 256, 512]
RT_KW = dict(gamma=1.4, limiter="Minmod", riemann="HLL",
             bc=["Periodic", "Periodic", "Periodic", "Periodic", "Reflexive", "Reflexive"],
             g=(0.0, 0.0, -0.1), xmax=(0.5, 0.5, 1.0))
# bytes of host memory the 3-D oracle needs: about 80 doubles per cell with ghosts
RT_HOST_BYTES = 80 * 8 * 260 * 260 * 516


def fields(rho, rhou, E):
    out = {"rho": rho, "E": E}
    for k in range(rhou.shape[0]):
        out[f"rhou_{k}"] = rhou[k]
    return out


def rel_linf(a, b):
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a - b)))


@pytest.fixture(scope="module")
def kh():
    """Oracle KH 2048^2: initial primitives, states after 10 and 20 steps,
    the dt sequence of the 20 steps."""
    from heraclespp_b200 import setups
    from oracle import Oracle

    o = Oracle(2, KH_NX, **KH_KW)
    prim = setups.kelvin_helmholtz(setups.Grid.from_domain(o))
    rho, rhou, E, fx = o.init_from_prim(*prim)
    _, it, st, dts10 = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=10, record_dts=True)
    assert (it, st) == (10, 0)
    s10 = (rho.copy(), rhou.copy(), E.copy())
    _, it, st, dts_more = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=10, record_dts=True)
    assert (it, st) == (10, 0)
    return prim, s10, (rho, rhou, E), np.concatenate([dts10, dts_more])


def test_kh2048_fp64_fused_bitwise(kh):
    from heraclespp_b200 import Domain

    prim, (rho, rhou, E), _, dts = kh
    d = Domain(2, KH_NX, precision="fp64", **KH_KW)
    d.set_state_from_prim(*prim)
    r = d.run(cfl=0.4, max_iter=10)
    assert r.iter == 10
    assert np.array_equal(d.dt_log()[:10], dts[:10])
    got = fields(*d.get_state())
    d.close()
    for name, ref in fields(rho, rhou, E).items():
        assert np.array_equal(got[name], ref), name


def test_kh2048_fast64_within_1e12(kh):
    """Fast FP64 on the benchmark grid: 10 steps with the oracle's dts, every
    field within 1e-12 relative L1 (ghost cells included)."""
    from heraclespp_b200 import Domain

    prim, (rho, rhou, E), _, dts = kh
    d = Domain(2, KH_NX, precision="fp64_fast", **KH_KW)
    d.set_state_from_prim(*prim)
    d.run(nsteps=10, dts=dts[:10])
    got = fields(*d.get_state())
    d.close()
    for name, ref in fields(rho, rhou, E).items():
        assert rel_l1(got[name], ref) < 1e-12, name


def test_kh2048_mixed_schedule9_every_field(kh):
    from heraclespp_b200 import Domain

    prim, _, (rho, rhou, E), dts = kh
    d = Domain(2, KH_NX, precision="fp32_mixed", **KH_KW)
    assert d.set_schedule(9) == 9
    d.set_state_from_prim(*prim)
    d.run(nsteps=20, dts=dts)
    got = fields(*d.get_state())
    d.close()
    ref = fields(rho, rhou, E)
    # relative L1 over the whole array (ghost images included), per field;
    # rhou_1 is the small transverse momentum (|v| ~ 0.01)
    l1_bound = {"rho": 2e-6, "E": 2e-6, "rhou_0": 2e-6, "rhou_1": 5e-5}
    for name in ref:
        l1 = rel_l1(got[name], ref[name])
        assert l1 < l1_bound[name], (name, l1)
        assert rel_linf(got[name], ref[name]) < 1e-3, name
    # schedule 10 stages the same rows by per-lane cp.async instead of TMA:
    # the same bits
    d = Domain(2, KH_NX, precision="fp32_mixed", **KH_KW)
    assert d.set_schedule(10) == 10
    d.set_state_from_prim(*prim)
    d.run(nsteps=20, dts=dts)
    got10 = fields(*d.get_state())
    d.close()
    for name in ref:
        assert np.array_equal(got10[name], got[name]), name


@pytest.fixture(scope="module")
def rt():
    import psutil

    if psutil.virtual_memory().available < 1.5 * RT_HOST_BYTES:
        pytest.skip(f"the 3-D oracle needs about {RT_HOST_BYTES / 1e9:.0f} GB of host memory")
    from heraclespp_b200 import setups
    from oracle import Oracle

    o = Oracle(3, RT_NX, **RT_KW)
    prim = setups.rayleigh_taylor_3d(setups.Grid.from_domain(o))
    rho, rhou, E, fx = o.init_from_prim(*prim)
    _, it, st, dts = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=3, record_dts=True)
    assert (it, st) == (3, 0)
    del o
    return prim, (rho, rhou, E), dts


def test_rt3d_fp64_fused_bitwise(rt):
    from heraclespp_b200 import Domain

    prim, (rho, rhou, E), dts = rt
    d = Domain(3, RT_NX, precision="fp64", **RT_KW)
    d.set_state_from_prim(*prim)
    r = d.run(cfl=0.4, max_iter=3)
    assert r.iter == 3
    assert np.array_equal(d.dt_log()[:3], dts)
    got = fields(*d.get_state())
    d.close()
    for name, ref in fields(rho, rhou, E).items():
        assert np.array_equal(got[name], ref), name


def test_rt3d_fast64_within_1e12(rt):
    """Fast FP64 on the 3-D benchmark grid: 3 steps with the oracle's dts,
    every field within 1e-12 relative L1 (the transverse momenta on the scale
    of the vertical one)."""
    from heraclespp_b200 import Domain

    prim, (rho, rhou, E), dts = rt
    d = Domain(3, RT_NX, precision="fp64_fast", **RT_KW)
    d.set_state_from_prim(*prim)
    d.run(nsteps=3, dts=dts)
    got = fields(*d.get_state())
    d.close()
    ref = fields(rho, rhou, E)
    for name in ("rho", "E", "rhou_2"):
        assert rel_l1(got[name], ref[name]) < 1e-12, name
    scale = float(np.sum(np.abs(ref["rhou_2"])))
    for name in ("rhou_0", "rhou_1"):
        assert float(np.sum(np.abs(got[name] - ref[name]))) / scale < 1e-12, name


def test_rt3d_mixed_column_march_every_field(rt):
    from heraclespp_b200 import Domain

    prim, (rho, rhou, E), dts = rt
    d = Domain(3, RT_NX, precision="fp32_mixed", **RT_KW)
    assert d.set_schedule(1) == 1
    d.set_state_from_prim(*prim)
    d.run(nsteps=3, dts=dts)
    got = fields(*d.get_state())
    d.close()
    ref = fields(rho, rhou, E)
    for name in ("rho", "E"):
        assert rel_l1(got[name], ref[name]) < 2e-7, name
        assert rel_linf(got[name], ref[name]) < 1e-5, name
    # the transverse momenta start at zero and stay ~1e-6: compare them on the
    # scale of the vertical momentum
    scale = float(np.sum(np.abs(ref["rhou_2"])))
    for name in ("rhou_0", "rhou_1", "rhou_2"):
        err = float(np.sum(np.abs(got[name] - ref[name]))) / scale
        assert err < 1e-4, (name, err)
