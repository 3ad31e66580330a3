"""Outputs and restarts with the reference's dataset set (hcl_write_output,
hcl_read_restart; io/config.yaml.cpp:7-265, io/io.cpp:185-420,
main.cpp:225-246).

* The file holds exactly the reference's datasets for the dimension and
  scalar count, with the interior fields equal to the oracle's: rho and E of
  the state, u and P from conv_cons_to_prim, T from the EOS temperature.
* A restart into a fresh handle of the same grid rebuilds the state as main()
  does after read_pdi -- conv_prim_to_cons on the interior, then the boundary
  sequence -- bit for bit against the oracle doing the same, restores the clock
  and the counters, and continues bit for bit like the oracle continuing from
  that state.
* A file of another grid is refused; the XDMF index lists every output."""
import numpy as np
import pytest

import heraclespp_b200 as hb
from cases import make_pair
from heraclespp_b200.output import read_index, read_output

pytestmark = pytest.mark.gpu


def interior(a, ndim, ng=2):
    sl = tuple(slice(ng, -ng) if k < ndim else slice(None) for k in (2, 1, 0))
    return a[sl]


@pytest.mark.parametrize("name,nfx", [("sod_1d_odd", 0), ("quad_2d", 2), ("rt_3d_ragged", 1)])
def test_output_then_restart(tmp_path, name, nfx):
    o, d, prim = make_pair(name, "fp64")
    ndim = o.ndim
    if nfx:
        from cases import CASES, oracle_kwargs
        from oracle import Oracle

        _, nx, kw, _, _ = CASES[name]
        o = Oracle(ndim, nx, nfx=nfx, **oracle_kwargs(kw))
        d.close()
        d = hb.Domain(ndim, nx, nfx=nfx, **kw)
    rho, rhou, E, fx = o.init_from_prim(*prim)
    if nfx:
        fx[:] = np.random.default_rng(3).uniform(0, 1, fx.shape)
        o.boundaries(rho, rhou, E, fx)
    d.set_state(rho, rhou, E, fx=fx if nfx else None)
    steps = 12
    t_o, it_o, st_o, _ = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=steps)
    r = d.run(cfl=0.4, max_iter=steps)
    assert r.iter == it_o == steps and r.t == t_o

    d.write_output(tmp_path, "result", 3, iter_output_id=2, time_output_id=-1, iteration=r.iter, t=r.t)
    f = tmp_path / "result_00000003.hclraw"
    data = read_output(f)
    expect = {"output_id", "iter_output_id", "time_output_id", "iter", "current_time", "gamma", "x0", "x1", "x2",
              "x0_ng", "x1_ng", "x2_ng", "rho", "P", "E", "T"} | {f"ux{k}" for k in range(ndim)} | \
        {f"fx{k}" for k in range(nfx)}
    assert set(data) == expect
    assert (data["output_id"], data["iter_output_id"], data["time_output_id"], data["iter"]) == (3, 2, -1, steps)
    assert data["current_time"] == t_o and data["gamma"] == 1.4
    # interior fields against the oracle's arrays of the same state
    u_o, P_o = o.conv_cons_to_prim(2, rho, rhou, E)
    T_o = np.vectorize(o.temperature)(rho, P_o)
    nxs = tuple(data["rho"].shape)
    assert nxs == interior(rho, ndim).shape
    assert np.array_equal(data["rho"], interior(rho, ndim))
    assert np.array_equal(data["E"], interior(E, ndim))
    assert np.array_equal(data["P"], interior(P_o, ndim))
    assert np.array_equal(data["T"], interior(T_o, ndim))
    for k in range(ndim):
        assert np.array_equal(data[f"ux{k}"], interior(u_o[k], ndim))
    for k in range(nfx):
        assert np.array_equal(data[f"fx{k}"], interior(fx[k], ndim))
    g = o.grid()
    for k in range(3):
        assert np.array_equal(data[f"x{k}"], g[f"x{k}"])
        ng = 2 if k < ndim else 0
        assert np.array_equal(data[f"x{k}_ng"], g[f"x{k}"][ng:len(g[f"x{k}"]) - ng])
    offsets = [off for _, _, off, _ in read_index(f)]
    assert all(off % 64 == 0 for off in offsets)

    # restart into a fresh handle: state from the primitives, clock, counters
    from cases import CASES

    _, nx, kw, _, _ = CASES[name]
    d2 = hb.Domain(ndim, nx, nfx=nfx, **kw)
    meta = d2.read_restart(f)
    assert meta == {"output_id": 3, "iter_output_id": 2, "time_output_id": -1, "iter": steps, "current_time": t_o}
    # the oracle rebuilds the state the same way (main.cpp:225-246 then :305-307)
    rho_r = np.zeros_like(rho)
    u_r = np.zeros_like(u_o)
    P_r = np.zeros_like(P_o)
    sl = tuple(slice(2, -2) if k < ndim else slice(None) for k in (2, 1, 0))
    rho_r[sl] = rho[sl]
    P_r[sl] = P_o[sl]
    for k in range(ndim):
        u_r[k][sl] = u_o[k][sl]
    m_r, E_r = o.conv_prim_to_cons(0, rho_r, u_r, P_r)
    fx_r = np.zeros_like(fx)
    if nfx:
        for k in range(nfx):
            fx_r[k][sl] = fx[k][sl]
    o.boundaries(rho_r, m_r, E_r, fx_r)
    fx_d = np.zeros_like(fx) if nfx else None
    s2 = d2.get_state(fx=fx_d)
    assert np.array_equal(s2[0], rho_r) and np.array_equal(s2[1], m_r) and np.array_equal(s2[2], E_r)
    if nfx:
        assert np.array_equal(fx_d, fx_r)
    # continuing: 8 more steps (max_iter is absolute) like the oracle's loop
    # started at t from the restarted state
    t2, it2, st2, _ = o.run(rho_r, m_r, E_r, fx_r, cfl=0.4, t_ini=t_o, max_iter=8)
    r2 = d2.run(cfl=0.4, max_iter=steps + 8)
    assert st2 == 0 and it2 == 8 and r2.iter == steps + 8 and r2.t == t2
    s3 = d2.get_state()
    assert np.array_equal(s3[0], rho_r) and np.array_equal(s3[1], m_r) and np.array_equal(s3[2], E_r)
    d2.close()
    d.close()
    assert (tmp_path / "result.xmf").exists()


def test_restart_refuses_another_grid(tmp_path):
    o, d, prim = make_pair("kh_2d_ragged", "fp64")
    d.set_state_from_prim(*prim)
    d.write_output(tmp_path, "kh", 0)
    other = hb.Domain(2, [37, 22], gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
    with pytest.raises(hb.HclError):
        other.read_restart(tmp_path / "kh_00000000.hclraw")
    with pytest.raises(hb.HclError):
        d.read_restart(tmp_path / "missing.hclraw")


def test_xdmf_lists_every_output(tmp_path):
    o, d, prim = make_pair("kh_2d", "fp64")
    d.set_state_from_prim(*prim)
    ts = []
    for k in range(3):
        r = d.run(cfl=0.4, nsteps=2)
        d.write_output(tmp_path, "kh", k, iteration=r.iter, t=r.t)
        ts.append(r.t)
    text = (tmp_path / "kh.xmf").read_text()
    for k in range(3):
        assert f"kh_{k:08d}.hclraw" in text
        assert f'Name="output_{k}"' in text
    idx = {n: off for n, _, off, _ in read_index(tmp_path / "kh_00000002.hclraw")}
    assert f'Seek="{idx["rho"]}"' in text
    d.close()
