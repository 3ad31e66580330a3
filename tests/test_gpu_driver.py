"""The .ini front end (hcl_create_from_ini) and the heracles_b200 driver:
the same input file the reference reads, run on the GPU, checked bitwise
against the oracle run of the same problem."""
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from heraclespp_b200 import setups
from oracle import Oracle

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
DRIVER = ROOT / "heraclespp_b200" / "bin" / "heracles_b200"

# inputs/shock_tube.ini of the reference with Nx0_glob = 1024 (Sod, 1024 cells)
SOD_INI = """
[Grid]
Nx0_glob = 1024
Nx1_glob = 1
Nx2_glob = 1
x0min = 0
x0max = 1

[Run]
t_end = 0.2
cfl = 0.4

[Output]
max_iter = 100000
time_frequency = 0.1
prefix = shock_tube

[Hydro]
reconstruction = Minmod
riemann_solver = HLLC

[Boundary Condition]
BC_X0 = NullGradient

[Perfect Gas]
gamma = 1.4

[Initialisation]
rho0 = 1
rho1 = 0.125
u0 = 0
u1 = 0
P0 = 1
P1 = 0.1
inter = 0.5
"""


def read_dump(path):
    b = Path(path).read_bytes()
    nd, n0, n1, n2 = struct.unpack("4i", b[:16])
    t = struct.unpack("d", b[16:24])[0]
    a = np.frombuffer(b[24:], dtype=np.float64)
    N = n0 * n1 * n2
    rho = a[:N].reshape(n2, n1, n0)
    rhou = a[N:N * (1 + nd)].reshape(nd, n2, n1, n0)
    E = a[N * (1 + nd):N * (2 + nd)].reshape(n2, n1, n0)
    return nd, t, rho, rhou, E


def sod_oracle():
    o = Oracle(1, [1024], gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 2)
    prim = setups.shock_tube(setups.Grid.from_domain(o))
    rho, rhou, E, fx = o.init_from_prim(*prim)
    t, it, st, _ = o.run(rho, rhou, E, fx, cfl=0.4, t_end=0.2, max_iter=100000, time_frequency=0.1)
    return t, it, rho, rhou, E


def test_driver_runs_reference_ini_bitwise(tmp_path):
    assert DRIVER.exists(), "driver not built"
    ini = tmp_path / "shock_tube.ini"
    ini.write_text(SOD_INI)
    dump = tmp_path / "out.bin"
    res = subprocess.run([str(DRIVER), str(ini), "--setup=shock_tube", f"--output={dump}"], capture_output=True,
                         text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    assert "Mean performance:" in res.stdout and "Mcell-updates/s" in res.stdout
    nd, t, rho, rhou, E = read_dump(dump)
    t_o, it_o, rho_o, rhou_o, E_o = sod_oracle()
    assert nd == 1 and t == t_o == 0.2
    assert f"number of iterations = {it_o}" in res.stdout
    assert np.array_equal(rho, rho_o) and np.array_equal(rhou, rhou_o) and np.array_equal(E, E_o)


def test_driver_rejects_unknown_keys(tmp_path):
    ini = tmp_path / "bad.ini"
    ini.write_text(SOD_INI.replace("riemann_solver = HLLC", "riemann_solver = Roe"))
    res = subprocess.run([str(DRIVER), str(ini)], capture_output=True, text=True, timeout=60)
    assert res.returncode != 0
    assert "Invalid riemann solver: Roe." in res.stderr
    ini.write_text(SOD_INI.replace("gamma = 1.4", "gamma = 1.0"))
    res = subprocess.run([str(DRIVER), str(ini)], capture_output=True, text=True, timeout=60)
    assert res.returncode != 0 and "Invalid gamma" in res.stderr


def test_driver_runs_passive_scalars_and_pressure_fix(tmp_path):
    """[Passive Scalar] nfx and [Pressure fix] On (both carried by the fused
    FP64 tile kernel): the driver's result equals the oracle's main loop bit
    for bit."""
    ini = tmp_path / "sod_pf.ini"
    ini.write_text(SOD_INI + "\n[Passive Scalar]\nnfx = 1\n\n[Pressure fix]\npressure_fix = On\neps_pf = 4\n")
    dump = tmp_path / "out.bin"
    res = subprocess.run([str(DRIVER), str(ini), "--setup=shock_tube", f"--output={dump}"], capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    nd, t, rho, rhou, E = read_dump(dump)
    o = Oracle(1, [1024], nfx=1, gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 2)
    prim = setups.shock_tube(setups.Grid.from_domain(o))
    r, m, e, fx = o.init_from_prim(*prim)
    r2, m2, e2, fx2 = (a.copy() for a in (r, m, e, fx))
    t_o, it_o, st_o, _ = o.run(r, m, e, fx, cfl=0.4, t_end=0.2, max_iter=100000, time_frequency=0.1,
                               pressure_fix=True, eps_pf=4.0)
    assert st_o == 0 and t == t_o == 0.2
    assert f"number of iterations = {it_o}" in res.stdout
    assert np.array_equal(rho, r) and np.array_equal(rhou, m) and np.array_equal(E, e)
    # the fix acts on this flow (eps_pf = 4: the post-shock and rarefaction
    # cells have internal energy below 4x their kinetic energy)
    o.run(r2, m2, e2, fx2, cfl=0.4, t_end=0.2, max_iter=100000, time_frequency=0.1)
    assert not np.array_equal(e2, e)


def test_driver_writes_outputs_at_the_reference_cadence(tmp_path):
    """--output-dir: an output at the start, at t = 0.1 (time_frequency) and at
    t_end, with the reference's dataset set; the last one holds the oracle's
    final state (same dt clamps to the output times), and restarting from the
    middle one with the library reaches the same final state."""
    from heraclespp_b200 import Domain
    from heraclespp_b200.output import read_output

    ini = tmp_path / "shock_tube.ini"
    ini.write_text(SOD_INI)
    res = subprocess.run([str(DRIVER), str(ini), "--setup=shock_tube", f"--output-dir={tmp_path}",
                          "--prefix=shock_tube"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    outs = [read_output(tmp_path / f"shock_tube_{k:08d}.hclraw") for k in range(3)]
    assert not (tmp_path / "shock_tube_00000003.hclraw").exists()
    assert [o["current_time"] for o in outs] == [0.0, 0.1, 0.2]
    assert [o["time_output_id"] for o in outs] == [-1, 0, 1]
    assert [o["output_id"] for o in outs] == [0, 1, 2]
    t_o, it_o, rho_o, rhou_o, E_o = sod_oracle()
    assert outs[2]["iter"] == it_o
    assert np.array_equal(outs[2]["rho"][0, 0], rho_o[0, 0, 2:-2])
    assert np.array_equal(outs[2]["E"][0, 0], E_o[0, 0, 2:-2])
    assert "shock_tube_00000002.hclraw" in (tmp_path / "shock_tube.xmf").read_text()
    # restart from t = 0.1 and run to t_end
    d = Domain(1, [1024], gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 2)
    meta = d.read_restart(tmp_path / "shock_tube_00000001.hclraw")
    assert meta["current_time"] == 0.1 and meta["iter"] == outs[1]["iter"]
    r = d.run(cfl=0.4, t_end=0.2, max_iter=100000)
    assert r.t == 0.2
    rho_r = d.get_state()[0]
    # the restart goes through the primitives (main.cpp:225-246): close, not bitwise
    assert float(np.abs(rho_r[0, 0, 2:-2] - rho_o[0, 0, 2:-2]).max()) < 1e-12
    d.close()
