"""bench.py's own arm on one GPU, with the optional sections off: one JSON
line carrying the keys the harness reads (metric, value, e2e with its
host-device bytes, the roofline of the step kernel against the measured HBM
peak, the kernel launch count, the clocks, the mixed-vs-FP64 accuracy)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_bench_json_line():
    cmd = [sys.executable, str(ROOT / "bench.py"), "--steps", "5", "--warmup", "3", "--e2e-chunk", "5",
           "--no-cpu-baseline", "--no-adjoint", "--no-ensemble", "--no-rt3d", "--no-stage-loop"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-3000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["metric"] == "Mcell-updates/s" and d["unit"] == "Mcell-updates/s" and d["n_gpus"] == 1
    assert d["steps"] == 5 and d["warmup"] == 3 and d["higher_is_better"] is True and d["scaling"] == "weak"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("kelvin_helmholtz_2d_2048x2048")
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["bytes_per_cell"] == 64
    assert 0 < r["frac"] < 1.5 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9
    assert r["traffic"] is None or r["traffic"] > 0
    assert d["gpu_launches"] >= 5
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
    acc = d["accuracy"]
    assert acc["steps_compared"] == 1000
    assert set(acc["fields"]) == {"rho", "rhou_0", "rhou_1", "E"}
    # the density bar (1e-6 relative L1) after the workload's 1000 steps
    assert acc["fields"]["rho"]["rel_l1"] < 1e-6
    for name, e in acc["fields"].items():
        assert e["rel_l1"] >= 0 and e["rel_linf"] >= 0, name
    assert d["e2e_state_copied_every_step"]["value"] > 0
