"""The benchmark's reference arm (bench.py --impl reference) runs on the host
cores alone and prints one JSON line with the keys the harness reads: the
metric and unit of the GPU arm, impl "reference", the CPU baseline that was
timed and an end-to-end entry with no host-device traffic."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
                          "--cpu-budget", "0.3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Mcell-updates/s" and d["unit"] == "Mcell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["n_gpus"] == 1
    assert d["config"]["workload"].startswith("kelvin_helmholtz_2d_2048x2048")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
