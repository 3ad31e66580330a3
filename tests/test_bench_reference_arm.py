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


def test_clock_summary_keeps_the_timed_window():
    """The clock record keeps the samples taken inside the timed region, or
    the nearest one on each side of a region shorter than the sampling
    period, and unions the throttle reasons seen there."""
    sys.path.insert(0, str(ROOT))
    import bench

    c = bench.ClockSampler(0)
    c.source = "test"
    c.samples = [(0.0, 1000.0, 1965.0, 300.0, set()), (1.0, 1965.0, 1965.0, 900.0, {"sw_power_cap"}),
                 (1.5, 1950.0, 1965.0, 950.0, set()), (3.0, 800.0, 1965.0, 200.0, {"hw_slowdown"})]
    c.window(0.9, 1.6)
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    c.window(1.6, 1.7)  # no sample inside: the neighbours on both sides
    s = c.summary()
    assert s["samples"] == 2 and s["reasons"] == ["hw_slowdown"] and s["sm_mhz"] == 1375.0
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]
