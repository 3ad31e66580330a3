"""Launch properties (shared-memory opt-ins, resident CTA counts) are cached
per device: the cache used by every kernel launcher computes one value per
device id, once, under concurrent callers (host-only build of the header)."""
import subprocess

from conftest import ROOT


def test_per_device_cache(tmp_path):
    exe = tmp_path / "per_device_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-pthread", "-I", str(ROOT / "heraclespp_b200" / "csrc"),
                    str(ROOT / "tests" / "per_device_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout


def test_launchers_use_per_device_cache():
    """No launcher keeps a process-wide function-static launch property."""
    import re

    csrc = ROOT / "heraclespp_b200" / "csrc"
    offenders = []
    for f in list(csrc.glob("*.cu")) + list(csrc.glob("*.cuh")):
        for n, line in enumerate(f.read_text().splitlines(), 1):
            if re.search(r"^\s*static\s+(const\s+)?int\s+\w+\s*=", line):
                offenders.append(f"{f.name}:{n}")
    assert not offenders, offenders
