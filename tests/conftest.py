"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and the built product library; the
rest run on CPU (oracle pins, host-side logic, C-ABI exports, gloo ranks).
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built sm_100a library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import build_oracle, oracle_lib_path

    if not oracle_lib_path().exists():
        build_oracle(ref=False)
    return True


@pytest.fixture(scope="session")
def ref_cell_available():
    p = ROOT / "oracle" / "_ref" / "libref_cell_2d.so"
    if not p.exists():
        from oracle import build_oracle

        build_oracle(ref=True)  # a no-op for the reference part when its sources are absent
    if not p.exists():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    return True
