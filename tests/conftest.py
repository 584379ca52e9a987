import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libfwb200.so")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    """The oracle libraries are built from oracle/fw_oracle.c when missing."""
    import subprocess

    need = [os.path.join(ROOT, "oracle", f) for f in ("liboracle_f32.so", "liboracle_f64.so", "liboracle_f32fma.so",
                                                          "liboracle_f32libm.so")]
    if not all(os.path.exists(p) for p in need):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    yield
