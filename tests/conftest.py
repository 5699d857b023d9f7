"""pytest configuration: the ``gpu`` marker and import paths.

``-m gpu`` tests need a CUDA device and the built library; ``-m "not gpu"`` tests run on
any host (the oracle against golden fixtures, host-side logic, ABI loading).
"""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "paulistrings-rs_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
