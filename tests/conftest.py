"""Shared test setup: repository root on sys.path and the ``gpu`` marker.

``-m "not gpu"`` runs the CPU suite (oracle, host logic, C-ABI loading);
``-m gpu`` runs the parity tests on a B200 through the C ABI.
"""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and runs the CUDA library")
