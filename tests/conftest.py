"""Test setup: the package `rang` (rang-core_b200/) and the CPU oracle
(oracle/) on the path, and the `gpu` marker for tests that need a B200."""

import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]
for p in (REPO / "rang-core_b200", REPO / "oracle", REPO / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
