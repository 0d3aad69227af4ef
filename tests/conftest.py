"""Test configuration: import paths and the `gpu` marker.

Tests marked `gpu` need a CUDA device and the built libqompsim.so; the rest
run on the CPU (oracle, host logic, C-ABI exports)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "compression-based-state-vector-simulator_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

os.environ.setdefault("QOMPSIM_QUIET", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")
