"""Shared test setup: import paths for the host package and the oracle, and
the `gpu` marker (tests that need a B200; everything else runs on CPU)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (os.path.join(ROOT, "powder-play_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libmpm_b200.so")
