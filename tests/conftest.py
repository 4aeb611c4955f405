"""Test configuration: the `gpu` marker and on-demand builds of both libraries."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    for d in ("oracle", "bitz_b200"):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, d)], check=True)


def has_gpu():
    try:
        import bitz_b200
        return bitz_b200.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
