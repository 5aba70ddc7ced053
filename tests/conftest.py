"""Shared test setup: import paths, the `gpu` marker, and in-tree builds.

CPU tests (-m "not gpu") cover the oracle against the reference's known-answer
cases and the committed fixtures, the synthetic generator, the host logic and
the C ABI's exported symbols. GPU tests (-m gpu) call the CUDA path through the
C ABI and compare with the oracle bit for bit.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "rivet-av1_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _make(target_dir):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, target_dir)], check=True)


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Builds the oracle and the package in-tree if they are missing or stale
    (a no-op when `__graft_entry__.build()` already ran)."""
    _make("oracle")
    _make("rivet-av1_b200") if os.listdir(os.path.join(ROOT, "rivet-av1_b200", "csrc")) and any(f.endswith(".cu") for f in os.listdir(os.path.join(ROOT, "rivet-av1_b200", "csrc"))) else None
    yield


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
