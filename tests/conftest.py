"""Test configuration: the `gpu` marker and the native / oracle builds."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the oracle and the native library if they are missing (they are
    normally built by __graft_entry__.build() and travel with the tree)."""
    oracle = ROOT / "oracle"
    if not (oracle / "liboracle_f64.so").exists() or not (oracle / "liboracle_f32.so").exists():
        subprocess.run(["make", "-C", str(oracle), "all"], check=True, capture_output=True)
    lib = ROOT / "virtualfluids_b200" / "libvfb200.so"
    if not lib.exists():
        from virtualfluids_b200 import build
        build.build()
    yield


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture
def cuda():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda:0")
