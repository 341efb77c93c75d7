"""Shared test setup: markers, build of the library and the oracle."""
import os
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def built_library():
    from aquarius_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def oracle_lib():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    import oracle_binding
    return oracle_binding


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
