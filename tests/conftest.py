"""Shared test set-up: import paths, the `gpu` marker, in-tree builds."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "laplacians.jl_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    import build as _pkg_build  # laplacians.jl_b200/build.py
    _pkg_build.build()
    import oracle as _oracle
    _oracle.build()


@pytest.fixture(scope="session")
def gpu_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
