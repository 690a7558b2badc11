"""Shared fixtures.  Tests marked ``gpu`` need a B200; everything else runs on
the CPU (the oracle, host logic, the C-ABI surface)."""

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    from galoisgpu_b200 import build as b

    lib = b.LIB
    if not lib.exists():
        b.build()
    from oracle import oracle as orc

    orc.build()


_ensure_built()


@pytest.fixture(scope="session")
def gft():
    import galoisgpu_b200

    return galoisgpu_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    return oracle


@pytest.fixture(scope="session")
def engine():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import galoisgpu_b200 as g

    e = g.Engine(0)
    yield e
    e.close()


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
