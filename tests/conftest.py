"""Shared pytest setup: import paths for the package and the CPU oracle, and
the `gpu` marker (tests that need a CUDA device)."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "old-gpuintegration_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def cub():
    import cubature

    cubature.load_library()
    return cubature


@pytest.fixture(scope="session")
def ctx(cub):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = cub.Context(0)
    yield c
    c.close()
