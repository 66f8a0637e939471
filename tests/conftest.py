"""Shared test set-up: the `gpu` marker, import paths and the CUDA library."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (str(ROOT), str(ROOT / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def fm_lib():
    """The product library, built in-tree if it is missing (fails loudly otherwise)."""
    import fumeng_b200
    from fumeng_b200 import build
    if not fumeng_b200.LIB_PATH.exists():
        build.build()
    return fumeng_b200.load_library()


@pytest.fixture(scope="session")
def ctx(fm_lib):
    import fumeng_b200
    c = fumeng_b200.Context(0)
    yield c
    c.close()
