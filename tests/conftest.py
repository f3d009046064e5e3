import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracles (built here from the reference's sources, or prebuilt where they are absent)."""
    from oracle import oracle as O
    need = [os.path.join(O.HERE, "liboracle.so"), os.path.join(O.HERE, "_ref", "libref_f.so")]
    if not all(os.path.exists(p) for p in need):
        O.build()
    return O


@pytest.fixture(scope="session")
def ctx():
    import little_renderer_b200 as L
    return L.Context(0)
