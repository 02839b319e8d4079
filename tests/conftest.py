import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "dpe-mvs-fast_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def ctx():
    import dpe_b200 as D

    c = D.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def small_scene():
    import scene as S

    return S.make_scene("small", seed=1)


@pytest.fixture(scope="session")
def tiny_scene():
    import scene as S

    return S.make_scene("tiny", seed=1)
