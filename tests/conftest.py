import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "rod-dynamics-3d_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds librodgpu.so / librodhost.so and the oracle once per session."""
    import build as pkg_build  # rod-dynamics-3d_b200/build.py
    pkg_build.build()
    import oracle
    oracle.build(ref=os.path.isdir(oracle.REF_TREE))
    yield
