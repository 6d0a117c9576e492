import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "pandora-2.0_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: parity at the benchmark configurations' full sizes (minutes)")


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, loaded; a GPU test fails (does not skip) without a device."""
    import pandora
    pandora.load(build_if_missing=True)
    n = pandora.device_count()
    assert n > 0, "no CUDA device visible: GPU tests need a B200"
    return pandora
