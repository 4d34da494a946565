import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
sys.set_int_max_str_digits(0)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle, build
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        build(with_reference=False)
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("reference library not built (oracle/_ref)")
    return Reference()


@pytest.fixture(scope="session")
def ff():
    import fastfib_b200
    fastfib_b200.lib()
    return fastfib_b200
