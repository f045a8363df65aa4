import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference checkout (its examples are read by a few CPU tests): $F2M_REFERENCE,
# else a sibling directory named "reference" next to this repository.
REFERENCE = os.environ.get("F2M_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: minutes of CPU time (run with F2M_SLOW_TESTS=1)")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("F2M_SLOW_TESTS"):
        return
    skip = pytest.mark.skip(reason="slow; set F2M_SLOW_TESTS=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def ctx():
    import f2m_b200
    c = f2m_b200.Context(0)
    yield c
    c.close()


def reference_file(rel):
    p = os.path.join(REFERENCE, rel)
    if not os.path.exists(p):
        pytest.skip("reference examples are not present on this machine")
    return p
