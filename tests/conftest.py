"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on a CPU-only host."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference's own host path, when it has been built here (oracle/_ref)."""
    from oracle.bindings import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libref.so not built (needs the reference tree)")
    return Reference()


@pytest.fixture(scope="session")
def pitzdaily():
    import numpy as np
    return dict(np.load(os.path.join(REPO, "tests", "golden", "pitzdaily.npz")))


@pytest.fixture(scope="session")
def case20():
    import numpy as np
    return dict(np.load(os.path.join(REPO, "tests", "golden", "case20.npz")))
