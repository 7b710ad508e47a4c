import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "lu2_ref_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def oracle():
    from oracle.build_oracle import build_oracle
    from oracle.oracle import OracleLib

    build_oracle()
    return OracleLib()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def lib():
    from lu2_b200 import _lib

    return _lib.load()


@pytest.fixture(scope="session")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a GPU")
    from lu2_b200 import Context

    c = Context(0)
    yield c
    c.close()
