import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "lu2_ref_golden.npz")


# measured parity errors, printed in the terminal summary of every run
PARITY_LOG: list[tuple[str, float, float, str]] = []


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    if not PARITY_LOG:
        return
    tr = terminalreporter
    tr.write_sep("-", "parity: measured relative error of x against its bar")
    for name, err, bar, note in PARITY_LOG:
        tr.write_line("%-58s %.3e  bar %.3e  %s%s" % (name, err, bar, "ok" if err < bar else "OVER", note))


@pytest.fixture
def parity():
    """record(name, err, bar, note=''): log a measured error and assert err < bar."""

    def record(name: str, err: float, bar: float, note: str = "") -> None:
        PARITY_LOG.append((name, float(err), float(bar), ("  " + note) if note else ""))
        assert err < bar, "%s: relative error %.3e not below %.3e %s" % (name, err, bar, note)

    return record


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
