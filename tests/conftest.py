import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads")


def pytest_collection_modifyitems(config, items):
    # Collect test files in name order, so tests/test_zz_* run last.
    items.sort(key=lambda it: (Path(str(it.fspath)).name, 0))


@pytest.fixture(scope="session")
def port():
    import oracle
    return oracle.Port()


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.REF_SO.exists():
        pytest.skip("reference build (oracle/_ref) not present")
    return oracle.Reference()


@pytest.fixture(scope="session")
def ctx():
    import dnaln_b200 as D
    c = D.Context(int(os.environ.get("DNALN_TEST_DEVICE", "0")))
    yield c
    c.close()
