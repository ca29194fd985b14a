import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

# the reference checkout: $SLM_REFERENCE, else a "reference" folder beside the repository
REFERENCE = os.environ.get("SLM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) and libslm_b200.so")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly (no skip) when run with -m gpu on a host without a
    # device; without -m gpu they are simply deselected by the marker filter.
    pass


@pytest.fixture(scope="session")
def reference_dir():
    if not os.path.isdir(os.path.join(REFERENCE, "python", "streamlines")):
        pytest.skip("reference checkout not present on this host")
    return REFERENCE
