import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C-ABI")


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("oracle/_ref/libcieref.so not built")
    ref = Reference(threads=4)
    yield ref
    ref.close()


@pytest.fixture(scope="session")
def golden():
    import json
    d = os.path.join(ROOT, "tests", "golden")
    return {name[:-5]: json.load(open(os.path.join(d, name))) for name in os.listdir(d) if name.endswith(".json")}
