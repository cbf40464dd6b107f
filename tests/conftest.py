import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "dns-solvers_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdnslbm.so")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()  # builds liblbmoracle.so if missing
    return oracle
