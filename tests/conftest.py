import glob
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "extended-rabitq_b200")
ORACLE_DIR = os.path.join(REPO, "oracle")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, ORACLE_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls liberq.so kernels")


def golden_cases():
    return sorted(os.path.basename(p)[:-6] for p in glob.glob(os.path.join(GOLDEN, "*.index")))


def load_golden(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    g["path"] = os.path.join(GOLDEN, name + ".index")
    return g


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build_oracle()
    return oracle
