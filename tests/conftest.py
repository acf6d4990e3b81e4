import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dirac-research_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")

for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    # The oracle and the library are built in place (both are quick, idempotent makes).
    subprocess.run(["make", "-s", "-C", ORACLE, "oracle"], check=True)
    subprocess.run(["make", "-s", "-C", PKG], check=True)


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return np.load(os.path.join(GOLDEN, name))

    return load


@pytest.fixture(scope="session")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import dirac_b200

    lib = dirac_b200.load()
    cc = lib.dgpu_device_check()
    assert cc >= 100, f"not an sm_100 device: {cc}"
    return dirac_b200
