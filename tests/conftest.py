"""Shared test setup: the `gpu` marker, the oracles and small helpers.

`-m "not gpu"` tests run on a host without a GPU (oracle vs golden vectors,
host logic, ABI symbol checks); `-m gpu` tests are the parity tests proper and
call the CUDA path through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import PortOracle

    return PortOracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import RefOracle

    return RefOracle()


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return int(d["n"]), d["records"], d["offsets"], int(d["basis"]), d["amplitudes"]
