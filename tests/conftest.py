"""Shared pytest configuration.

GPU tests are marked ``gpu`` and call the CUDA library through its C ABI; the
rest run on CPU (oracle vs golden fixtures, host logic, library symbol table).
"""

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "torch-sim_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name))
    out = {}
    for k in d.files:
        grp, _, key = k.partition("/")
        out.setdefault(grp, {})[key] = d[k]
    return out


@pytest.fixture(scope="session")
def golden():
    return {n: load_golden(f"{n}.npz") for n in ("nl", "models", "md", "fire", "math",
                                                  "thermostats", "pairforces", "npt",
                                                  "crescale")}
