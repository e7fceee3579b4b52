"""Shared test setup: import paths, the `gpu` marker and fixtures.

CPU tests (-m "not gpu") cover the oracle against the reference's known answers, the
host logic and the C ABI surface.  GPU tests (-m gpu) call the CUDA library through its
C ABI and compare it with the oracle on the same inputs.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "machinig-sim_b200"
GOLDEN = ROOT / "tests" / "golden"
for p in (str(PKG), str(ROOT / "oracle"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmcs.so")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle

    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def mcs_lib():
    """libmcs.so, built in-tree if needed (nvcc cross-compiles without a GPU)."""
    sys.path.insert(0, str(PKG))
    import build as mcs_build  # machinig-sim_b200/build.py

    mcs_build.build()
    from mcs import _lib

    return _lib.load()


@pytest.fixture(scope="session")
def ctx(mcs_lib):
    """A context on cuda:0; GPU tests fail (not skip) when the device is missing."""
    from mcs import Context

    c = Context(0)
    yield c
    c.close()


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}
