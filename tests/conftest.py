"""Shared fixtures.  `-m gpu` tests need a CUDA device and libppb.so; the
rest run on CPU.  The oracle (oracle/) is imported here only as the checker."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "peakpatch.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libppb.so")


@pytest.fixture(scope="session")
def ora():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def fortran_table(ora):
    return ora.read_homeltab(os.path.join(GOLDEN, "HomelTab_fortran.dat"))


@pytest.fixture(scope="session")
def julia_table(ora):
    return ora.read_homeltab(os.path.join(GOLDEN, "HomelTab_julia.dat"))


@pytest.fixture(scope="session")
def eh_pk():
    from peakpatch_b200 import powerspec
    return powerspec.eh_table()


def filter_bank(n_filters=20, rmin=1.5, rmax=30.0):
    """Top-hat bank Rf = 1.5 * 20^((i-1)/19) Mpc/h (log-spaced 1.5..30)."""
    i = np.arange(n_filters)
    return [(int(k) + 1, 1.686, float(rmin * (rmax / rmin) ** (k / (n_filters - 1)))) for k in i]


@pytest.fixture(scope="session")
def ctx():
    """GPU context (gpu tests only)."""
    from peakpatch_b200 import Context
    c = Context(0)
    yield c
    c.close()
