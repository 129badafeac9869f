import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def pkg():
    return ge.load_package()


@pytest.fixture(scope="session")
def orc():
    o = ge.load_oracle()
    o.build()
    return o


@pytest.fixture(scope="session")
def cuda():
    """Initialises CUDA on device 0.  GPU tests do not fall back to anything:
    a missing library or device is an error on a GPU machine."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device in this environment")
    torch.cuda.set_device(0)
    pk = ge.load_package()
    pk.colsolve.lib()  # raises if libtg_colsolve.so is missing
    return torch


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def prec_fn(f, lf):
    """A transcendental function for the numpy transcriptions: on float64
    values the C library's (through math, as the oracle calls it), on long
    double values numpy's long double ufunc, so a transcription fed long
    double inputs evaluates the same formulas to ~1e-19."""
    vf = np.vectorize(f, otypes=[float])

    def g(*args):
        if any(np.asarray(a).dtype == np.longdouble for a in args):
            return lf(*args)
        return vf(*args)
    return g
