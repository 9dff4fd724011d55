"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def gpu_ctx():
    import gat_b200 as G

    ctx = G.Context(0)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def host_ctx():
    import gat_b200 as G

    ctx = G.Context(-1)
    yield ctx
    ctx.close()


def csr_equal(off_a, val_a, off_b, val_b):
    return np.array_equal(np.asarray(off_a, np.int64), np.asarray(off_b, np.int64)) and np.array_equal(
        np.asarray(val_a, np.int64), np.asarray(val_b, np.int64))
