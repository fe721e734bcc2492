"""Test configuration.

Tests marked ``gpu`` run the B200 backend on a GPU and compare it with the
CPU oracle (oracle/) or the reference's golden values; everything else runs on
the CPU (oracle against golden vectors, host logic, library symbols, stub
generation through NVRTC, which needs no GPU).
"""

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA backend)")


@pytest.fixture(autouse=True)
def _configuration_restored():
    """Every test starts from the configuration the previous one found: a
    test that changes keys (inc_mode, staged_min_size ...) cannot leak them."""
    from pyop2_b200 import configuration as cfg
    saved = dict(cfg._config)
    yield
    if cfg._config != saved:
        cfg._config.clear()
        cfg._config.update(saved)
        cfg._generation[0] += 1


@pytest.fixture(scope="session")
def backend():
    """The B200 backend, initialised once per session.  On a machine with a
    GPU a failure here is an error, not a skip: the CUDA path must run."""
    from pyop2_b200 import op2
    op2.init(backend="b200")
    return "b200"


@pytest.fixture(scope="session")
def golden_matrices():
    with open(os.path.join(GOLDEN, "matrices.json")) as f:
        return json.load(f)


def py2_shuffle(x, random_fn):
    """random.shuffle(x, random) of Python 2 (and Python 3 before 3.11): for i
    from len-1 down to 1, swap x[i] with x[int(random() * (i + 1))].  The
    reference tests shuffle their maps with a constant random function."""
    for i in reversed(range(1, len(x))):
        j = int(random_fn() * (i + 1))
        x[i], x[j] = x[j], x[i]
    return x


def reference_seed():
    """The reference tests' _seed() (test_indirect_loop.py:40-41)."""
    return 0.02041724


def rel_err(a, b):
    """Normwise relative error max|a-b| / max(max|b|, tiny)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.size == b.size, "compared arrays differ in size: %s vs %s" % (a.shape, b.shape)
    a, b = a.reshape(-1), b.reshape(-1)
    scale = max(np.abs(b).max() if b.size else 0.0, 1e-300)
    return float(np.abs(a - b).max() / scale) if a.size else 0.0
