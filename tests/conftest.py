import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden_kernels():
    return load_golden("kernels_n9.npz")


@pytest.fixture(scope="session", params=["problem_b2n3.npz",
                                         "problem_b4n3.npz"])
def golden_problem(request):
    return load_golden(request.param)


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle import Restatement
    return Restatement()


def fine_of(g):
    return {k: g["fine_" + k] for k in ("oC", "oE", "oN", "uC", "f", "x0")}
