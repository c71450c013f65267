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


@pytest.fixture(scope="session")
def golden_box():
    return load_golden("buildA_fv.npz")


@pytest.fixture(scope="session")
def golden_band():
    return load_golden("band.npz")


def box_case(g, tag):
    """One VbuildA_fv case of buildA_fv.npz: sizes, ipkey, the input maps,
    the pre-filled output arrays and the reference's outputs."""
    nx, ny, nz = (int(g[f"{tag}_{k}"]) for k in ("nx", "ny", "nz"))
    inputs = {k: np.ascontiguousarray(g[f"{tag}_{k}"])
              for k in ("xf", "yf", "zf", "gxcf", "gycf", "gzcf", "a1cf",
                        "a2cf", "a3cf", "ccf", "fcf")}
    return dict(n=(nx, ny, nz), ipkey=int(g[f"{tag}_ipkey"]), inputs=inputs,
                init=g[f"{tag}_init"], out=g[f"{tag}_out"],
                ipc=g[f"{tag}_ipc"], numdia=int(g[f"{tag}_numdia"]))


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
