"""The C++ drop-in class (include/PBE_pmgc_class_b200.h): a host program
written against the reference's PBE_linear_problem API (tests/cpp/
pbe_class_app.cc) builds with g++ against the header and the library, and on
the GPU its cycle-by-cycle loop and its solve() give the Python class's
solve bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "multigrid_b200")


def build_app(tmp_path) -> str:
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not found")
    if not os.path.exists(os.path.join(LIBDIR, "libpmg_b200.so")):
        pytest.skip("libpmg_b200.so not built")
    exe = str(tmp_path / "pbe_class_app")
    subprocess.run([gxx, "-std=c++20", "-O1", "-Wall", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "pbe_class_app.cc"),
                    "-L", LIBDIR, "-lpmg_b200", f"-Wl,-rpath,{LIBDIR}",
                    "-o", exe], check=True)
    return exe


def test_class_header_builds(tmp_path):
    assert os.path.exists(build_app(tmp_path))


@pytest.mark.gpu
def test_class_app_matches_python_class(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from multigrid_b200 import PBELinearProblem, WORKLOADS
    from multigrid_b200.molecule import REFERENCE_PHYSICS
    exe = build_app(tmp_path)
    w = WORKLOADS["pb65"]  # base 4, 4 levels, 0.5 A: the app's 65^3 problem
    assert (w.base, w.nlev, w.box) == (4, 4, 32.0)
    atoms = np.ascontiguousarray(w.atoms(), dtype=np.float64)
    (tmp_path / "atoms.bin").write_bytes(atoms.tobytes())
    out = subprocess.run([exe, str(tmp_path / "atoms.bin"),
                          str(tmp_path / "out.bin")], check=True,
                         capture_output=True, text=True)
    loop_cycles, solve_cycles, relres = out.stdout.split()
    x = np.fromfile(tmp_path / "out.bin", dtype=np.float64)
    n3 = w.n ** 3
    x_loop, x_solve = x[:n3], x[n3:]
    with PBELinearProblem(w.base, w.nlev, w.box, "fp64",
                          dict(REFERENCE_PHYSICS)) as p:
        p.set_atoms(atoms)
        p.buildmultilevelops()
        r = p.solve(tol=1e-10, max_cycles=100)
        want = p.potential().ravel()
    assert int(loop_cycles) == int(solve_cycles) == r.cycles
    assert float(relres) < 1e-10
    assert np.array_equal(x_solve, want)
    assert np.array_equal(x_loop, want)
