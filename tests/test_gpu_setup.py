"""GPU set-up of the finest level from atoms (pmg_setup_fine_d,
pmg_problem_set_atoms) against the host set-up (pmg_setup_fine, itself pinned
to the reference's set-up).

Bit-exact for the face and centre coefficients and the charges; the
Debye-Hueckel boundary uses CUDA's exp and must agree to 1e-14 of its
largest value.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from multigrid_b200 import PBELinearProblem, WORKLOADS, _lib  # noqa: E402
from multigrid_b200.molecule import REFERENCE_PHYSICS  # noqa: E402
from multigrid_b200.problem import physics_struct, setup_fine  # noqa: E402

KEYS = ("oC", "oE", "oN", "uC", "f", "x0")


def gpu_setup(n, h, atoms, physics):
    out = {k: torch.empty(n ** 3, dtype=torch.float64, device="cuda")
           for k in KEYS}
    atoms = np.ascontiguousarray(atoms, dtype=np.float64)
    ph = physics_struct(physics)
    rc = _lib.lib.pmg_setup_fine_d(
        n, h, atoms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        len(atoms), ctypes.byref(ph),
        *[ctypes.c_void_p(out[k].data_ptr()) for k in KEYS], None)
    _lib.check("pmg_setup_fine_d", rc)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def cases():
    w = WORKLOADS["pb65"]
    yield "pb65-probe", w.n, w.h, w.atoms(), w.physics
    yield "pb65-vdw", w.n, w.h, w.atoms(), dict(REFERENCE_PHYSICS)
    rng = np.random.default_rng(5)
    n, h = 41, 0.45
    at = np.column_stack([rng.uniform(2, (n - 3) * h, (60, 3)),
                          rng.uniform(1.0, 2.2, 60), rng.normal(0, 0.5, 60)])
    # atoms on the faces (off the boundary grid points, where the
    # Debye-Hueckel term is singular): marks at the edge, and trilinear
    # corners beyond the last grid plane (skipped)
    at[0, :3] = (0.0, 1.11, 2.22)
    at[1, :3] = ((n - 1) * h, 1.23, (n - 1) * h - 0.31)
    yield "ragged", n, h, at, w.physics


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: c[0])
def test_gpu_setup_matches_host(case):
    _, n, h, atoms, physics = case
    host = setup_fine(n, h, atoms, physics)
    dev = gpu_setup(n, h, atoms, physics)
    for k in ("oC", "oE", "oN", "uC", "f"):
        assert np.array_equal(dev[k], host[k].ravel()), k
    x0h = host["x0"].ravel()
    assert np.abs(dev["x0"] - x0h).max() <= 1e-14 * np.abs(x0h).max()


def test_gpu_setup_without_atoms():
    n, h = 17, 0.5
    dev = gpu_setup(n, h, np.zeros((0, 5)), dict(REFERENCE_PHYSICS))
    host = setup_fine(n, h, np.zeros((0, 5)), dict(REFERENCE_PHYSICS))
    for k in KEYS:
        assert np.array_equal(dev[k], host[k].ravel()), k


def test_gpu_setup_rejects_atom_outside_grid():
    n, h = 17, 0.5
    atoms = np.array([[1.0, 1.0, 9.0, 1.5, 1.0]])  # 9.0 > 16 * 0.5
    with pytest.raises(_lib.PmgError) as e:
        gpu_setup(n, h, atoms, dict(REFERENCE_PHYSICS))
    assert e.value.status == _lib.PMG_ERR_ARG


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_from_atoms_matches_host_setup(precision):
    w = WORKLOADS["pb65"]
    atoms = w.atoms()
    fine = setup_fine(w.n, w.h, atoms, w.physics)
    with PBELinearProblem(w.base, w.nlev, w.box, precision, w.physics) as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        r1 = p.solve(tol=1e-10, max_cycles=60)
        x1 = p.potential().ravel().copy()
        p.set_atoms(atoms)
        p.buildmultilevelops()
        r2 = p.solve(tol=1e-10, max_cycles=60)
        x2 = p.potential().ravel().copy()
    assert abs(r1.cycles - r2.cycles) <= 1
    assert np.linalg.norm(x1 - x2) <= 1e-12 * np.linalg.norm(x1)
