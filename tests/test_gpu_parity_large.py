"""Whole solves at the benchmark grids against the reference's own FP64 solve.

The reference class (oracle/_ref, the reference's PBE_pmgc_class.h and pmgc
kernels compiled from its own sources, OpenMP build) solves each problem on
the host cores; the GPU solves the same fine-level inputs:

* pb161 (161^3, 5 levels, 5000 atoms) and pb257 (257^3, 5 levels): the plain
  FP64 GPU solve must take the same number of V-cycles and be within 1e-12
  relative L2 of the reference's potential; the mixed-precision solve
  (float V-cycles inside double refinement, its deeper hierarchy) and the
  fp64-fast solve (double V-cycles in the same structure) within 1e-8
  relative L2 and 1e-8 relative max-norm, at relative residual 1e-10.
* three molecules of the batched set (97^3, 129^3 and 161^3 grids at
  0.5 A): solved together through the batched runtime from their atoms
  (set-up on the GPU), each within 1e-8 of the reference's solve of the
  host set-up of the same atoms.

The reference solve takes seconds (161^3) to about ten seconds (257^3) on
the host cores; each is run once per module.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from multigrid_b200 import PBELinearProblem, WORKLOADS  # noqa: E402
from multigrid_b200.molecule import batch_workloads  # noqa: E402
from multigrid_b200.problem import setup_fine  # noqa: E402
from multigrid_b200.serve import batch_solve  # noqa: E402
from oracle.oracle import Reference, reference_available  # noqa: E402

if not reference_available(omp=True):  # pragma: no cover
    pytest.skip("oracle/_ref (the reference built from its sources) is not "
                "built", allow_module_level=True)

TOL_FP64 = 1e-12
TOL_MIXED = 1e-8


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def reference():
    return Reference(omp=True)


@pytest.fixture(scope="module", params=["pb161", "pb257"])
def workload(request, reference):
    """(workload, fine inputs, reference potential, reference cycles)."""
    w = WORKLOADS[request.param]
    fine = setup_fine(w.n, w.h, w.atoms(), w.physics)
    x, cycles, hist = reference.solve(w.base, w.nlev, fine, tol=1e-10,
                                      max_cycles=100)
    assert hist[-1] / hist[0] < 1e-10
    return w, fine, x, cycles


def gpu_solve(w, fine, precision):
    with PBELinearProblem(w.base, w.nlev, w.box, precision, w.physics) as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        res = p.solve(tol=1e-10, max_cycles=100)
        return res, p.potential().ravel().copy(), p.nlev


def test_fp64_matches_reference_solve(workload):
    w, fine, xr, cr = workload
    res, x, nlev = gpu_solve(w, fine, "fp64")
    assert nlev == w.nlev  # the class's hierarchy
    assert res.relres < 1e-10
    assert res.cycles == cr, (w.name, res.cycles, cr)
    err = rel_l2(x, xr)
    assert err <= TOL_FP64, (w.name, err)


@pytest.mark.parametrize("precision", ["mixed", "fp64-fast"])
def test_refinement_paths_within_tolerance_of_reference_solve(workload,
                                                              precision):
    """The mixed solve and the fastest all-double solve (fp64-fast: not the
    reference's cycle) against the reference's potential."""
    w, fine, xr, _ = workload
    res, x, _ = gpu_solve(w, fine, precision)
    assert res.relres < 1e-10
    e2, em = rel_l2(x, xr), rel_max(x, xr)
    assert e2 <= TOL_MIXED and em <= TOL_MIXED, (w.name, e2, em)


def test_batched_molecules_match_reference(reference):
    """One molecule of each of the grids 97^3, 129^3 and 161^3 from the
    batched set, solved together (mixed) through the batched runtime from
    their atoms, against the reference's FP64 solve of each."""
    picked = {}
    for w in batch_workloads(96):
        if w.n in (97, 129, 161) and w.n not in picked:
            picked[w.n] = w
    assert sorted(picked) == [97, 129, 161]
    mols = [picked[n] for n in sorted(picked)]
    items, outs = [], []
    for w in mols:
        out = np.empty(w.n ** 3)
        outs.append(out)
        items.append(dict(base=w.base, nlev=w.nlev, box=w.box,
                          precision="mixed", atoms=w.atoms(),
                          physics=w.physics, out=out))
    done = batch_solve(items, budget_bytes=16 << 30)
    for c in done:
        assert c.ok, c.message
        assert c.relres < 1e-10
    for w, x in zip(mols, outs):
        fine = setup_fine(w.n, w.h, w.atoms(), w.physics)
        xr, _, _ = reference.solve(w.base, w.nlev, fine, tol=1e-10,
                                   max_cycles=100)
        e2, em = rel_l2(x, xr), rel_max(x, xr)
        assert e2 <= TOL_MIXED and em <= TOL_MIXED, (w.n, e2, em)
