"""MG-preconditioned CG on the GPU (pmg_pcg_solve) against the CPU
restatement of the reference app's outer solver (CG_solver with the class as
preconditioner), itself pinned to the reference's own run (test_oracle).

FP64: after a fixed number of iterations the iterate is within 1e-12
relative L2 of the restatement's. Mixed (float V-cycle preconditioner):
converges to 1e-10 and lands within 1e-8 of the FP64 oracle's solve.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from conftest import fine_of  # noqa: E402
from multigrid_b200 import PBELinearProblem, WORKLOADS  # noqa: E402
from multigrid_b200._lib import PmgError  # noqa: E402
from multigrid_b200.problem import setup_fine  # noqa: E402


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def pb65():
    w = WORKLOADS["pb65"]
    return w, setup_fine(w.n, w.h, w.atoms(), w.physics)


@pytest.mark.parametrize("iters", [1, 3, 8])
def test_fp64_pcg_iterates_match_restatement(golden_problem, restatement,
                                             iters):
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    fine = fine_of(g)
    xo, co, ho = restatement.pcg(base, nlev, fine, iters)
    with PBELinearProblem(base, nlev, box, "fp64") as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        res = p.pcg_solve(tol=0.0, max_iters=iters)
        x = p.potential().ravel()
    assert res.cycles == co == iters
    assert rel_l2(x, xo) <= 1e-12
    assert np.allclose(res.history, ho, rtol=1e-9, atol=0)


def test_fp64_pcg_to_tolerance_on_pb65(pb65, restatement):
    w, fine = pb65
    xo, co, _ = restatement.pcg(w.base, w.nlev, fine, 100, tol=1e-10)
    xs, cs, _ = restatement.solve(w.base, w.nlev, fine, tol=1e-10)
    with PBELinearProblem(w.base, w.nlev, w.box, "fp64") as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        res = p.pcg_solve(tol=1e-10, max_iters=100)
        x = p.potential().ravel()
    assert abs(res.cycles - co) <= 1
    assert res.relres < 1e-10
    assert res.cycles <= cs
    assert rel_l2(x, xo) <= 1e-10
    assert rel_l2(x, xs) <= 1e-9


def test_mixed_pcg_error_vs_fp64_oracle(pb65, restatement):
    w, fine = pb65
    xs, _, _ = restatement.solve(w.base, w.nlev, fine, tol=1e-10)
    with PBELinearProblem(w.base, w.nlev, w.box, "mixed") as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        res = p.pcg_solve(tol=1e-10, max_iters=100)
        x = p.potential().ravel()
    assert res.relres < 1e-10
    assert rel_l2(x, xs) <= 1e-8
    assert np.abs(x - xs).max() / np.abs(xs).max() <= 1e-8


def test_pcg_after_vcycles_and_state_errors(golden_problem):
    """PCG continues from the loaded (or already improved) iterate and
    leaves the right-hand side intact for later solves."""
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    with PBELinearProblem(base, nlev, box, "fp64") as p:
        with pytest.raises(PmgError) as e:
            p.pcg_solve()
        assert e.value.status == -7
        p.set_fine(**fine_of(g))
        p.buildmultilevelops()
        r1 = p.solve(tol=1e-4, max_cycles=50)
        r0_after = p.compute_residual_2()
        res = p.pcg_solve(tol=1e-6, max_iters=50)
        assert res.history[0] == pytest.approx(r0_after, rel=1e-12)
        # the true residual against the untouched right-hand side
        true_res = p.compute_residual_2()
        assert true_res <= 2e-6 * r0_after
        r2 = p.solve(tol=1e-3, max_cycles=50)
        assert r2.history[0] == pytest.approx(true_res, rel=1e-12)
        assert r2.relres < 1e-3
        with pytest.raises(PmgError) as e:
            p.pcg_solve(max_iters=5000)
        assert e.value.status == -1
    assert r1.cycles > 0
