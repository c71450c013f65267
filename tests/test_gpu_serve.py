"""Serving runtime (pmg_server_*) and batched solves on the GPU.

The contract: a request's result does not depend on what else is in flight.
Every solve here is compared bit for bit (potential and cycle count) with
the same solve run alone through the problem handle in the server's
throughput mode; admission never holds more device memory than the budget.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from conftest import fine_of  # noqa: E402
from multigrid_b200 import PBELinearProblem, WORKLOADS  # noqa: E402
from multigrid_b200 import _lib  # noqa: E402
from multigrid_b200.problem import setup_fine  # noqa: E402
from multigrid_b200.serve import Server, batch_solve  # noqa: E402


@pytest.fixture(scope="module")
def cases(golden_kernels):
    """(base, nlev, box, fine, precision) of grids 17^3 .. 65^3."""
    import conftest
    out = []
    for name in ("problem_b2n3.npz", "problem_b4n3.npz"):
        g = conftest.load_golden(name)
        fi = fine_of(g)
        for prec in ("fp64", "mixed"):
            out.append((int(g["base"]), int(g["nlev"]), float(g["box"]), fi,
                        prec))
    w = WORKLOADS["pb65"]
    fi = setup_fine(w.n, w.h, w.atoms(), w.physics)
    for prec in ("mixed", "fp64"):
        out.append((w.base, w.nlev, w.box, fi, prec))
    return out


def solve_alone(base, nlev, box, fine, prec):
    with PBELinearProblem(base, nlev, box, prec) as p:
        p.set_throughput_mode(True)  # the server's kernel choice
        p.set_fine(**fine)
        p.buildmultilevelops()
        r = p.solve(tol=1e-10, max_cycles=100)
        return r.cycles, p.potential().ravel().copy()


@pytest.fixture(scope="module")
def alone(cases):
    return [solve_alone(*c) for c in cases]


def test_mix_equals_alone(cases, alone):
    """All requests in flight together (twice over, so problems are reused)
    give exactly the results of the solves run alone."""
    reqs = cases + cases
    outs = [np.empty(len(c[3]["f"].ravel())) for c in reqs]
    with Server(budget_bytes=8 << 30, max_inflight=16) as srv:
        for i, ((b, nl, bx, fi, pr), o) in enumerate(zip(reqs, outs)):
            srv.submit(b, nl, bx, fi, pr, out=o, tag=i)
        done = srv.drain(len(reqs))
        st = srv.stats()
    assert sorted(c.tag for c in done) == list(range(len(reqs)))
    bad = []
    for c in done:
        assert c.ok, c.message
        cyc, x = alone[c.tag % len(cases)]
        assert c.cycles == cyc
        assert c.relres < 1e-10
        if not np.array_equal(outs[c.tag], x):
            b, nl, _, _, pr = reqs[c.tag]
            bad.append((c.tag, b, nl, pr,
                        float(np.abs(outs[c.tag] - x).max())))
        assert c.t_submit <= c.t_admit <= c.t_done
    assert not bad, bad
    assert st["completed"] == len(reqs)
    # the second round reused hierarchies of the first where it could
    assert st["created_problems"] <= len(reqs)
    assert st["peak_bytes"] <= 8 << 30


def test_budget_admission_serialises(cases, alone):
    """With room for one problem at a time, requests of two shapes run one
    after another (evicting the idle problem of the other shape) and the
    held bytes never exceed the budget."""
    from multigrid_b200.molecule import level_n, levels_for
    need = []
    for b, n, _, _, pr in cases[4:6]:
        if pr == "mixed":  # the server's default hierarchy for mixed
            b, n = levels_for(level_n(b, n), max_levels=12, min_coarse=5)
        need.append(PBELinearProblem.device_bytes(b, n, pr))
    budget = max(need) + 1024
    assert sum(need) > budget
    f1 = cases[4][3]
    seq = [0, 1, 0, 1]
    outs = [np.empty(len(f1["f"].ravel())) for _ in seq]
    with Server(budget_bytes=budget, max_inflight=8) as srv:
        for i, s in enumerate(seq):
            b, n, bx, fi, pr = cases[4 + s]
            srv.submit(b, n, bx, fi, pr, out=outs[i], tag=i)
        done = srv.drain(len(seq))
        st = srv.stats()
    assert st["peak_bytes"] <= budget
    assert st["evicted_problems"] >= 2
    for c in done:
        assert c.ok, c.message
        cyc, x = alone[4 + seq[c.tag]]
        assert c.cycles == cyc
        assert np.array_equal(outs[c.tag], x)


def test_request_larger_than_budget(cases):
    b, n, bx, fi, pr = cases[0]
    with Server(budget_bytes=1024, max_inflight=2) as srv:
        srv.submit(b, n, bx, fi, pr, tag=7)
        (c,) = srv.drain(1)
    assert c.tag == 7 and c.status == _lib.PMG_ERR_BUDGET


def test_device_inputs_and_batch_order(cases, alone):
    """batch_solve returns completions in request order; device-resident
    inputs and outputs work like host ones."""
    items = []
    for (b, n, bx, fi, pr) in cases:
        dev = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).cuda()
               for k, v in fi.items()}
        out = torch.empty_like(dev["f"])
        items.append(dict(base=b, nlev=n, box=bx, fine=dev, precision=pr,
                          out=out))
    torch.cuda.synchronize()
    res = batch_solve(items, budget_bytes=8 << 30, max_inflight=8)
    for i, (c, it) in enumerate(zip(res, items)):
        assert c.ok, c.message
        assert c.tag == i
        cyc, x = alone[i]
        assert c.cycles == cyc
        assert np.array_equal(it["out"].cpu().numpy(), x)


def test_requests_from_atoms_match_problem_handle():
    """Requests carrying atoms (GPU set-up in the worker) give the results of
    PBELinearProblem.set_atoms + solve, alone and mixed with array
    requests."""
    w = WORKLOADS["pb65"]
    atoms = w.atoms()
    want = {}
    for prec in ("fp64", "mixed"):
        with PBELinearProblem(w.base, w.nlev, w.box, prec, w.physics) as p:
            p.set_throughput_mode(True)  # the server's kernel choice
            p.set_atoms(atoms)
            p.buildmultilevelops()
            r = p.solve(tol=1e-10, max_cycles=100)
            want[prec] = (r.cycles, p.potential().ravel().copy())
    fine = setup_fine(w.n, w.h, atoms, w.physics)
    outs = {}
    with Server(budget_bytes=8 << 30, max_inflight=8) as srv:
        for i, prec in enumerate(("fp64", "mixed", "fp64", "mixed")):
            outs[i] = np.empty(w.n ** 3)
            if i < 2:
                srv.submit(w.base, w.nlev, w.box, None, prec, out=outs[i],
                           tag=i, atoms=atoms, physics=w.physics)
            else:  # array requests in the same mix
                srv.submit(w.base, w.nlev, w.box, fine, prec, out=outs[i],
                           tag=i)
        done = srv.drain(4)
    for c in done:
        assert c.ok, c.message
        if c.tag < 2:
            prec = ("fp64", "mixed")[c.tag]
            assert c.cycles == want[prec][0]
            assert np.array_equal(outs[c.tag], want[prec][1])
