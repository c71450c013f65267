"""Whole PMG solves on the GPU through the problem handle (C ABI) against
the CPU restatement and the reference's golden solves.

FP64: the potential must be within 1e-12 relative L2 of the oracle with the
same number of V-cycles; the hierarchy bit-identical to the restatement's.
Mixed precision (float V-cycles inside double refinement): within 1e-8
relative L2 of the FP64 oracle at relative residual 1e-10.
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

TOL_FP64 = 1e-12
TOL_MIXED = 1e-8


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("trilinear", [False, True])
def test_fp64_solve_matches_reference(golden_problem, trilinear):
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    sfx = "_trilin" if trilinear else ""
    with PBELinearProblem(base, nlev, box, "fp64") as p:
        p.set_fine(**fine_of(g))
        p.buildmultilevelops(trilinear=trilinear)
        res = p.solve(tol=1e-10, max_cycles=60)
        x = p.potential().ravel()
    assert res.cycles == int(g["cycles" + sfx])
    assert res.relres < 1e-10
    assert rel_l2(x, g["x" + sfx]) <= TOL_FP64


def test_hierarchy_bitexact_vs_restatement(golden_problem, restatement):
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    ho = restatement.hierarchy(base, nlev, fine_of(g))
    with PBELinearProblem(base, nlev, box, "fp64") as p:
        p.set_fine(**fine_of(g))
        p.buildmultilevelops()
        for L in range(1, nlev):
            P, A = p.get_level(L)
            assert np.array_equal(P, ho[L][0]), L
            assert np.array_equal(A, ho[L][1]), L


def test_single_vcycles_match_restatement(golden_problem, restatement):
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    with PBELinearProblem(base, nlev, box, "fp64") as p:
        p.set_fine(**fine_of(g))
        p.buildmultilevelops()
        r0 = p.compute_residual_2()
        for _ in range(3):
            p.v_cycle()
        r3 = p.compute_residual_2()
        x = p.potential().ravel()
    xo, c, hist = restatement.solve(base, nlev, fine_of(g), tol=0.0,
                                    max_cycles=3)
    assert c == 3
    assert abs(r0 / hist[0] - 1) < 1e-12
    assert abs(r3 / hist[3] - 1) < 1e-6
    assert rel_l2(x, xo) <= TOL_FP64


def test_mixed_solve_close_to_fp64(golden_problem):
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    with PBELinearProblem(base, nlev, box, "mixed") as p:
        p.set_fine(**fine_of(g))
        p.buildmultilevelops()
        res = p.solve(tol=1e-10, max_cycles=60)
        x = p.potential().ravel()
    assert res.relres < 1e-10
    assert res.cycles <= int(g["cycles"]) + 3
    assert rel_l2(x, g["x"]) <= TOL_MIXED


@pytest.fixture(scope="module")
def pb65():
    w = WORKLOADS["pb65"]
    return w, setup_fine(w.n, w.h, w.atoms(), w.physics)


def test_pb65_fp64_matches_restatement(pb65, restatement):
    w, fine = pb65
    xo, co, ho = restatement.solve(w.base, w.nlev, fine, tol=1e-10,
                                   max_cycles=60)
    with PBELinearProblem(w.base, w.nlev, w.box, "fp64") as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        res = p.solve(tol=1e-10, max_cycles=60)
        x = p.potential().ravel()
    assert res.cycles == co
    assert rel_l2(x, xo) <= TOL_FP64


def test_pb65_mixed_error_vs_fp64_oracle(pb65, restatement):
    w, fine = pb65
    xo, co, _ = restatement.solve(w.base, w.nlev, fine, tol=1e-10,
                                  max_cycles=60)
    with PBELinearProblem(w.base, w.nlev, w.box, "mixed") as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        res = p.solve(tol=1e-10, max_cycles=60)
        x = p.potential().ravel()
    assert res.relres < 1e-10
    assert rel_l2(x, xo) <= TOL_MIXED
    assert np.abs(x - xo).max() / np.abs(xo).max() <= TOL_MIXED


def test_state_errors():
    with PBELinearProblem(2, 3, 8.0, "fp64") as p:
        with pytest.raises(PmgError) as e:
            p.buildmultilevelops()
        assert e.value.status == -7
        with pytest.raises(PmgError) as e:
            p.solve()
        assert e.value.status == -7
    with PBELinearProblem(2, 3, 8.0, "mixed") as p:
        with pytest.raises(PmgError):
            p.v_cycle()


def test_nan_input_reports_divergence(golden_problem):
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    fine = fine_of(g)
    f = fine["f"].copy()
    n = base * 2 ** nlev + 1
    f[(n // 2) * n * n + (n // 2) * n + n // 2] = np.nan
    fine["f"] = f
    with PBELinearProblem(base, nlev, box, "fp64") as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        with pytest.raises(PmgError) as e:
            p.solve(tol=1e-10, max_cycles=5)
        assert e.value.status == -4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_loop_equals_host_loop(pb65, precision):
    """The one-launch solve (stop test on the GPU, while node) takes the same
    decisions as the host-driven loop (one launch + read-back per cycle, used
    under phase timing): same cycles, same residual history, same bits."""
    w, fine = pb65
    out = {}
    for mode in ("device", "host"):
        with PBELinearProblem(w.base, w.nlev, w.box, precision) as p:
            p.set_profiling(mode == "host")
            p.set_fine(**fine)
            p.buildmultilevelops()
            res = p.solve(tol=1e-10, max_cycles=60)
            out[mode] = (res, p.potential().ravel().copy())
    (rd, xd), (rh, xh) = out["device"], out["host"]
    assert rd.cycles == rh.cycles > 0
    assert np.array_equal(rd.history, rh.history)
    assert np.array_equal(xd, xh)


def test_async_solves_overlap_and_match_alone(pb65, golden_problem):
    """Solves started together on their own streams (pmg_solve_start) give
    exactly the results of the same solves run one at a time."""
    w, fine = pb65
    g = golden_problem
    cases = [(w.base, w.nlev, w.box, fine, "mixed"),
             (w.base, w.nlev, w.box, fine, "fp64"),
             (int(g["base"]), int(g["nlev"]), float(g["box"]), fine_of(g),
              "fp64"),
             (int(g["base"]), int(g["nlev"]), float(g["box"]), fine_of(g),
              "mixed")]
    alone = []
    for base, nlev, box, fi, prec in cases:
        with PBELinearProblem(base, nlev, box, prec) as p:
            p.set_fine(**fi)
            p.buildmultilevelops()
            r = p.solve(tol=1e-10, max_cycles=60)
            alone.append((r.cycles, p.potential().ravel().copy()))
    probs = [PBELinearProblem(b, n, bx, pr) for b, n, bx, _, pr in cases]
    try:
        for p, (_, _, _, fi, _) in zip(probs, cases):
            p.set_fine(**fi)
            p.buildmultilevelops()
        for p in probs:
            p.solve_start(tol=1e-10, max_cycles=60)
        results = [p.solve_finish() for p in probs]
        for p, r, (c, x) in zip(probs, results, alone):
            assert r.cycles == c
            assert np.array_equal(p.potential().ravel(), x)
            assert p.solve_done()
    finally:
        for p in probs:
            p.close()


def test_zero_cycles_and_double_start(golden_problem):
    g = golden_problem
    with PBELinearProblem(int(g["base"]), int(g["nlev"]), float(g["box"]),
                          "fp64") as p:
        p.set_fine(**fine_of(g))
        p.buildmultilevelops()
        res = p.solve(tol=1e-10, max_cycles=0)
        assert res.cycles == 0 and res.relres == 1.0
        p.solve_start(tol=1e-10, max_cycles=3)
        with pytest.raises(PmgError) as e:
            p.solve_start(tol=1e-10, max_cycles=3)
        assert e.value.status == -7
        assert p.solve_finish().cycles == 3
        with pytest.raises(PmgError):
            p.solve_finish()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reused_handle_solves_like_a_fresh_one(golden_problem, precision):
    """A second problem loaded into the same handle solves exactly like a
    fresh handle (no state of the first solve, e.g. the warm start of the
    coarsest CG, carries over)."""
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    fine = fine_of(g)
    other = dict(fine)
    other["f"] = fine["f"] * -0.5 + 0.1
    with PBELinearProblem(base, nlev, box, precision) as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        r1 = p.solve(tol=1e-10, max_cycles=60)
        x1 = p.potential().ravel().copy()
    with PBELinearProblem(base, nlev, box, precision) as p:
        p.set_fine(**other)
        p.buildmultilevelops()
        p.solve(tol=1e-10, max_cycles=60)
        p.set_fine(**fine)
        p.buildmultilevelops()
        r2 = p.solve(tol=1e-10, max_cycles=60)
        x2 = p.potential().ravel().copy()
    assert r1.cycles == r2.cycles
    assert np.array_equal(r1.history, r2.history)
    assert np.array_equal(x1, x2)


def test_host_loop_switch_gives_the_same_solve(golden_problem):
    """pmg_problem_set_host_loop: the host-driven cycles (for profilers) and
    the one-graph solve give the same bits."""
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    out = []
    for host in (False, True):
        with PBELinearProblem(base, nlev, box, "mixed") as p:
            p.set_host_loop(host)
            p.set_fine(**fine_of(g))
            p.buildmultilevelops()
            r = p.solve(tol=1e-10, max_cycles=60)
            out.append((r.cycles, p.potential().ravel().copy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_smoother_tile_edges_give_the_same_solve(pb65, precision):
    """pmg_set_autotune: the 27-point smoother's tile edge (fixed 8, 16 or
    32, the size rule, or measured) changes speed only: every choice gives
    the same cycles and the same potential, bit for bit."""
    from multigrid_b200 import _lib
    w, fine = pb65
    out = []
    try:
        for mode in (8, 16, 32, 0, 1):
            _lib.check("pmg_set_autotune", _lib.lib.pmg_set_autotune(mode))
            with PBELinearProblem(w.base, w.nlev, w.box, precision,
                                  w.physics) as p:
                p.set_fine(**fine)
                p.buildmultilevelops()
                r = p.solve(tol=1e-10, max_cycles=100)
                out.append((r.cycles, p.potential().ravel().copy()))
        assert _lib.lib.pmg_set_autotune(5) == _lib.PMG_ERR_ARG
    finally:
        _lib.lib.pmg_set_autotune(1)
    for cyc, x in out[1:]:
        assert cyc == out[0][0]
        assert np.array_equal(x, out[0][1])


def test_throughput_mode_same_solve_within_tolerance(pb65):
    """pmg_problem_set_throughput_mode: the mixed path's lowest levels in
    one CTA instead of the cluster: the same cycle count and a potential
    equal to rounding (sums in another order); FP64 is untouched."""
    w, fine = pb65
    out = {}
    for prec in ("mixed", "fp64"):
        for mode in (False, True):
            with PBELinearProblem(w.base, w.nlev, w.box, prec,
                                  w.physics) as p:
                p.set_throughput_mode(mode)
                p.set_fine(**fine)
                p.buildmultilevelops()
                r = p.solve(tol=1e-10, max_cycles=100)
                out[prec, mode] = (r.cycles, p.potential().ravel().copy())
    assert np.array_equal(out["fp64", False][1], out["fp64", True][1])
    c0, x0 = out["mixed", False]
    c1, x1 = out["mixed", True]
    assert abs(c0 - c1) <= 1
    assert np.linalg.norm(x1 - x0) <= 1e-9 * np.linalg.norm(x0)


@pytest.mark.parametrize("precision", ["mixed", "fp64-fast", "fp64"])
def test_coded_couplings_give_the_same_bits(pb65, precision):
    """The class's fine operator has two coupling values per direction, so
    the finest smoother and defect read code bytes (on the refinement paths'
    correction and on the FP64 cycle's colour-split copies of x and f); the
    solve is bit-identical to the one reading the coupling arrays (for FP64:
    the reference layout's kernels). An
    operator with more values per direction is not coded and solves the
    same with the switch on or off; so does one whose double couplings take
    a third value that rounds to a float table value (coded for the float
    passes of the mixed path, not for fp64-fast), and one whose centre
    coefficient takes a third value for some coupling code (couplings coded,
    oC read from its array)."""
    w, fine = pb65
    out = {}
    for case in ("class", "random", "ulp", "oc3"):
        f = dict(fine)
        rng = np.random.default_rng(1)
        oE = np.array(f["oE"], copy=True)
        flat = oE.reshape(-1)
        pick = rng.choice(flat.size, 50, replace=False)
        if case == "random":  # a third value in oE: no coding
            flat[pick] = flat[pick] * 1.01
        elif case == "ulp":  # a third double, the same float
            flat[pick] = np.nextafter(flat[pick], np.inf)
        elif case == "oc3":  # oC off its code's two values at a few points
            oC = np.array(f["oC"], copy=True).reshape(w.n, w.n, w.n)
            oC[w.n // 2, w.n // 2, 5:9] *= 1.0001
            f["oC"] = oC.reshape(-1)
        f["oE"] = oE
        for on in (True, False):
            with PBELinearProblem(w.base, w.nlev, w.box, precision,
                                  w.physics) as p:
                p.set_coded_couplings(on)
                p.set_fine(**f)
                p.buildmultilevelops()
                coded = p.coded_couplings()
                r = p.solve(tol=1e-10, max_cycles=100)
                out[case, on] = (coded, r.cycles, p.potential().ravel().copy())
    assert out["class", True][0] and not out["class", False][0]
    assert not out["random", True][0]
    assert out["ulp", True][0] == (precision == "mixed")
    assert out["oc3", True][0]
    for case in ("class", "random", "ulp", "oc3"):
        assert out[case, True][1] == out[case, False][1]
        assert np.array_equal(out[case, True][2], out[case, False][2])


def test_fp64_fast_solves_golden_problems(golden_problem):
    """fp64-fast (double V-cycles on the correction equation, deep
    hierarchy, coded colour-split finest level) reaches relative residual
    1e-10 and agrees with the reference's FP64 solve to the stopping
    tolerance (1e-8 relative L2: it is not the reference's cycle, so it does
    not agree to rounding)."""
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    with PBELinearProblem(base, nlev, box, "fp64-fast") as p:
        p.set_fine(**fine_of(g))
        p.buildmultilevelops()
        res = p.solve(tol=1e-10, max_cycles=60)
        x = p.potential().ravel()
    assert res.relres < 1e-10
    assert res.cycles <= int(g["cycles"]) + 3
    assert rel_l2(x, g["x"]) <= TOL_MIXED


def test_pb65_fp64_fast_vs_oracle_and_pcg(pb65, restatement):
    """pb65: fp64-fast against the FP64 oracle (1e-8 relative L2 and
    max-norm), and as the preconditioner of the outer CG."""
    w, fine = pb65
    xo, co, _ = restatement.solve(w.base, w.nlev, fine, tol=1e-10,
                                  max_cycles=60)
    with PBELinearProblem(w.base, w.nlev, w.box, "fp64-fast",
                          w.physics) as p:
        p.set_fine(**fine)
        p.buildmultilevelops()
        assert p.coded_couplings()
        res = p.solve(tol=1e-10, max_cycles=60)
        x = p.potential().ravel().copy()
        assert res.relres < 1e-10 and res.cycles <= co + 3
        assert rel_l2(x, xo) <= TOL_MIXED
        assert np.abs(x - xo).max() / np.abs(xo).max() <= TOL_MIXED
        p.set_fine(**fine)
        p.buildmultilevelops()
        pr = p.pcg_solve(tol=1e-10, max_iters=60)
        xp = p.potential().ravel()
    assert pr.relres < 1e-10
    assert rel_l2(xp, xo) <= TOL_MIXED


@pytest.mark.parametrize("throughput", [False, True])
@pytest.mark.parametrize("base,nlev", [(2, 2), (2, 3), (2, 4), (1, 5)])
def test_mixed_lowest_levels_shapes(base, nlev, throughput):
    """The mixed path runs its levels up to 17^3 in one launch (a cluster of
    CTAs, or one CTA in throughput mode). Hierarchies whose top bottom level
    is 1, 2, 3 and 4 levels up (9^3 over 5^3 ... 33^3 over a 3^3 coarsest
    level): the solve reaches 1e-10 and its potential matches the FP64
    solve's within 1e-8."""
    from multigrid_b200.molecule import Workload, level_n
    n = level_n(base, nlev)
    w = Workload("shape", base, nlev, 0.8, 12, 0.25 * 0.8 * (n - 1), 11)
    fine = setup_fine(w.n, w.h, w.atoms(), w.physics)
    out = {}
    for prec in ("fp64", "mixed"):
        with PBELinearProblem(base, nlev, w.box, prec, w.physics) as p:
            p.set_throughput_mode(throughput)
            p.set_fine(**fine)
            p.buildmultilevelops()
            r = p.solve(tol=1e-10, max_cycles=100)
            assert r.relres < 1e-10, (prec, r.cycles, r.relres)
            out[prec] = p.potential().ravel().copy()
    x0, x1 = out["fp64"], out["mixed"]
    assert np.linalg.norm(x1 - x0) <= 1e-8 * np.linalg.norm(x0)


@pytest.mark.parametrize("name", ["pb65", "pb161", "pb257"])
def test_tma_staged_smoother_gives_the_same_bits(name):
    """The mixed path's 27-point smoother with each tile staged by
    tensor-memory access (padded float levels, tile edges by size: 33^3 of
    pb65; 21^3, 41^3, 81^3 of pb161; 33^3, 65^3, 129^3 of pb257) against the
    per-point-load kernel: the same cycles and the same potential, bit for
    bit."""
    from multigrid_b200.problem import set_tma_staging
    w = WORKLOADS[name]
    fine = setup_fine(w.n, w.h, w.atoms(), w.physics)
    out = {}
    try:
        for tma in (True, False):
            set_tma_staging(tma)
            with PBELinearProblem(w.base, w.nlev, w.box, "mixed",
                                  w.physics) as p:
                p.set_fine(**fine)
                p.buildmultilevelops()
                r = p.solve(tol=1e-10, max_cycles=100)
                out[tma] = (r.cycles, p.potential().ravel().copy())
    finally:
        set_tma_staging(True)
    assert out[True][0] == out[False][0]
    assert np.array_equal(out[True][1], out[False][1])


def test_tma_stage_wait_runs_out_and_reports(pb65):
    """The staged smoother's waits are bounded: with every stage expecting
    16 bytes more than its boxes deliver (pmg_test_tma_short_delivery), each
    wait runs out, the kernel records it and returns, and the solve reports
    PMG_ERR_TIMEOUT; a new problem afterwards solves normally on the same
    context, bit for bit as before."""
    from multigrid_b200 import _lib
    w, fine = pb65

    def solve():
        with PBELinearProblem(w.base, w.nlev, w.box, "mixed",
                              w.physics) as p:
            p.set_fine(**fine)
            p.buildmultilevelops()
            r = p.solve(tol=1e-10, max_cycles=100)
            return r.cycles, p.potential().ravel().copy()

    before = solve()
    _lib.check("pmg_test_tma_short_delivery",
               _lib.lib.pmg_test_tma_short_delivery(16))
    try:
        with pytest.raises(PmgError) as e:
            solve()
        assert e.value.status == _lib.PMG_ERR_TIMEOUT
        assert b"did not arrive" in _lib.lib.pmg_last_error()
    finally:
        _lib.check("pmg_test_tma_short_delivery",
                   _lib.lib.pmg_test_tma_short_delivery(0))
    after = solve()
    assert after[0] == before[0]
    assert np.array_equal(after[1], before[1])


@pytest.mark.parametrize("precision", ["mixed", "fp64-fast", "fp64"])
@pytest.mark.parametrize("name", ["pb49", "pb65", "pb161", "pb257"])
def test_streamed_finest_pass_gives_the_same_bits(name, precision):
    """The refinement paths' finest colour passes, defect (mixed) and
    refinement residual with the level's rows streamed through shared memory
    by tensor-map boxes and bulk copies (row blocks of 8 or 4, planes in
    chunks that fill the GPU once) against the per-point-load kernels: the
    same cycles and the same potential, bit for bit. 49^3 leaves a last row
    block of 7 rows (3 for blocks of 4); 161^3 and 257^3 are the benchmark
    grids."""
    from multigrid_b200.molecule import Workload
    from multigrid_b200.problem import set_finest_streaming
    w = (Workload("pb49", 3, 4, 0.5, 300, 8.0, 5) if name == "pb49"
         else WORKLOADS[name])
    fine = setup_fine(w.n, w.h, w.atoms(), w.physics)
    out = {}
    try:
        for on in (True, False):
            set_finest_streaming(on)
            with PBELinearProblem(w.base, w.nlev, w.box, precision,
                                  w.physics) as p:
                p.set_fine(**fine)
                p.buildmultilevelops()
                assert p.coded_couplings()
                assert p.finest_streamed() == on
                r = p.solve(tol=1e-10, max_cycles=100)
                assert r.relres < 1e-10
                out[on] = (r.cycles, p.potential().ravel().copy())
    finally:
        set_finest_streaming(True)
    assert out[True][0] == out[False][0]
    assert np.array_equal(out[True][1], out[False][1])


def test_streamed_pass_wait_runs_out_and_reports(pb65):
    """The streamed finest pass's stage waits are bounded: fp64-fast (whose
    coarse smoother stages nothing, so the finest pass is the only staged
    kernel) with every stage expecting 16 bytes more than its copies
    deliver reports PMG_ERR_TIMEOUT; a new problem afterwards solves bit for
    bit as before on the same context."""
    from multigrid_b200 import _lib
    w, fine = pb65

    def solve():
        with PBELinearProblem(w.base, w.nlev, w.box, "fp64-fast",
                              w.physics) as p:
            p.set_fine(**fine)
            p.buildmultilevelops()
            r = p.solve(tol=1e-10, max_cycles=100)
            return r.cycles, p.potential().ravel().copy()

    before = solve()
    _lib.check("pmg_test_tma_short_delivery",
               _lib.lib.pmg_test_tma_short_delivery(16))
    try:
        with pytest.raises(PmgError) as e:
            solve()
        assert e.value.status == _lib.PMG_ERR_TIMEOUT
        assert b"did not arrive" in _lib.lib.pmg_last_error()
    finally:
        _lib.check("pmg_test_tma_short_delivery",
                   _lib.lib.pmg_test_tma_short_delivery(0))
    after = solve()
    assert after[0] == before[0]
    assert np.array_equal(after[1], before[1])
