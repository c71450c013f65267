"""CUDA kernels against the CPU restatement and the reference's golden
outputs, through the C ABI (multigrid_b200.pmgc -> libpmg_b200.so).

Double-precision kernels keep the reference's per-point operation order and
are built with --fmad=false: smoothers, matvec, residual and transfers must
match the reference bit for bit; the builders must match the restatement
bit for bit (same loops) and the reference to 1e-13 of the array's maximum.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from multigrid_b200 import pmgc  # noqa: E402

DEV = torch.device("cuda:0")


def T(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def H(t):
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def rand_case(n, seed):
    rng = np.random.default_rng(seed)
    op27 = [rng.uniform(0.5, 2.0, n ** 3) for _ in range(14)]
    op27[0] = rng.uniform(28.0, 40.0, n ** 3)
    op7 = [rng.uniform(20.0, 30.0, n ** 3)] + [rng.uniform(0.5, 2.0, n ** 3)
                                              for _ in range(3)]
    return dict(op27=op27, op7=op7, cc=rng.uniform(0.0, 0.5, n ** 3),
                f=rng.normal(size=n ** 3), x0=rng.normal(size=n ** 3),
                rng=rng)


@pytest.mark.parametrize("iad,zi", [(0, 0), (1, 0), (0, 1)])
def test_gs7_matches_reference(golden_kernels, iad, zi):
    g = golden_kernels
    n = int(g["nf"])
    op7 = g["op7"]
    x = T(g["x0"])
    pmgc.Vgsrb7x(n, n, n, T(op7[0]), T(g["cc"]), T(g["f"]), T(op7[1]),
                 T(op7[2]), T(op7[3]), x, itmax=2, iadjoint=iad,
                 zero_init=zi)
    name = f"a{iad}z{zi}"
    assert np.array_equal(H(x), g["gs7_" + name])


@pytest.mark.parametrize("iad,zi", [(0, 0), (1, 0), (0, 1)])
def test_gs27_matches_reference(golden_kernels, iad, zi):
    g = golden_kernels
    n = int(g["nf"])
    x = T(g["x0"])
    pmgc.Vgsrb27x(n, n, n, [T(a) for a in g["op27"]], T(g["cc"]), T(g["f"]),
                  x, itmax=2, zero_init=zi, iadjoint=iad)
    assert np.array_equal(H(x), g[f"gs27_a{iad}z{zi}"])


def test_matvec_mresid_match_reference(golden_kernels):
    g = golden_kernels
    n = int(g["nf"])
    op7 = [T(a) for a in g["op7"]]
    op27 = [T(a) for a in g["op27"]]
    cc, f, x = T(g["cc"]), T(g["f"]), T(g["x0"])
    y = torch.zeros(n ** 3, dtype=torch.float64, device=DEV)
    pmgc.Vmatvec7_1s(n, n, n, op7[0], cc, op7[1], op7[2], op7[3], x, y)
    assert np.array_equal(H(y), g["matvec7"])
    y.zero_()
    pmgc.Vmatvec27_1s(n, n, n, op27, cc, x, y)
    assert np.array_equal(H(y), g["matvec27"])
    y.zero_()
    pmgc.Vmresid7_1s(n, n, n, op7[0], cc, f, op7[1], op7[2], op7[3], x, y)
    assert np.array_equal(H(y), g["mresid7"])
    y.zero_()
    pmgc.Vmresid27_1s(n, n, n, op27, cc, f, x, y)
    assert np.array_equal(H(y), g["mresid27"])


def test_transfers_match_reference(golden_kernels):
    g = golden_kernels
    nf, nc = int(g["nf"]), int(g["nc"])
    P = [T(a) for a in g["P_rand"]]
    e = torch.zeros(nf ** 3, dtype=torch.float64, device=DEV)
    pmgc.VinterpPMG2(nc, nc, nc, nf, nf, nf, T(g["xc"]), e, P)
    assert np.array_equal(H(e), g["interp"])
    r = torch.zeros(nc ** 3, dtype=torch.float64, device=DEV)
    pmgc.Vrestrc2(nf, nf, nf, nc, nc, nc, T(g["x0"]), r, P)
    assert np.array_equal(H(r), g["restrict"])


def test_builders_match_reference(golden_kernels):
    g = golden_kernels
    nf, nc = int(g["nf"]), int(g["nc"])
    op7 = [T(a) for a in g["op7"]]
    op27 = [T(a) for a in g["op27"]]
    P = [torch.zeros(nc ** 3, dtype=torch.float64, device=DEV)
         for _ in range(27)]
    pmgc.VbuildPb_op7(nf, nf, nf, nc, nc, nc, *op7, P)
    assert rel(np.stack([H(t) for t in P]), g["P_op7"]) <= 1e-13
    pmgc.VbuildPb_op27(nf, nf, nf, nc, nc, nc, op27, P)
    got = np.stack([H(t) for t in P])
    for s in range(27):
        assert rel(got[s], g["P_op27"][s]) <= 1e-13, s
    pmgc.VbuildPb_trilin(nf, nf, nf, nc, nc, nc, P)
    assert np.array_equal(np.stack([H(t) for t in P]), g["P_trilin"])
    Pr = [T(a) for a in g["P_rand"]]
    out = [torch.zeros(nc ** 3, dtype=torch.float64, device=DEV)
           for _ in range(14)]
    pmgc.VbuildG_7(nf, nf, nf, nc, nc, nc, Pr, *op7, out)
    for s in range(14):
        assert rel(H(out[s]), g["G7"][s]) <= 1e-13, s
    pmgc.VbuildG_27(nf, nf, nf, nc, nc, nc, Pr, op27, out)
    for s in range(14):
        assert rel(H(out[s]), g["G27"][s]) <= 1e-13, s


@pytest.mark.parametrize("nf", [17, 33])
def test_builders_bitexact_vs_restatement(restatement, nf):
    nc = (nf - 1) // 2 + 1
    c = rand_case(nf, nf)
    P = [torch.zeros(nc ** 3, dtype=torch.float64, device=DEV)
         for _ in range(27)]
    Po = [np.zeros(nc ** 3) for _ in range(27)]
    for kind in (7, 27):
        ops = c["op7"] if kind == 7 else c["op27"]
        if kind == 7:
            pmgc.VbuildPb_op7(nf, nf, nf, nc, nc, nc, *[T(a) for a in ops], P)
        else:
            pmgc.VbuildPb_op27(nf, nf, nf, nc, nc, nc, [T(a) for a in ops], P)
        restatement.buildP_op(nf, nc, ops, Po)
        for s in range(27):
            assert np.array_equal(H(P[s]), Po[s]), (kind, s)
        Pr = [c["rng"].uniform(0.05, 1.0, nc ** 3) for _ in range(27)]
        out = [torch.zeros(nc ** 3, dtype=torch.float64, device=DEV)
               for _ in range(14)]
        oo = [np.zeros(nc ** 3) for _ in range(14)]
        if kind == 7:
            pmgc.VbuildG_7(nf, nf, nf, nc, nc, nc, [T(a) for a in Pr],
                           *[T(a) for a in ops], out)
        else:
            pmgc.VbuildG_27(nf, nf, nf, nc, nc, nc, [T(a) for a in Pr],
                            [T(a) for a in ops], out)
        restatement.buildG(nf, nc, Pr, ops, oo)
        for s in range(14):
            assert np.array_equal(H(out[s]), oo[s]), (kind, s)


@pytest.mark.parametrize("n", [17, 33, 65, 97])
def test_smoothers_bitexact_large(restatement, n):
    c = rand_case(n, 100 + n)
    for iad, zi in ((0, 0), (1, 1)):
        x = T(c["x0"])
        xo = c["x0"].copy()
        o = c["op7"]
        pmgc.Vgsrb7x(n, n, n, T(o[0]), None, T(c["f"]), T(o[1]), T(o[2]),
                     T(o[3]), x, itmax=3, iadjoint=iad, zero_init=zi)
        restatement.gsrb7x(n, o[0], np.zeros(n ** 3), c["f"], o[1], o[2],
                           o[3], xo, itmax=3, iadjoint=iad, zero_init=zi)
        assert np.array_equal(H(x), xo)
        x = T(c["x0"])
        xo = c["x0"].copy()
        pmgc.Vgsrb27x(n, n, n, [T(a) for a in c["op27"]], None, T(c["f"]), x,
                      itmax=2, zero_init=zi, iadjoint=iad)
        restatement.gsrb27x(n, c["op27"], np.zeros(n ** 3), c["f"], xo,
                            itmax=2, iadjoint=iad, zero_init=zi)
        assert np.array_equal(H(x), xo)


def test_float_smoothers_track_double():
    n = 33
    c = rand_case(n, 7)
    o = c["op7"]
    xd = T(c["x0"])
    xf = T(c["x0"], torch.float32)
    pmgc.Vgsrb7x(n, n, n, T(o[0]), None, T(c["f"]), T(o[1]), T(o[2]),
                 T(o[3]), xd, itmax=2)
    pmgc.Vgsrb7x(n, n, n, *[T(a, torch.float32) for a in (o[0],)], None,
                 T(c["f"], torch.float32),
                 *[T(a, torch.float32) for a in o[1:]], xf, itmax=2)
    assert rel(H(xf), H(xd)) < 1e-5
    xd = T(c["x0"])
    xf = T(c["x0"], torch.float32)
    pmgc.Vgsrb27x(n, n, n, [T(a) for a in c["op27"]], None, T(c["f"]), xd, 2)
    pmgc.Vgsrb27x(n, n, n, [T(a, torch.float32) for a in c["op27"]], None,
                  T(c["f"], torch.float32), xf, 2)
    assert rel(H(xf), H(xd)) < 1e-5


def test_float_kernels_track_double():
    """The _f matvec, residual and transfer entry points against the _d ones
    on the same float-rounded inputs: only the arithmetic's precision
    differs, so each result agrees to 1e-5 of its maximum."""
    nf, nc = 33, 17
    c = rand_case(nf, 11)
    r32 = [np.float32(a).astype(np.float64)
           for a in c["op7"] + c["op27"] + [c["cc"], c["f"], c["x0"]]]
    o7d, o27d = r32[:4], r32[4:18]
    cc, f, x = r32[18:]

    def both(call, n_out):
        got = []
        for dt in (torch.float64, torch.float32):
            y = torch.zeros(n_out, dtype=dt, device=DEV)
            call(lambda a: T(a, dt), y)
            got.append(H(y))
        assert np.abs(got[0]).max() > 0
        assert rel(got[1], got[0]) < 1e-5
        return got

    both(lambda t, y: pmgc.Vmatvec7_1s(nf, nf, nf, t(o7d[0]), t(cc),
                                       t(o7d[1]), t(o7d[2]), t(o7d[3]),
                                       t(x), y), nf ** 3)
    both(lambda t, y: pmgc.Vmatvec27_1s(nf, nf, nf, [t(a) for a in o27d],
                                        t(cc), t(x), y), nf ** 3)
    both(lambda t, y: pmgc.Vmresid7_1s(nf, nf, nf, t(o7d[0]), t(cc), t(f),
                                       t(o7d[1]), t(o7d[2]), t(o7d[3]),
                                       t(x), y), nf ** 3)
    both(lambda t, y: pmgc.Vmresid27_1s(nf, nf, nf, [t(a) for a in o27d],
                                        t(cc), t(f), t(x), y), nf ** 3)
    P = [np.float32(c["rng"].uniform(0.05, 1.0, nc ** 3)).astype(np.float64)
         for _ in range(27)]
    xc = np.float32(c["rng"].normal(size=nc ** 3)).astype(np.float64)
    both(lambda t, y: pmgc.Vrestrc2(nf, nf, nf, nc, nc, nc, t(x), y,
                                    [t(a) for a in P]), nc ** 3)
    both(lambda t, y: pmgc.VinterpPMG2(nc, nc, nc, nf, nf, nf, t(xc), y,
                                       [t(a) for a in P]), nf ** 3)


def _box_gpu(c):
    """Runs pmg_VbuildA_fv_d on a box_case-style dict; returns the six
    outputs (oC cc fc oE oN uC) and the host bookkeeping."""
    out = [T(a) for a in c["init"]]
    inp = [T(c["inputs"][k]) for k in ("xf", "yf", "zf", "gxcf", "gycf",
                                       "gzcf", "a1cf", "a2cf", "a3cf", "ccf",
                                       "fcf")]
    ipc, numdia = pmgc.VbuildA_fv(*c["n"], c["ipkey"], *out, *inp)
    return np.stack([H(t) for t in out]), ipc, numdia


@pytest.mark.parametrize("tag", ["c9", "r11"])
def test_box_builder_matches_reference(golden_box, tag):
    """VbuildA_fv (pmgc/buildAd.cc:63-212) bit for bit against the
    reference's outputs; the shell keeps the caller's values."""
    from conftest import box_case
    c = box_case(golden_box, tag)
    got, ipc, numdia = _box_gpu(c)
    assert np.array_equal(got, c["out"])
    assert ipc == list(c["ipc"]) and numdia == c["numdia"]


@pytest.mark.parametrize("n", [(33, 33, 33), (65, 49, 40)])
def test_box_builder_bitexact_vs_restatement(restatement, n):
    from tests.golden.make_golden import box_inputs
    c = box_inputs(np.random.default_rng(sum(n)), *n)
    want = [np.ascontiguousarray(a) for a in c["init"].copy()]
    restatement.buildA_fv(*n, 2, c, want)
    got, _, _ = _box_gpu(dict(n=n, ipkey=2, inputs=c, init=c["init"]))
    assert np.array_equal(got, np.stack(want))


def test_packed_matvec_mresid_match_reference(golden_kernels):
    """Vmatvec / Vmresid with the operator packed as APBS keeps it
    (matvecd.cc:244-260, 513-529), dispatched on ipc[10]."""
    g = golden_kernels
    n = int(g["nf"])
    cc, f, x = T(g["cc"]), T(g["f"]), T(g["x0"])
    for key, ac in (("7", T(g["op7"])), ("27", T(g["op27"]))):
        y = torch.zeros(n ** 3, dtype=torch.float64, device=DEV)
        pmgc.Vmatvec(n, n, n, ac, cc, x, y)
        assert np.array_equal(H(y), g["matvec" + key])
        y.zero_()
        pmgc.Vmresid(n, n, n, ac, cc, f, x, y)
        assert np.array_equal(H(y), g["mresid" + key])


@pytest.mark.parametrize("kind,n", [(7, 17), (7, 33), (27, 17)])
def test_cghs_matches_restatement(restatement, kind, n):
    """Vcghs (cgd.cc:60-125): the same iteration count as the CPU
    restatement and the iterate within 1e-12 of it (the sums are ordered
    differently); the stop by count; itmax 0 does nothing."""
    from test_oracle import spd_case
    ops, cc, f = spd_case(n, kind, n + kind)
    x0 = np.random.default_rng(n).normal(size=n ** 3) * 0.1
    xo = x0.copy()
    it_o, _ = restatement.cghs(n, n, n, ops, cc, f, xo, 500, 1e-10)
    ac = T(np.stack(ops))
    work = [torch.zeros(n ** 3, dtype=torch.float64, device=DEV)
            for _ in range(3)]
    x = T(x0)
    it = pmgc.Vcghs(n, n, n, ac, T(cc), T(f), x, *work, 500, 1e-10)
    assert it == it_o and 0 < it < 500
    assert rel(H(x), xo) <= 1e-12
    x = T(x0)
    assert pmgc.Vcghs(n, n, n, ac, T(cc), T(f), x, *work, 3, 1e-10) == 3
    x = T(x0)
    assert pmgc.Vcghs(n, n, n, ac, T(cc), T(f), x, *work, 0, 1e-10) == 0
    assert np.array_equal(H(x), x0)
    z = torch.zeros(n ** 3, dtype=torch.float64, device=DEV)
    assert pmgc.Vcghs(n, n, n, ac, T(cc), z, z.clone(), *work, 10,
                      1e-10) == 0


def test_cg_level_matches_reference(golden_problem, restatement):
    g = golden_problem
    base = int(g["base"])
    n1 = 2 * base + 1
    A1 = [T(a) for a in g["A1"]]
    x = torch.zeros(n1 ** 3, dtype=torch.float64, device=DEV)
    iters = pmgc.cg_level(n1, n1, n1, A1, T(g["cg_rhs"]), x)
    assert iters > 0
    assert rel(H(x), g["cg_x"]) <= 1e-12
    xo = np.zeros(n1 ** 3)
    it_o = restatement.cg(n1, [np.ascontiguousarray(a) for a in g["A1"]],
                          g["cg_rhs"], xo)
    assert iters == it_o


def test_cg_level_iteration_cap_reports_timeout(golden_problem):
    from multigrid_b200._lib import PmgError
    g = golden_problem
    base = int(g["base"])
    n1 = 2 * base + 1
    x = torch.zeros(n1 ** 3, dtype=torch.float64, device=DEV)
    with pytest.raises(PmgError) as e:
        pmgc.cg_level(n1, n1, n1, [T(a) for a in g["A1"]], T(g["cg_rhs"]), x,
                      thresh=0.0, max_iters=3)
    assert e.value.status == -5
    # the context stays usable
    torch.cuda.synchronize()
    assert torch.isfinite(x).all()
