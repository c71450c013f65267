"""The CPU restatement (oracle/pmg_oracle.c) against the reference's own
outputs: the golden fixtures made by tests/golden/make_golden.py from the
reference PMG class and pmgc kernels, and — where the reference-built oracle
(oracle/_ref) is present — random cases run through it directly.

Per-point kernels (smoothers, matvec, residual, transfers) keep the
reference's operation order and must match bit for bit; the builders are a
generic formulation and must match to rounding; whole solves to 1e-12
relative L2 with the same number of cycles.
"""
import os

import numpy as np
import pytest

from conftest import box_case, fine_of
from oracle.oracle import Reference, Restatement, reference_available

TOL_BUILD = 1e-13   # builders: relative to the array's max magnitude
TOL_SOLVE = 1e-12   # potential: relative L2


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_gs7_bitexact(restatement, golden_kernels):
    g = golden_kernels
    n, op7 = int(g["nf"]), g["op7"]
    for name, iad, zi in (("a0z0", 0, 0), ("a1z0", 1, 0), ("a0z1", 0, 1)):
        x = g["x0"].copy()
        restatement.gsrb7x(n, op7[0], g["cc"], g["f"], op7[1], op7[2], op7[3],
                           x, itmax=2, iadjoint=iad, zero_init=zi)
        assert np.array_equal(x, g["gs7_" + name]), name


def test_gs27_bitexact(restatement, golden_kernels):
    g = golden_kernels
    n = int(g["nf"])
    op = [np.ascontiguousarray(a) for a in g["op27"]]
    for name, iad, zi in (("a0z0", 0, 0), ("a1z0", 1, 0), ("a0z1", 0, 1)):
        x = g["x0"].copy()
        restatement.gsrb27x(n, op, g["cc"], g["f"], x, itmax=2, iadjoint=iad,
                            zero_init=zi)
        assert np.array_equal(x, g["gs27_" + name]), name


def test_matvec_mresid_bitexact(restatement, golden_kernels):
    g = golden_kernels
    n = int(g["nf"])
    op7 = [np.ascontiguousarray(a) for a in g["op7"]]
    op27 = [np.ascontiguousarray(a) for a in g["op27"]]
    for ops, key in ((op7, "7"), (op27, "27")):
        y = np.zeros(n ** 3)
        restatement.matvec(n, ops, g["cc"], g["x0"], y)
        assert np.array_equal(y, g["matvec" + key])
        r = np.zeros(n ** 3)
        restatement.mresid(n, ops, g["cc"], g["f"], g["x0"], r)
        assert np.array_equal(r, g["mresid" + key])


def test_transfers_bitexact(restatement, golden_kernels):
    g = golden_kernels
    nf, nc = int(g["nf"]), int(g["nc"])
    P = [np.ascontiguousarray(a) for a in g["P_rand"]]
    e = np.zeros(nf ** 3)
    restatement.interp2(nc, nf, g["xc"], e, P)
    assert np.array_equal(e, g["interp"])
    r = np.zeros(nc ** 3)
    restatement.restrc2(nf, nc, g["x0"], r, P)
    assert np.array_equal(r, g["restrict"])


def test_build_prolongation(restatement, golden_kernels):
    g = golden_kernels
    nf, nc = int(g["nf"]), int(g["nc"])
    for ops, key in (([np.ascontiguousarray(a) for a in g["op7"]], "P_op7"),
                     ([np.ascontiguousarray(a) for a in g["op27"]], "P_op27")):
        P = [np.zeros(nc ** 3) for _ in range(27)]
        restatement.buildP_op(nf, nc, ops, P)
        for s in range(27):
            assert rel(P[s], g[key][s]) <= TOL_BUILD, (key, s)
    P = [np.zeros(nc ** 3) for _ in range(27)]
    restatement.buildP_trilin(nc, P)
    assert np.array_equal(np.stack(P), g["P_trilin"])


def test_build_galerkin(restatement, golden_kernels):
    g = golden_kernels
    nf, nc = int(g["nf"]), int(g["nc"])
    P = [np.ascontiguousarray(a) for a in g["P_rand"]]
    for ops, key in (([np.ascontiguousarray(a) for a in g["op7"]], "G7"),
                     ([np.ascontiguousarray(a) for a in g["op27"]], "G27")):
        out = [np.zeros(nc ** 3) for _ in range(14)]
        restatement.buildG(nf, nc, P, ops, out)
        for s in range(14):
            assert rel(out[s], g[key][s]) <= TOL_BUILD, (key, s)


@pytest.mark.parametrize("tag", ["c9", "r11"])
def test_box_builder_bitexact(restatement, golden_box, tag):
    """VbuildA_fv (pmgc/buildAd.cc:63-212): operator, kappa term, source
    with the Dirichlet values folded in, bit for bit; shell untouched; the
    ipc/numdia bookkeeping."""
    c = box_case(golden_box, tag)
    out = [np.ascontiguousarray(a) for a in c["init"].copy()]
    ipc, numdia = restatement.buildA_fv(*c["n"], c["ipkey"], c["inputs"],
                                        out)
    assert np.array_equal(np.stack(out), c["out"])
    assert np.array_equal(ipc, c["ipc"]) and numdia == c["numdia"]


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
def test_box_builder_vs_reference_random():
    import ctypes
    from tests.golden.make_golden import box_inputs
    rng = np.random.default_rng(77)
    c = box_inputs(rng, 13, 17, 17)
    want = c["init"].copy()
    got = [np.ascontiguousarray(a) for a in c["init"].copy()]
    ref = Reference()
    D = ctypes.POINTER(ctypes.c_double)
    ipc = (ctypes.c_int * 12)()
    nd = ctypes.c_int()
    ref.lib.pmgref_VbuildA_fv(
        13, 17, 17, 5, ctypes.byref(nd), ipc,
        *[want[s].ctypes.data_as(D) for s in range(6)],
        *[c[k].ctypes.data_as(D) for k in Restatement.BOX_IN])
    ipc2, nd2 = Restatement().buildA_fv(13, 17, 17, 5, c, got)
    assert np.array_equal(np.stack(got), want)
    assert list(ipc2) == list(ipc) and nd2 == nd.value


def spd_case(n, kind, seed):
    """A symmetric positive definite operator (strictly diagonally dominant,
    positive couplings), kappa map, right-hand side; zero shell."""
    rng = np.random.default_rng(seed)
    cols = 4 if kind == 7 else 14
    ops = [rng.uniform(0.5, 2.0, n ** 3) for _ in range(cols)]
    ops[0] = rng.uniform(60.0, 80.0, n ** 3)
    return ops, rng.uniform(0.0, 0.5, n ** 3), rng.normal(size=n ** 3)


def dense_operator(n, ops, cc):
    """The interior block of A as a dense matrix (x fastest), from the
    restatement's matvec applied to unit vectors."""
    m = (n - 2) ** 3
    idx = [((k * n) + j) * n + i for k in range(1, n - 1)
           for j in range(1, n - 1) for i in range(1, n - 1)]
    A = np.empty((m, m))
    r = Restatement()
    for c, q in enumerate(idx):
        e = np.zeros(n ** 3)
        e[q] = 1.0
        y = np.zeros(n ** 3)
        r.matvec(n, ops, cc, e, y)
        A[:, c] = y[idx]
    return A, idx


@pytest.mark.parametrize("kind", [7, 27])
def test_cghs_restatement_solves_the_system(restatement, kind):
    """Vcghs (pmgc/cgd.cc:60-125) as documented converges to the solution
    of the interior system with a zero shell; the counted iterations stop
    at the tolerance and at itmax."""
    n = 7
    ops, cc, f = spd_case(n, kind, 5 + kind)
    A, idx = dense_operator(n, ops, cc)
    assert np.allclose(A, A.T)
    want = np.linalg.solve(A, f[idx])
    x = np.zeros(n ** 3)
    it, r = restatement.cghs(n, n, n, ops, cc, f, x, 200, 1e-12)
    assert 0 < it < 200
    assert np.abs(x[idx] - want).max() <= 1e-10 * np.abs(want).max()
    assert np.sqrt(np.sum(r[idx] ** 2)) <= 1e-12 * np.sqrt(np.sum(f[idx] ** 2))
    x3 = np.zeros(n ** 3)
    assert restatement.cghs(n, n, n, ops, cc, f, x3, 3, 1e-12)[0] == 3
    x0 = np.zeros(n ** 3)
    assert restatement.cghs(n, n, n, ops, cc, f, x0, 0, 1e-12)[0] == 0
    assert not x0.any()


def apbs_params(n, nlev, **kw):
    """0-based iparm / rparm of the APBS driver (Vpackmg order,
    mgsubd.cc:538-576): linear, Galerkin coarsening, CG coarse solve."""
    p = dict(nx=n, ny=n, nz=n, nlev=nlev, nu1=2, nu2=2, mgkey=0, itmax=60,
             istop=1, iinfo=0, ipkey=0, mode=0, mgprol=1, mgcoar=2,
             mgdisc=0, mgsmoo=1, mgsolv=0, iperf=0, errtol=1e-10)
    p.update(kw)
    iparm = [0] * 25
    for i, k in ((2, "nx"), (3, "ny"), (4, "nz"), (5, "nlev"), (6, "nu1"),
                 (7, "nu2"), (8, "mgkey"), (9, "itmax"), (10, "istop"),
                 (11, "iinfo"), (13, "ipkey"), (15, "mode"), (16, "mgprol"),
                 (17, "mgcoar"), (18, "mgdisc"), (19, "mgsmoo"),
                 (20, "mgsolv"), (21, "iperf")):
        iparm[i] = p[k]
    rparm = [0.0] * 12
    rparm[0] = p["errtol"]
    return iparm, rparm


def apbs_maps(n, seed, h=0.5):
    """Box-method inputs on a uniform mesh: smooth dielectric-like face maps,
    kappa, source and boundary values."""
    rng = np.random.default_rng(seed)
    g = np.arange(n) * h
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    eps = 2.0 + 76.0 / (1.0 + np.exp(-(np.sqrt((x - g[-1] / 2) ** 2 +
                                               (y - g[-1] / 2) ** 2 +
                                               (z - g[-1] / 2) ** 2) - 2.0)))
    eps = eps.ravel()
    return dict(xf=g.copy(), yf=g.copy(), zf=g.copy(),
                gxcf=rng.normal(0.0, 0.1, n * n * 2),
                gycf=rng.normal(0.0, 0.1, n * n * 2),
                gzcf=rng.normal(0.0, 0.1, n * n * 2),
                a1cf=eps.copy(), a2cf=eps.copy(), a3cf=eps.copy(),
                ccf=np.full(n ** 3, 0.05), fcf=rng.normal(0.0, 1.0, n ** 3))


@pytest.mark.parametrize("mgsmoo,mgprol,mgsolv,mgcoar", [
    (1, 1, 0, 2), (1, 0, 0, 2), (4, 1, 0, 2), (1, 1, 1, 2), (1, 1, 0, 0),
    (1, 0, 1, 0)])
def test_apbs_driver_restatement_solves_the_box_system(restatement, mgsmoo,
                                                        mgprol, mgsolv,
                                                        mgcoar):
    """The restated APBS driver (Vmgdriv -> Vbuildops -> Vmvcs) converges
    to the direct solution of the box-method system it builds, with the
    boundary values on the shell."""
    n, nlev = 17, 3
    maps = apbs_maps(n, 3)
    iparm, rparm = apbs_params(n, nlev, mgsmoo=mgsmoo, mgprol=mgprol,
                               mgsolv=mgsolv, mgcoar=mgcoar)
    u = np.zeros(n ** 3)
    it, ierr, ratio = restatement.mgdriv(iparm, rparm, u, maps)
    assert ierr == 0 and 1 < it < 60 and ratio <= 1e-10
    out = [np.zeros(n ** 3) for _ in range(6)]
    restatement.buildA_fv(n, n, n, 0, maps, out)
    oC, cc, fc, oE, oN, uC = out
    A, idx = dense_operator(n, [oC, oE, oN, uC], cc)
    want = np.linalg.solve(A, fc[idx])
    assert np.abs(u[idx] - want).max() <= 1e-8 * np.abs(want).max()
    # faces written x, then y, then z (edges keep the later face's value)
    u3 = u.reshape(n, n, n)
    gx = maps["gxcf"].reshape(2, n, n)
    gy = maps["gycf"].reshape(2, n, n)
    gz = maps["gzcf"].reshape(2, n, n)
    c = slice(1, -1)
    assert np.array_equal(u3[c, c, 0], gx[0, c, c])
    assert np.array_equal(u3[c, c, -1], gx[1, c, c])
    assert np.array_equal(u3[c, 0, :], gy[0, c, :])
    assert np.array_equal(u3[c, -1, :], gy[1, c, :])
    assert np.array_equal(u3[0], gz[0]) and np.array_equal(u3[-1], gz[1])


def test_band_solver_bitexact(restatement, golden_band):
    """Vbuildband / Vdpbfa / Vdpbsl (buildBd.cc, mlinpckd.cc): the band of a
    7-point operator and its factor bit for bit; the factor and the solve of
    a 27-point band bit for bit; the 27-point band solves the dense
    system."""
    g = golden_band
    n = int(g["n"])
    abd, nb, m, lda = restatement.buildband(n, [np.ascontiguousarray(a)
                                                for a in g["op7"]])
    assert restatement.dpbfa(abd, lda, nb, m) == 0
    assert np.array_equal(abd, g["band7"])
    x = g["b7"].copy()
    restatement.dpbsl(abd, lda, nb, m, x)
    assert np.array_equal(x, g["x7"])
    ops27 = [np.ascontiguousarray(a) for a in g["op27"]]
    abd, nb, m, lda = restatement.buildband(n, ops27)
    assert np.array_equal(abd, g["band27"])
    assert restatement.dpbfa(abd, lda, nb, m) == int(g["info27"]) == 0
    assert np.array_equal(abd, g["fac27"])
    x = g["b27"].copy()
    restatement.dpbsl(abd, lda, nb, m, x)
    assert np.array_equal(x, g["x27"])
    A, idx = dense_operator(n, ops27, np.zeros(n ** 3))
    y = np.zeros(n ** 3)
    y[idx] = x
    Ax = np.zeros(n ** 3)
    restatement.matvec(n, ops27, np.zeros(n ** 3), y, Ax)
    assert np.abs(Ax[idx] - g["b27"]).max() <= 1e-12 * np.abs(g["b27"]).max()


@pytest.mark.parametrize("nlev,mgsolv,mgcoar", [(4, 0, 2), (4, 1, 2),
                                                 (4, 1, 0), (1, 1, 2)])
def test_apbs_driver_restatement_extreme_levels(restatement, nlev, mgsolv,
                                                 mgcoar):
    """The restated driver down to a 3^3 coarsest level (one unknown) and
    with a single level (the coarse solve alone), for both coarse solvers:
    the same box-system solution."""
    n = 17
    maps = apbs_maps(n, 40 + nlev)
    iparm, rparm = apbs_params(n, nlev, mgsolv=mgsolv, mgcoar=mgcoar,
                               itmax=80)
    u = np.zeros(n ** 3)
    it, ierr, ratio = restatement.mgdriv(iparm, rparm, u, maps)
    out = [np.zeros(n ** 3) for _ in range(6)]
    restatement.buildA_fv(n, n, n, 0, maps, out)
    oC, cc, fc, oE, oN, uC = out
    if nlev == 1 and mgsolv == 1:
        # one direct band solve of the operator without cc (the band holds
        # ac only, as the reference's Vbuildband)
        A0, idx = dense_operator(n, [oC, oE, oN, uC], np.zeros(n ** 3))
        want = np.linalg.solve(A0, fc[idx])
        assert it == 1
    else:
        A, idx = dense_operator(n, [oC, oE, oN, uC], cc)
        want = np.linalg.solve(A, fc[idx])
        assert ierr == 0 and ratio <= 1e-10
    assert np.abs(u[idx] - want).max() <= 1e-8 * np.abs(want).max()


def test_hierarchy(restatement, golden_problem):
    g = golden_problem
    base, nlev = int(g["base"]), int(g["nlev"])
    hier = restatement.hierarchy(base, nlev, fine_of(g))
    for L, (P, A) in hier.items():
        for s in range(27):
            assert rel(P[s], g[f"P{L}"][s]) <= TOL_BUILD, (L, "P", s)
        for s in range(14):
            assert rel(A[s], g[f"A{L}"][s]) <= 1e-12, (L, "A", s)


def test_cg_level1(restatement, golden_problem):
    g = golden_problem
    base = int(g["base"])
    n1 = 2 * base + 1
    A1 = [np.ascontiguousarray(a) for a in g["A1"]]
    x = np.zeros(n1 ** 3)
    restatement.cg(n1, A1, g["cg_rhs"], x)
    assert rel(x, g["cg_x"]) <= 1e-12


@pytest.mark.parametrize("trilinear", [False, True])
def test_solve(restatement, golden_problem, trilinear):
    g = golden_problem
    base, nlev = int(g["base"]), int(g["nlev"])
    sfx = "_trilin" if trilinear else ""
    x, cycles, hist = restatement.solve(base, nlev, fine_of(g), tol=1e-10,
                                        max_cycles=60, trilinear=trilinear)
    assert cycles == int(g["cycles" + sfx])
    xr = g["x" + sfx]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= TOL_SOLVE
    h = g["hist" + sfx]
    # early residual norms agree closely; late ones are rounding-dominated
    assert abs(hist[1] / h[1] - 1) < 1e-9


def test_setup_matches_reference(golden_problem):
    from multigrid_b200.molecule import REFERENCE_PHYSICS
    from multigrid_b200.problem import setup_fine
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    n = base * 2 ** nlev + 1
    out = setup_fine(n, box / (n - 1), g["atoms"], REFERENCE_PHYSICS)
    for k in ("oC", "oE", "oN", "uC", "f", "x0"):
        assert np.array_equal(out[k], g["fine_" + k]), k


def test_oracle_setup_matches_reference_golden(golden_problem, restatement):
    """The restated set-up (pmgo_setup_fine) at the reference's constants
    gives the reference's own set-up bit for bit."""
    from multigrid_b200.molecule import REFERENCE_PHYSICS
    g = golden_problem
    base, nlev, box = int(g["base"]), int(g["nlev"]), float(g["box"])
    n = base * 2 ** nlev + 1
    out = restatement.setup_fine(n, box / (n - 1), g["atoms"],
                                 REFERENCE_PHYSICS)
    for k in ("oC", "oE", "oN", "uC", "f", "x0"):
        assert np.array_equal(out[k], g["fine_" + k]), k


@pytest.mark.parametrize("probe", [0.0, 1.4])
@pytest.mark.parametrize("n,h,natoms,radius", [(33, 0.5, 150, 5.0),
                                               (41, 0.4, 400, 6.0)])
def test_oracle_setup_bitexact_vs_product_host_setup(restatement, probe, n,
                                                     h, natoms, radius):
    """The oracle's own set-up (what the reference arm of the benchmark and
    the parity tests feed the reference with) and the product's host set-up
    give the same bits, with and without the probe surface, at the PB
    workloads' physics."""
    from multigrid_b200.molecule import DEFAULT_PHYSICS, synthetic_atoms
    from multigrid_b200.problem import setup_fine
    box = h * (n - 1)
    atoms = synthetic_atoms(natoms, radius, 40 + n, (box / 2,) * 3)
    phys = dict(DEFAULT_PHYSICS, probe_radius=probe)
    a = restatement.setup_fine(n, h, atoms, phys)
    b = setup_fine(n, h, atoms, phys)
    for k in a:
        assert np.array_equal(a[k], b[k]), (probe, k)
    # the probe surface changes the dielectric maps (solute grows)
    if probe > 0:
        vdw = restatement.setup_fine(n, h, atoms,
                                     dict(DEFAULT_PHYSICS, probe_radius=0.0))
        assert (a["oE"] <= vdw["oE"]).all() and (a["oE"] < vdw["oE"]).any()


def test_oracle_setup_rejects_atoms_outside(restatement):
    from multigrid_b200.molecule import DEFAULT_PHYSICS
    with pytest.raises(ValueError):
        restatement.setup_fine(9, 0.5, np.array([[10.0, 1.0, 1.0, 1.5, 1.0]]),
                               DEFAULT_PHYSICS)


# -------- direct comparison with the reference-built oracle (if built) --------
needs_ref = pytest.mark.skipif(not reference_available(),
                               reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("base,nlev", [(2, 3), (4, 2), (3, 4), (4, 4)])
def test_solve_vs_reference(restatement, base, nlev):
    from multigrid_b200.molecule import REFERENCE_PHYSICS, synthetic_atoms
    from multigrid_b200.problem import setup_fine
    ref = Reference()
    n = base * 2 ** nlev + 1
    h = 0.5
    box = h * (n - 1)
    atoms = synthetic_atoms(3 * n, box / 5, 100 + n, (box / 2,) * 3)
    fine = setup_fine(n, h, atoms, REFERENCE_PHYSICS)
    xr, cr, _ = ref.solve(base, nlev, fine, tol=1e-10, max_cycles=60)
    xo, co, _ = restatement.solve(base, nlev, fine, tol=1e-10, max_cycles=60)
    assert co == cr
    assert np.linalg.norm(xo - xr) / np.linalg.norm(xr) <= TOL_SOLVE


@needs_ref
def test_setup_vs_reference_random():
    from multigrid_b200.molecule import REFERENCE_PHYSICS, synthetic_atoms
    from multigrid_b200.problem import setup_fine
    ref = Reference()
    for base, nlev, box in ((4, 3, 16.0), (4, 4, 32.0), (3, 4, 24.0)):
        n = base * 2 ** nlev + 1
        atoms = synthetic_atoms(60, box / 4, 7 + base, (box / 2,) * 3)
        a = ref.setup(base, nlev, atoms, 0.15, 2.0)
        b = setup_fine(n, box / (n - 1), atoms, REFERENCE_PHYSICS)
        for k in a:
            assert np.array_equal(a[k], b[k]), (base, nlev, k)


@pytest.mark.skipif(not reference_available(), reason="reference not built")
@pytest.mark.parametrize("iters", [1, 3, 8])
def test_pcg_restatement_matches_reference(golden_problem, restatement,
                                           iters):
    """The app's MG-preconditioned CG (CG_Solver.h:45-242 with the class as
    preconditioner) after a fixed number of iterations, restatement against
    the reference run through its own solver object."""
    from oracle.oracle import Reference
    g = golden_problem
    base, nlev = int(g["base"]), int(g["nlev"])
    fine = fine_of(g)
    xo, c, _ = restatement.pcg(base, nlev, fine, iters)
    xr = Reference().pcg(base, nlev, fine, iters)
    assert c == iters
    assert np.linalg.norm(xo - xr) <= 1e-13 * np.linalg.norm(xr)


def test_pcg_restatement_converges_to_the_solve(golden_problem, restatement):
    g = golden_problem
    base, nlev = int(g["base"]), int(g["nlev"])
    fine = fine_of(g)
    xs, cs, _ = restatement.solve(base, nlev, fine, tol=1e-10)
    xo, c, h = restatement.pcg(base, nlev, fine, 100, tol=1e-10)
    assert 0 < c <= cs
    assert h[-1] / h[0] < 1e-10
    assert np.linalg.norm(xo - xs) <= 1e-9 * np.linalg.norm(xs)


def test_reference_fine_couplings_are_two_valued(golden_problem):
    """The property the mixed path's coded couplings rest on, checked on the
    reference's own set-up (PBE_pmgc_class.h:248-318): over the couplings
    the interior points read, oE, oN and uC each take two values (inside and
    outside dielectric), in double and after rounding to float."""
    g = golden_problem
    n = int(g["base"]) * 2 ** int(g["nlev"]) + 1
    f = fine_of(g)
    sl = slice(1, n - 1)
    a = {k: f[k].reshape(n, n, n) for k in ("oE", "oN", "uC")}
    lo = slice(0, n - 1)  # along the coupling: the lower face of i = 2 too
    read = {"oE": a["oE"][sl, sl, lo].ravel(),   # [k, j, i]
            "oN": a["oN"][sl, lo, sl].ravel(),
            "uC": a["uC"][lo, sl, sl].ravel()}
    for k, v in read.items():
        assert len(np.unique(v)) <= 2, k
        assert len(np.unique(v.astype(np.float32))) <= 2, k


# -------- file formats against the reference's own reader and writer --------
PQR_TEXT = """REMARK   1 synthetic PQR for the reader comparison
REMARK   6 Total charge on this protein: 0.0000 e
ATOM      1  N   ARG     1      -8.544   3.578  14.046  0.1305 1.8240
ATOM      2  CA  ARG     1      -7.776   3.484  12.790 -0.0223 1.9080
HETATM    3  O   HOH     2       1.5e1  -0.25   7.125  -0.8340 1.7683
ATOM      4  CB  ARG A   1      -7.640   2.025  12.309  0.0118 1.9080
ATOM      5  CG  ARG     1      -6.000   2.000   3.000  0.0000 0.0000
TER
END
"""


@needs_ref
def test_pqr_reader_matches_reference(tmp_path):
    """pmg_read_pqr and the reference's read_pqr_file (fileio.cc:10-53) on
    the same file: the same atoms, bit for bit (rows with a chain field have
    eleven fields and are skipped by both)."""
    from multigrid_b200.fileio import read_pqr
    path = tmp_path / "mol.pqr"
    path.write_text(PQR_TEXT)
    ours = read_pqr(str(path))
    ref = Reference().read_pqr(str(path))
    assert ours.shape == (4, 5)
    assert np.array_equal(ours, ref)


@needs_ref
def test_pqr_reader_matches_reference_on_its_molecule():
    """The reference's own molecule file 1PIT.pqr, read by both readers."""
    from oracle.oracle import reference_tree
    from multigrid_b200.fileio import read_pqr
    tree = reference_tree()
    if tree is None or not os.path.exists(os.path.join(tree, "1PIT.pqr")):
        pytest.skip("the reference tree is not on this machine")
    path = os.path.join(tree, "1PIT.pqr")
    ours = read_pqr(path)
    ref = Reference().read_pqr(path)
    assert len(ours) == 892
    assert np.array_equal(ours, ref)


@needs_ref
@pytest.mark.parametrize("shape", [0, 1])
def test_dx_writer_matches_reference_byte_for_byte(tmp_path, shape):
    """pmg_write_dx and the reference's print_dx_to_stream
    (Domain.h:136-185) write the same bytes for the same array, origin and
    box, on a non-cubic and a cubic grid."""
    from multigrid_b200.fileio import write_dx
    ref = Reference()
    n0, n1, n2 = (s + 2 for s in ref.DX_SHAPES[shape])  # slowest first
    rng = np.random.default_rng(shape)
    vals = rng.normal(size=(n0, n1, n2)) * 10.0 ** rng.integers(-5, 5,
                                                                (n0, n1, n2))
    vals[0, 0, :3] = [0.0, -0.0, 1.0]
    origin, box = (-1.5, 2.25, 1e-3), 12.5
    want = ref.write_dx(shape, vals.ravel(), origin, box)
    path = tmp_path / "v.dx"
    write_dx(str(path), vals, origin=origin, box_length=box)
    got = path.read_text()
    assert got == want
