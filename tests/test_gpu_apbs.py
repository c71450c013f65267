"""The APBS driver on the GPU (pmg_Vmgdriv_d: Vmgdriv -> Vbuildops -> Vmvcs,
pmgc/mgdrvd.cc, pmgc/mgsubd.cc, pmgc/mgcsd.cc) against the CPU restatement
(oracle/pmg_oracle.c pmgo_mgdriv) on the same inputs.

Every kernel of the driver matches the restatement bit for bit (builders,
smoothers, residuals, transfers); the interior sums (damping, CG dot
products, stop norms) are added in a different order, so the cycle counts
must agree and the potential within 1e-12 relative; the boundary faces bit
for bit.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from multigrid_b200 import pmgc  # noqa: E402
from multigrid_b200._lib import PmgError  # noqa: E402
from test_oracle import apbs_maps, apbs_params  # noqa: E402

DEV = torch.device("cuda:0")
BOX_IN = ("xf", "yf", "zf", "gxcf", "gycf", "gzcf", "a1cf", "a2cf", "a3cf",
          "ccf", "fcf")


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64,
                           device=DEV)


def run_gpu(iparm, rparm, maps, n, tcf=None):
    u = torch.full((n ** 3,), 7.0, dtype=torch.float64, device=DEV)
    t = T(tcf) if tcf is not None else None
    it, ierr, ratio = pmgc.Vmgdriv(iparm, rparm, u,
                                   *[T(maps[k]) for k in BOX_IN], tcf=t)
    torch.cuda.synchronize()
    return u.cpu().numpy(), it, ierr, ratio, (t.cpu().numpy()
                                              if t is not None else None)


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("n,nlev,kw", [
    (17, 3, dict()),
    (17, 3, dict(mgprol=0)),
    (17, 3, dict(mgsmoo=4, itmax=80)),
    (33, 4, dict(istop=0, errtol=1e-6)),
    (17, 2, dict(nu1=1, nu2=3, mgkey=1)),
    (17, 3, dict(mgsolv=1)),
    (33, 4, dict(mgsolv=1, mgprol=0)),
    (17, 3, dict(mgcoar=0)),
    (33, 4, dict(mgcoar=0, mgsolv=1)),
    (17, 4, dict(mgsolv=1)),  # 3^3 coarsest level: one unknown in the band
])
def test_apbs_driver_matches_restatement(restatement, n, nlev, kw):
    maps = apbs_maps(n, n + nlev)
    iparm, rparm = apbs_params(n, nlev, **kw)
    uo = np.zeros(n ** 3)
    it_o, ie_o, r_o = restatement.mgdriv(iparm, rparm, uo, maps)
    u, it, ierr, ratio, _ = run_gpu(iparm, rparm, maps, n)
    assert (it, ierr) == (it_o, ie_o) and it > 1
    assert rel(u, uo) <= 1e-12
    assert abs(ratio - r_o) <= 1e-6 * r_o
    shell = np.ones((n, n, n), bool)
    shell[1:-1, 1:-1, 1:-1] = False
    assert np.array_equal(u.reshape(n, n, n)[shell],
                          uo.reshape(n, n, n)[shell])


@pytest.mark.parametrize("istop", [2, 3])
def test_apbs_driver_iterate_stop_tests(restatement, istop):
    """istop 2 (L1 change of the iterate, tcf overwritten with it) and 3
    (L2 error against a given true solution)."""
    n, nlev = 17, 3
    maps = apbs_maps(n, 21)
    if istop == 2:
        tcf = np.random.default_rng(4).normal(size=n ** 3) * 1e-3
    else:  # the converged solution as the true one
        tcf = np.zeros(n ** 3)
        restatement.mgdriv(*apbs_params(n, nlev, errtol=1e-14), tcf, maps)
    iparm, rparm = apbs_params(n, nlev, istop=istop, errtol=1e-9)
    to = tcf.copy()
    uo = np.zeros(n ** 3)
    it_o, ie_o, _ = restatement.mgdriv(iparm, rparm, uo, maps, to)
    u, it, ierr, _, t = run_gpu(iparm, rparm, maps, n, tcf)
    assert (it, ierr) == (it_o, ie_o) and ierr == 0
    assert rel(u, uo) <= 1e-12
    if istop == 2:
        assert rel(t, to) <= 1e-12
    else:
        assert np.array_equal(t, tcf)


def test_apbs_driver_one_level_and_itmax(restatement):
    n = 9
    maps = apbs_maps(n, 2)
    iparm, rparm = apbs_params(n, 1)
    uo = np.zeros(n ** 3)
    assert restatement.mgdriv(iparm, rparm, uo, maps)[0] == 1
    u, it, ierr, _, _ = run_gpu(iparm, rparm, maps, n)
    assert it == 1 and rel(u, uo) <= 1e-12
    iparm, rparm = apbs_params(17, 3, itmax=2, errtol=1e-30)
    maps = apbs_maps(17, 2)
    _, it, ierr, _, _ = run_gpu(iparm, rparm, maps, 17)
    assert (it, ierr) == (2, 1)


@pytest.mark.parametrize("kw", [dict(mgcoar=1), dict(mgsolv=2),
                                dict(mgsmoo=0), dict(mode=1), dict(nlev=5),
                                dict(istop=4), dict(mgdisc=1)])
def test_apbs_driver_rejects_untranslated_options(kw):
    n = 17
    kw = dict(kw)
    nlev = kw.pop("nlev", 3)
    iparm, rparm = apbs_params(n, nlev, **kw)
    with pytest.raises(PmgError) as e:
        run_gpu(iparm, rparm, apbs_maps(n, 1), n)
    assert e.value.status == -1


def test_band_solver_matches_reference(golden_band):
    """Vbuildband (band storage and Vdpbfa), Vdpbfa and Vdpbsl bit for bit
    against the reference's (buildBd.cc, mlinpckd.cc); the 27-point band
    stored where the matvec reads its couplings and factored as the
    reference factors it."""
    g = golden_band
    n = int(g["n"])
    nb = (n - 2) ** 3
    for kind in (7, 27):
        ac = T(g[f"op{kind}"])
        m = (n - 2) ** 2 + (0 if kind == 7 else n - 1)
        acB = torch.full(((m + 1) * nb,), 3.0, dtype=torch.float64,
                         device=DEV)
        key, ipcB = pmgc.Vbuildband(n, n, n, ac, acB)
        want = g["band7"] if kind == 7 else g["fac27"]
        assert key == 0 and ipcB == [nb, m, m + 1, 1]
        assert np.array_equal(acB.cpu().numpy(), want)
        x = T(g[f"b{kind}"])
        pmgc.Vdpbsl(acB, m + 1, nb, m, x)
        assert np.array_equal(x.cpu().numpy(), g[f"x{kind}"])
    m = (n - 2) ** 2 + n - 1
    abd = T(g["band27"])
    assert pmgc.Vdpbfa(abd, m + 1, nb, m) == 0
    assert np.array_equal(abd.cpu().numpy(), g["fac27"])
    bad = T(-g["band27"])
    assert pmgc.Vdpbfa(bad, m + 1, nb, m) == 1


# ---- Vmvcs on a hierarchy the caller built (APBS packed storage) ----------
def packed_hierarchy(n, nlev, maps, mgsolv=0):
    """Vbuildops done by hand through the C ABI into APBS's packed
    multilevel storage (Vbuildstr's iz table, pmgc/mgsubd.cc:266-345):
    box-method fine operator, operator-based prolongation, Galerkin coarse
    operators with restricted cc and fc, and for mgsolv 1 the factored band
    one level below the coarsest."""
    sizes = [n]
    for _ in range(nlev - 1):
        sizes.append((sizes[-1] - 1) // 2 + 1)
    n3 = [s ** 3 for s in sizes]
    cols = [4] + [14] * (nlev - 1)
    nreal = nlev + (1 if mgsolv == 1 else 0)
    iz = np.zeros((nreal, 50), dtype=np.int64)  # column-major iz(50, lev)
    iz[0, :] = 1
    for lev in range(1, nreal):
        m = n3[lev - 1]
        iz[lev, 0] = iz[lev - 1, 0] + m
        iz[lev, 4] = iz[lev - 1, 4] + 100
        iz[lev, 5] = iz[lev - 1, 5] + 100
        iz[lev, 6] = iz[lev - 1, 6] + cols[lev - 1] * m
        if lev < nlev:
            iz[lev, 10] = iz[lev - 1, 10] + 27 * n3[lev]
    tot = sum(n3)
    band_len = 0
    if mgsolv == 1:
        nc = sizes[-1] - 2
        m = nc * nc + nc + 1
        band_len = (m + 1) * nc ** 3
    ac = torch.zeros(iz[nlev - 1, 6] - 1 + cols[-1] * n3[-1] + band_len,
                     dtype=torch.float64, device=DEV)
    pc = torch.zeros(max(1, iz[nlev - 1, 10] - 1), dtype=torch.float64,
                     device=DEV)
    cc = torch.zeros(tot, dtype=torch.float64, device=DEV)
    fc = torch.zeros(tot, dtype=torch.float64, device=DEV)
    ipc = np.zeros(100 * nreal, dtype=np.int64)

    def lv(lev):  # views of level lev (1-based)
        o, m = iz[lev - 1, 0] - 1, n3[lev - 1]
        a0 = iz[lev - 1, 6] - 1
        return (ac[a0:a0 + cols[lev - 1] * m].view(cols[lev - 1], m),
                cc[o:o + m], fc[o:o + m])

    A1, c1, f1 = lv(1)
    ip, _ = pmgc.VbuildA_fv(n, n, n, 0, A1[0], c1, f1, A1[1], A1[2], A1[3],
                            *[T(maps[k]) for k in BOX_IN])
    ipc[0:12] = ip
    for lev in range(2, nlev + 1):
        nf, ncs = sizes[lev - 2], sizes[lev - 1]
        Af, cf, ff = lv(lev - 1)
        Ac, cC, fC = lv(lev)
        p0 = iz[lev - 2, 10] - 1
        P = [pc[p0 + q * n3[lev - 1]: p0 + (q + 1) * n3[lev - 1]]
             for q in range(27)]
        if lev == 2:
            pmgc.VbuildPb_op7(nf, nf, nf, ncs, ncs, ncs, Af[0], Af[1], Af[2],
                              Af[3], P)
            pmgc.VbuildG_7(nf, nf, nf, ncs, ncs, ncs, P, Af[0], Af[1], Af[2],
                           Af[3], list(Ac))
        else:
            pmgc.VbuildPb_op27(nf, nf, nf, ncs, ncs, ncs, list(Af), P)
            pmgc.VbuildG_27(nf, nf, nf, ncs, ncs, ncs, P, list(Af), list(Ac))
        pmgc.Vrestrc2(nf, nf, nf, ncs, ncs, ncs, cf, cC, P)
        pmgc.Vrestrc2(nf, nf, nf, ncs, ncs, ncs, ff, fC, P)
        ipc[100 * (lev - 1) + 10] = 27
    if mgsolv == 1:
        Ac, _, _ = lv(nlev)
        b0 = iz[nlev, 6] - 1
        key, ipb = pmgc.Vbuildband(sizes[-1], sizes[-1], sizes[-1], Ac,
                                   ac[b0:b0 + band_len])
        assert key == 0
        ipc[100 * nlev:100 * nlev + 4] = ipb
    torch.cuda.synchronize()
    return dict(iz=iz.ravel(), ipc=ipc, ac=ac, pc=pc, cc=cc, fc=fc,
                tot=tot, nreal=nreal)


@pytest.mark.parametrize("n,nlev,kw", [
    (17, 3, dict()),
    (33, 4, dict(istop=0, errtol=1e-6)),
    (17, 3, dict(mgsolv=1)),
    (17, 3, dict(mgsmoo=4, itmax=80)),
])
def test_vmvcs_on_packed_hierarchy_matches_driver(restatement, n, nlev, kw):
    """pmg_Vmvcs_d (Vmvcs, pmgc/mgcsd.cc:61-531) on a hierarchy built
    through the C ABI in APBS's packed storage, from a zero iterate: the
    same cycles as the restated driver (pmgo_mgdriv) on the same inputs,
    the interior potential within 1e-12, and bit for bit the GPU driver's
    (which runs the same kernels after its own Vbuildops)."""
    maps = apbs_maps(n, n + nlev + 7)
    iparm, rparm = apbs_params(n, nlev, **kw)
    h = packed_hierarchy(n, nlev, maps, mgsolv=iparm[20])
    x = torch.zeros(h["tot"], dtype=torch.float64, device=DEV)
    w0 = torch.zeros_like(x)
    w = [torch.zeros(n ** 3, dtype=torch.float64, device=DEV)
         for _ in range(3)]
    it, ierr = pmgc.Vmvcs(n, n, n, x, h["iz"], w0, *w, istop=iparm[10],
                          itmax=iparm[9], nlev=nlev, ipc=h["ipc"],
                          pc=h["pc"], ac=h["ac"], cc=h["cc"], fc=h["fc"],
                          nlev_real=h["nreal"], mgsolv=iparm[20],
                          errtol=rparm[0], nu1=iparm[6], nu2=iparm[7],
                          mgsmoo=iparm[19])
    torch.cuda.synchronize()
    u = x[:n ** 3].cpu().numpy().reshape(n, n, n)[1:-1, 1:-1, 1:-1]
    uo = np.zeros(n ** 3)
    it_o, ie_o, _ = restatement.mgdriv(iparm, rparm, uo, maps)
    uo = uo.reshape(n, n, n)[1:-1, 1:-1, 1:-1]
    assert (it, ierr) == (it_o, ie_o) and it > 1
    assert rel(u, uo) <= 1e-12
    ug, it_g, _, _, _ = run_gpu(iparm, rparm, maps, n)
    assert it_g == it
    assert np.array_equal(u, ug.reshape(n, n, n)[1:-1, 1:-1, 1:-1])


def test_vmvcs_rejects_bad_tables():
    n, nlev = 17, 3
    maps = apbs_maps(n, 5)
    h = packed_hierarchy(n, nlev, maps)
    x = torch.zeros(h["tot"], dtype=torch.float64, device=DEV)
    w = [torch.zeros(n ** 3, dtype=torch.float64, device=DEV)
         for _ in range(4)]
    bad = h["ipc"].copy()
    bad[100 + 10] = 9  # not a stencil size
    with pytest.raises(PmgError):
        pmgc.Vmvcs(n, n, n, x, h["iz"], *w, istop=1, itmax=5, nlev=nlev,
                   ipc=bad, pc=h["pc"], ac=h["ac"], cc=h["cc"], fc=h["fc"])
    with pytest.raises(PmgError):  # the band level is missing
        pmgc.Vmvcs(n, n, n, x, h["iz"], *w, istop=1, itmax=5, nlev=nlev,
                   ipc=h["ipc"], pc=h["pc"], ac=h["ac"], cc=h["cc"],
                   fc=h["fc"], mgsolv=1)
