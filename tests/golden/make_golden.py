"""Generates the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own PBE_pmgc_class.h and pmgc kernels, compiled against
the host SYCL shim (oracle/_ref/libpmgc_ref.so, built by `make -C oracle`
from the reference tree), on small seeded inputs and stores inputs and
outputs as compressed .npz files. The reference tree is only needed to
regenerate them:

    make -C oracle -j8 && python tests/golden/make_golden.py [group ...]

(groups: kernels, problems, box_operator, band; all by default).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from multigrid_b200.molecule import synthetic_atoms  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def random_op27(rng, n):
    """Diagonally dominant symmetric 27-point operator (14 diagonals)."""
    a = [rng.uniform(0.5, 2.0, n ** 3) for _ in range(14)]
    a[0] = rng.uniform(28.0, 40.0, n ** 3)
    return a


def kernels(ref: Reference) -> None:
    L = ref.lib
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)

    def d(a):
        return a.ctypes.data_as(D)

    def pp(arrs):
        return (D * len(arrs))(*[d(a) for a in arrs])

    rng = np.random.default_rng(20261203)
    nf, nc = 9, 5
    op27 = random_op27(rng, nf)
    op7 = [rng.uniform(20.0, 30.0, nf ** 3)] + [
        rng.uniform(0.5, 2.0, nf ** 3) for _ in range(3)]
    cc = rng.uniform(0.0, 0.5, nf ** 3)
    f = rng.normal(0.0, 1.0, nf ** 3)
    x0 = rng.normal(0.0, 1.0, nf ** 3)
    out = dict(nf=nf, nc=nc, op27=np.stack(op27), op7=np.stack(op7), cc=cc,
               f=f, x0=x0)
    for name, iad, zi in (("a0z0", 0, 0), ("a1z0", 1, 0), ("a0z1", 0, 1)):
        x = x0.copy()
        L.pmgref_Vgsrb7x(nf, nf, nf, d(op7[0]), d(cc), d(f), d(op7[1]),
                         d(op7[2]), d(op7[3]), d(x), 2, iad, zi)
        out["gs7_" + name] = x
        x = x0.copy()
        L.pmgref_Vgsrb27x(nf, nf, nf, pp(op27), d(cc), d(f), d(x), 2, iad, zi)
        out["gs27_" + name] = x
    y = np.zeros(nf ** 3)
    L.pmgref_Vmatvec7_1s(nf, nf, nf, d(op7[0]), d(cc), d(op7[1]), d(op7[2]),
                         d(op7[3]), d(x0), d(y))
    out["matvec7"] = y.copy()
    y[:] = 0
    L.pmgref_Vmatvec27_1s(nf, nf, nf, pp(op27), d(cc), d(x0), d(y))
    out["matvec27"] = y.copy()
    y[:] = 0
    L.pmgref_Vmresid7_1s(nf, nf, nf, d(op7[0]), d(cc), d(f), d(op7[1]),
                         d(op7[2]), d(op7[3]), d(x0), d(y))
    out["mresid7"] = y.copy()
    y[:] = 0
    L.pmgref_Vmresid27_1s(nf, nf, nf, pp(op27), d(cc), d(f), d(x0), d(y))
    out["mresid27"] = y.copy()
    # prolongation / Galerkin builders
    P7 = [np.zeros(nc ** 3) for _ in range(27)]
    L.pmgref_VbuildPb_op7(nf, nf, nf, nc, nc, nc, d(op7[0]), d(op7[1]),
                          d(op7[2]), d(op7[3]), pp(P7))
    out["P_op7"] = np.stack(P7)
    P27 = [np.zeros(nc ** 3) for _ in range(27)]
    L.pmgref_VbuildPb_op27(nf, nf, nf, nc, nc, nc, pp(op27), pp(P27))
    out["P_op27"] = np.stack(P27)
    Pt = [np.zeros(nc ** 3) for _ in range(27)]
    L.pmgref_VbuildPb_trilin(nf, nf, nf, nc, nc, nc, pp(Pt))
    out["P_trilin"] = np.stack(Pt)
    Prand = [rng.uniform(0.05, 1.0, nc ** 3) for _ in range(27)]
    out["P_rand"] = np.stack(Prand)
    G7 = [np.zeros(nc ** 3) for _ in range(14)]
    L.pmgref_VbuildG_7(nf, nf, nf, nc, nc, nc, pp(Prand), d(op7[0]),
                       d(op7[1]), d(op7[2]), d(op7[3]), pp(G7))
    out["G7"] = np.stack(G7)
    G27 = [np.zeros(nc ** 3) for _ in range(14)]
    L.pmgref_VbuildG_27(nf, nf, nf, nc, nc, nc, pp(Prand), pp(op27), pp(G27))
    out["G27"] = np.stack(G27)
    # transfers
    xc = rng.normal(0.0, 1.0, nc ** 3)
    e = np.zeros(nf ** 3)
    L.pmgref_VinterpPMG2(nc, nc, nc, nf, nf, nf, d(xc), d(e), pp(Prand))
    out["xc"] = xc
    out["interp"] = e
    rc_ = np.zeros(nc ** 3)
    L.pmgref_Vrestrc2(nf, nf, nf, nc, nc, nc, d(x0), d(rc_), pp(Prand))
    out["restrict"] = rc_
    np.savez_compressed(os.path.join(OUT, "kernels_n9.npz"), **out)


def problems(ref: Reference) -> None:
    # set-up from atoms at the reference's constants, then hierarchy and
    # solve on the same grid: (base 2, nlev 3) = 17^3 and (4, 3) = 33^3
    for base, nlev, box, natoms, seed in ((2, 3, 8.0, 12, 11),
                                          (4, 3, 16.0, 40, 12)):
        n = base * 2 ** nlev + 1
        atoms = synthetic_atoms(natoms, box / 5, seed, (box / 2,) * 3)
        fine = ref.setup(base, nlev, atoms, 0.15, 2.0)
        x, cycles, hist = ref.solve(base, nlev, fine, tol=1e-10,
                                    max_cycles=60)
        xt, ct, ht = ref.solve(base, nlev, fine, tol=1e-10, max_cycles=60,
                               trilinear=True)
        hier = ref.hierarchy(base, nlev, fine)
        out = dict(base=base, nlev=nlev, box=box, atoms=atoms,
                   ionic_strength=0.15, ion_radius=2.0, x=x, cycles=cycles,
                   hist=hist, x_trilin=xt, cycles_trilin=ct, hist_trilin=ht,
                   **{"fine_" + k: v for k, v in fine.items()})
        for L_, (P, A) in hier.items():
            out[f"P{L_}"] = P
            out[f"A{L_}"] = A
        # coarsest-level CG of the class on level 1 of this hierarchy
        P1, A1 = hier[1]
        n1 = base * 2 + 1
        rng = np.random.default_rng(seed)
        rhs = rng.normal(0.0, 1.0, n1 ** 3)
        xcg = np.zeros(n1 ** 3)
        ref.cg_level1(base, nlev, [np.ascontiguousarray(a) for a in A1], rhs,
                      xcg)
        out["cg_rhs"] = rhs
        out["cg_x"] = xcg
        np.savez_compressed(os.path.join(OUT, f"problem_b{base}n{nlev}.npz"),
                            **out)
        print(f"b{base}n{nlev}: n={n} cycles={cycles} (trilinear {ct})")


def box_inputs(rng, nx, ny, nz):
    """Inputs of the APBS box-method builder: non-uniform mesh lines,
    dielectric-like face maps, kappa and source maps, boundary values, and
    output arrays pre-filled with noise (the shell must stay untouched)."""
    def mesh(n):
        return np.cumsum(rng.uniform(0.3, 0.7, n)) - 5.0
    return dict(
        nx=nx, ny=ny, nz=nz, ipkey=3,
        xf=mesh(nx), yf=mesh(ny), zf=mesh(nz),
        gxcf=rng.normal(0.0, 1.0, ny * nz * 2),
        gycf=rng.normal(0.0, 1.0, nx * nz * 2),
        gzcf=rng.normal(0.0, 1.0, nx * ny * 2),
        a1cf=rng.uniform(2.0, 80.0, nx * ny * nz),
        a2cf=rng.uniform(2.0, 80.0, nx * ny * nz),
        a3cf=rng.uniform(2.0, 80.0, nx * ny * nz),
        ccf=rng.uniform(0.0, 0.5, nx * ny * nz),
        fcf=rng.normal(0.0, 1.0, nx * ny * nz),
        init=rng.normal(0.0, 1.0, (6, nx * ny * nz)))


def box_operator(ref: Reference) -> None:
    """VbuildA_fv (pmgc/buildAd.cc:63-212) on a cube and on a grid with
    nx != ny (the reference's launch takes its k extent from ny, so nz ==
    ny keeps every plane built)."""
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)

    def d(a):
        return a.ctypes.data_as(D)

    rng = np.random.default_rng(20261204)
    out = {}
    for tag, (nx, ny, nz) in (("c9", (9, 9, 9)), ("r11", (11, 9, 9))):
        c = box_inputs(rng, nx, ny, nz)
        o = c["init"].copy()
        ipc = (ctypes.c_int * 12)()
        numdia = ctypes.c_int(-1)
        ref.lib.pmgref_VbuildA_fv(
            nx, ny, nz, c["ipkey"], ctypes.byref(numdia), ipc,
            *[d(o[s]) for s in range(6)],
            *[d(c[k]) for k in ("xf", "yf", "zf", "gxcf", "gycf", "gzcf",
                                "a1cf", "a2cf", "a3cf", "ccf", "fcf")])
        for k, v in c.items():
            out[f"{tag}_{k}"] = v
        out[f"{tag}_out"] = o  # oC cc fc oE oN uC
        out[f"{tag}_ipc"] = np.array(ipc[:], dtype=np.int32)
        out[f"{tag}_numdia"] = numdia.value
    np.savez_compressed(os.path.join(OUT, "buildA_fv.npz"), **out)


def zero_shell_op(rng, n, kind):
    """Symmetric positive definite operator with zero coefficients on the
    shell (as operators built on the interior have them)."""
    a = [rng.uniform(0.5, 2.0, n ** 3) for _ in range(4 if kind == 7 else 14)]
    a[0] = rng.uniform(60.0, 80.0, n ** 3)
    shell = np.ones((n, n, n), bool)
    shell[1:-1, 1:-1, 1:-1] = False
    for v in a:
        v.reshape(n, n, n)[shell] = 0.0
    return a


def band(ref: Reference) -> None:
    """The reference's banded coarse solver (buildBd.cc, mlinpckd.cc): its
    Vbuildband (band storage + Vdpbfa) of a 7-point operator, and its Vdpbfa
    and Vdpbsl on the band of a 27-point operator stored by the
    restatement (whose 27-point band keeps the matvec's couplings)."""
    import ctypes
    from oracle.oracle import Restatement
    D = ctypes.POINTER(ctypes.c_double)

    def d(a):
        return a.ctypes.data_as(D)

    rng = np.random.default_rng(20261205)
    n = 7
    mx = n - 2
    out = dict(n=n)
    a7 = zero_shell_op(rng, n, 7)
    ac = np.ascontiguousarray(np.stack(a7).ravel())
    m = mx * mx
    acB = np.zeros((m + 1) * mx ** 3)
    ipcB = (ctypes.c_int * 4)()
    key = ref.lib.pmgref_Vbuildband(n, n, n, 7, d(ac), ipcB, d(acB))
    b = rng.normal(size=mx ** 3)
    x = b.copy()
    ref.lib.pmgref_Vdpbsl(d(acB), m + 1, mx ** 3, m, d(x))
    out.update(op7=np.stack(a7), band7=acB, ipcB7=np.array(ipcB[:]),
               key7=key, b7=b, x7=x)
    a27 = zero_shell_op(rng, n, 27)
    abd, nb, m, lda = Restatement().buildband(n, a27)
    fac = abd.copy()
    info = ref.lib.pmgref_Vdpbfa(d(fac), lda, nb, m)
    b = rng.normal(size=nb)
    x = b.copy()
    ref.lib.pmgref_Vdpbsl(d(fac), lda, nb, m, d(x))
    out.update(op27=np.stack(a27), band27=abd, fac27=fac, info27=info,
               b27=b, x27=x)
    np.savez_compressed(os.path.join(OUT, "band.npz"), **out)


GROUPS = {"kernels": kernels, "problems": problems,
          "box_operator": box_operator, "band": band}

if __name__ == "__main__":
    ref = Reference()
    for name in sys.argv[1:] or list(GROUPS):
        GROUPS[name](ref)
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
