"""Python access to the PMG oracle (TEST INFRASTRUCTURE ONLY).

Two CPU implementations of the reference algorithm, used as checkers by
tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py:

* ``Restatement`` — oracle/pmg_oracle.c, a plain-C restatement of the
  reference PMG path (libpmg_oracle.so, built from this repository).
* ``Reference``   — the reference's own PBE_pmgc_class.h and pmgc kernels
  compiled against the host SYCL shim (oracle/_ref/libpmgc_ref*.so, built by
  oracle/Makefile from the reference sources where they are available).

The product (multigrid_b200) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
D = ctypes.POINTER(ctypes.c_double)
PP = ctypes.POINTER(ctypes.POINTER(ctypes.c_double))

OP14 = ("oC", "oE", "oN", "uC", "oNE", "oNW", "uE", "uW", "uN", "uS", "uNE",
        "uNW", "uSE", "uSW")


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(D)


def _pp(arrs):
    return (D * len(arrs))(*[_d(a) for a in arrs])


def build_restatement() -> str:
    """Compiles oracle/pmg_oracle.c (make -C oracle restatement)."""
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    return os.path.join(HERE, "libpmg_oracle.so")


class _PmgoOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("a", D * 14)]


class Restatement:
    """oracle/pmg_oracle.c through ctypes (numpy float64 arrays)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "libpmg_oracle.so")
        if not os.path.exists(path):
            path = build_restatement()
        self.lib = L = ctypes.CDLL(path)
        L.pmgo_solve.restype = ctypes.c_int
        L.pmgo_hierarchy.restype = ctypes.c_long
        L.pmgo_residual2.restype = ctypes.c_double
        L.pmgo_ideal_lambda.restype = ctypes.c_double
        L.pmgo_cg.restype = ctypes.c_int
        L.pmgo_pcg.restype = ctypes.c_int
        L.pmgo_pcg.argtypes = [ctypes.c_int, ctypes.c_int] + [D] * 6 + [
            ctypes.c_int, ctypes.c_double, D, D]
        L.pmgo_solve.argtypes = [ctypes.c_int, ctypes.c_int] + [D] * 6 + [
            ctypes.c_double, ctypes.c_int, ctypes.c_int, D, D]
        L.pmgo_hierarchy.argtypes = [ctypes.c_int, ctypes.c_int] + [D] * 4 + [
            ctypes.c_int, D, ctypes.c_long]
        L.pmgo_residual2.argtypes = [ctypes.c_int] * 3 + [
            ctypes.POINTER(_PmgoOp), D, D]
        L.pmgo_ideal_lambda.argtypes = [ctypes.c_int] * 3 + [
            ctypes.POINTER(_PmgoOp), D, D]
        L.pmgo_cg.argtypes = [ctypes.c_int] * 3 + [
            ctypes.POINTER(_PmgoOp), D, D, ctypes.c_double]

    @staticmethod
    def op(arrays) -> _PmgoOp:
        kind = 7 if len(arrays) == 4 else 27
        ptrs = [_d(a) for a in arrays] + [None] * (14 - len(arrays))
        return _PmgoOp(kind, (D * 14)(*ptrs))

    def gsrb7x(self, n, oC, cc, fc, oE, oN, uC, x, itmax=1, iadjoint=0,
               zero_init=False):
        self.lib.pmgo_gsrb7x(n, n, n, _d(oC), _d(cc), _d(fc), _d(oE), _d(oN),
                             _d(uC), _d(x), itmax, iadjoint, int(zero_init))

    def gsrb27x(self, n, op14, cc, fc, x, itmax=1, iadjoint=0,
                zero_init=False):
        self.lib.pmgo_gsrb27x(n, n, n, _pp(op14), _d(cc), _d(fc), _d(x),
                              itmax, iadjoint, int(zero_init))

    def matvec(self, n, ops, cc, x, y):
        o = self.op(ops)
        self.lib.pmgo_matvec(n, n, n, ctypes.byref(o),
                             _d(cc) if cc is not None else None, _d(x), _d(y))

    def mresid(self, n, ops, cc, fc, x, r):
        o = self.op(ops)
        self.lib.pmgo_mresid(n, n, n, ctypes.byref(o),
                             _d(cc) if cc is not None else None, _d(fc),
                             _d(x), _d(r))

    def restrc2(self, nf, nc, xin, xout, p27):
        self.lib.pmgo_restrc2(nf, nf, nf, nc, nc, nc, _d(xin), _d(xout),
                              _pp(p27))

    def interp2(self, nc, nf, xin, xout, p27):
        self.lib.pmgo_interp2(nc, nc, nc, nf, nf, nf, _d(xin), _d(xout),
                              _pp(p27))

    def buildP_op(self, nf, nc, ops, p27):
        o = self.op(ops)
        self.lib.pmgo_buildP_op(nf, nf, nf, nc, nc, nc, ctypes.byref(o),
                                _pp(p27))

    def buildP_trilin(self, nc, p27):
        self.lib.pmgo_buildP_trilin(nc, nc, nc, _pp(p27))

    def cghs(self, nx, ny, nz, ops, cc, fc, x, itmax, errtol, iresid=0):
        """APBS CG (Vcghs) from x (updated in place); returns (iters, r)."""
        o = self.op(ops)
        n3 = nx * ny * nz
        p, ap, r = np.zeros(n3), np.zeros(n3), np.zeros(n3)
        self.lib.pmgo_cghs.argtypes = [ctypes.c_int] * 3 + [
            ctypes.POINTER(_PmgoOp)] + [D] * 6 + [ctypes.c_int,
                                                  ctypes.c_double,
                                                  ctypes.c_int]
        it = self.lib.pmgo_cghs(nx, ny, nz, ctypes.byref(o), _d(cc), _d(fc),
                                _d(x), _d(p), _d(ap), _d(r), int(itmax),
                                float(errtol), int(iresid))
        return it, r

    def mgdriv(self, iparm, rparm, u, maps, tcf=None):
        """APBS driver (linear); iparm/rparm 0-based sequences, u updated in
        place, maps: dict of BOX_IN arrays. Returns (iters, ierror,
        final stop ratio)."""
        ip = (ctypes.c_int * len(iparm))(*iparm)
        rp = (ctypes.c_double * len(rparm))(*rparm)
        it, ie, rs = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self.lib.pmgo_mgdriv.restype = ctypes.c_int
        rc = self.lib.pmgo_mgdriv(ip, rp, _d(u),
                                  *[_d(maps[k]) for k in self.BOX_IN],
                                  _d(tcf) if tcf is not None else None,
                                  ctypes.byref(it), ctypes.byref(ie),
                                  ctypes.byref(rs))
        if rc != 0:
            raise RuntimeError(f"pmgo_mgdriv returned {rc}")
        return it.value, ie.value, rs.value

    def buildband(self, n, ops):
        """Band storage of the interior operator (not yet factored);
        returns (abd, nb, m, lda)."""
        o = self.op(ops)
        mx = n - 2
        m = mx * mx if len(ops) == 4 else mx * mx + mx + 1
        abd = np.zeros((m + 1) * mx ** 3)
        nn, mm, ll = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.pmgo_buildband(n, n, n, ctypes.byref(o), ctypes.byref(nn),
                                ctypes.byref(mm), ctypes.byref(ll), _d(abd))
        return abd, nn.value, mm.value, ll.value

    def dpbfa(self, abd, lda, n, m):
        self.lib.pmgo_dpbfa.restype = ctypes.c_int
        return self.lib.pmgo_dpbfa(_d(abd), lda, n, m)

    def dpbsl(self, abd, lda, n, m, b):
        self.lib.pmgo_dpbsl(_d(abd), lda, n, m, _d(b))

    BOX_IN = ("xf", "yf", "zf", "gxcf", "gycf", "gzcf", "a1cf", "a2cf",
              "a3cf", "ccf", "fcf")

    def buildA_fv(self, nx, ny, nz, ipkey, inputs, out6):
        """Box-method fine builder; inputs: dict of BOX_IN arrays, out6:
        oC cc fc oE oN uC (written on the interior). Returns (ipc,
        numdia)."""
        ipc = (ctypes.c_int * 12)()
        numdia = ctypes.c_int(-1)
        self.lib.pmgo_buildA_fv(nx, ny, nz, ipkey, ctypes.byref(numdia), ipc,
                                *[_d(a) for a in out6],
                                *[_d(inputs[k]) for k in self.BOX_IN])
        return np.array(ipc[:], dtype=np.int32), numdia.value

    def buildG(self, nf, nc, p27, ops, out14):
        o = self.op(ops)
        self.lib.pmgo_buildG(nf, nf, nf, nc, nc, nc, _pp(p27),
                             ctypes.byref(o), _pp(out14))

    def defect(self, n, ops, f, x, r):
        o = self.op(ops)
        self.lib.pmgo_defect(n, n, n, ctypes.byref(o), _d(f), _d(x), _d(r))

    def residual2(self, n, ops, f, x) -> float:
        o = self.op(ops)
        return self.lib.pmgo_residual2(n, n, n, ctypes.byref(o), _d(f), _d(x))

    def ideal_lambda(self, n, ops, x, r) -> float:
        o = self.op(ops)
        return self.lib.pmgo_ideal_lambda(n, n, n, ctypes.byref(o), _d(x),
                                          _d(r))

    def setup_fine(self, n: int, h: float, atoms: np.ndarray,
                   physics: dict) -> dict:
        """Fine-level arrays (oC, oE, oN, uC, f, x0) from atoms with the
        restated set-up (pmg_oracle_setup.c); physics as the product's dict
        (eps_in, eps_out, ionic_strength, ion_radius, temperature,
        probe_radius)."""
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        out = {k: np.empty(n ** 3) for k in ("oC", "oE", "oN", "uC", "f",
                                             "x0")}
        L = self.lib
        L.pmgo_setup_fine.restype = ctypes.c_int
        L.pmgo_setup_fine.argtypes = [ctypes.c_int, ctypes.c_double, D,
                                      ctypes.c_int] + [ctypes.c_double] * 6 \
            + [D] * 6
        rc = L.pmgo_setup_fine(
            n, h, _d(atoms), int(atoms.shape[0]), physics["eps_in"],
            physics["eps_out"], physics["ionic_strength"],
            physics["ion_radius"], physics["temperature"],
            physics.get("probe_radius", 0.0),
            *[_d(out[k]) for k in ("oC", "oE", "oN", "uC", "f", "x0")])
        if rc != 0:
            raise ValueError(f"pmgo_setup_fine returned {rc}")
        return out

    def cg(self, n, op14, rhs, x, thresh=1e-8) -> int:
        o = self.op(op14)
        return self.lib.pmgo_cg(n, n, n, ctypes.byref(o), _d(rhs), _d(x),
                                thresh)

    def solve(self, base, nlev, fine: dict, tol=1e-10, max_cycles=100,
              trilinear=False):
        n = base * 2 ** nlev + 1
        x = np.empty(n ** 3)
        hist = np.zeros(max_cycles + 1)
        args = [_d(np.ascontiguousarray(fine[k], dtype=np.float64).ravel())
                for k in ("oC", "oE", "oN", "uC", "f", "x0")]
        c = self.lib.pmgo_solve(base, nlev, *args, tol, max_cycles,
                                int(trilinear), _d(x), _d(hist))
        if c < 0:
            raise MemoryError("pmgo_solve: allocation failed")
        return x, c, hist[:c + 1]

    def pcg(self, base, nlev, fine: dict, max_iters, tol=0.0):
        """MG-preconditioned CG (pmgo_pcg): (x, iterations, history)."""
        n = base * 2 ** nlev + 1
        x = np.empty(n ** 3)
        hist = np.zeros(max_iters + 1)
        args = [_d(np.ascontiguousarray(fine[k], dtype=np.float64).ravel())
                for k in ("oC", "oE", "oN", "uC", "f", "x0")]
        c = self.lib.pmgo_pcg(base, nlev, *args, max_iters, tol, _d(x),
                              _d(hist))
        if c < 0:
            raise MemoryError("pmgo_pcg: allocation failed")
        return x, c, hist[:c + 1]

    def hierarchy(self, base, nlev, fine: dict, trilinear=False):
        cap = sum(41 * (base * 2 ** L + 1) ** 3 for L in range(1, nlev))
        out = np.empty(cap)
        args = [_d(np.ascontiguousarray(fine[k], dtype=np.float64).ravel())
                for k in ("oC", "oE", "oN", "uC")]
        got = self.lib.pmgo_hierarchy(base, nlev, *args, int(trilinear),
                                      _d(out), cap)
        if got != cap:
            raise RuntimeError("pmgo_hierarchy failed")
        return split_hierarchy(out, base, nlev)


def split_hierarchy(flat: np.ndarray, base: int, nlev: int) -> dict:
    """{L: (P (27, n_L^3), A (14, n_L^3))} from the flat hierarchy layout."""
    out, off = {}, 0
    for L in range(nlev - 1, 0, -1):
        n3 = (base * 2 ** L + 1) ** 3
        blk = flat[off:off + 41 * n3].reshape(41, n3)
        out[L] = (blk[:27], blk[27:])
        off += 41 * n3
    return out


class _RefFine(ctypes.Structure):
    _fields_ = [(k, D) for k in ("oC", "oE", "oN", "uC", "f", "x0")]


def reference_tree() -> str | None:
    """The reference tree oracle/_ref was built from, when it is present on
    this machine (its data files, e.g. the PQR inputs); else None."""
    try:
        with open(os.path.join(HERE, "_ref", "reference_dir.txt")) as f:
            path = f.read().strip()
    except OSError:
        return None
    return path if path and os.path.isdir(path) else None


def reference_available(omp: bool = False) -> bool:
    name = "libpmgc_ref_omp.so" if omp else "libpmgc_ref.so"
    return os.path.exists(os.path.join(HERE, "_ref", name))


class Reference:
    """The reference's own PMG class and kernels (oracle/_ref)."""

    def __init__(self, omp: bool = False):
        name = "libpmgc_ref_omp.so" if omp else "libpmgc_ref.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} not built (make -C oracle needs the reference tree)")
        self.lib = L = ctypes.CDLL(path)
        L.pmgref_hierarchy.restype = ctypes.c_long
        self._keep = []

    def configs(self):
        b = (ctypes.c_int * 64)()
        nl = (ctypes.c_int * 64)()
        bx = (ctypes.c_double * 64)()
        cnt = self.lib.pmgref_configs(b, nl, bx, 64)
        return [(b[i], nl[i], bx[i]) for i in range(cnt)]

    def _fine(self, fine: dict):
        arrs = [np.ascontiguousarray(fine[k], dtype=np.float64).ravel()
                for k in ("oC", "oE", "oN", "uC", "f", "x0")]
        self._keep = arrs
        return _RefFine(*[_d(a) for a in arrs])

    def solve(self, base, nlev, fine: dict, tol=1e-10, max_cycles=100,
              trilinear=False):
        n = base * 2 ** nlev + 1
        x = np.empty(n ** 3)
        hist = np.zeros(max_cycles + 1)
        c = ctypes.c_int()
        f = self._fine(fine)
        rc = self.lib.pmgref_solve(base, nlev, ctypes.byref(f),
                                   ctypes.c_double(tol), max_cycles,
                                   int(trilinear), _d(x), _d(hist),
                                   ctypes.byref(c))
        if rc != 0:
            raise KeyError(f"reference oracle has no ({base}, {nlev}) grid")
        return x, c.value, hist[:c.value + 1]

    def pcg(self, base, nlev, fine: dict, iters: int):
        """The app's MG-preconditioned CG for exactly `iters` iterations
        (pmgref_pcg); returns the iterate."""
        n = base * 2 ** nlev + 1
        x = np.empty(n ** 3)
        f = self._fine(fine)
        rc = self.lib.pmgref_pcg(base, nlev, ctypes.byref(f), iters, _d(x))
        if rc != 0:
            raise KeyError(f"reference oracle has no ({base}, {nlev}) grid")
        return x

    def cycles(self, base, nlev, fine: dict, ncycles: int):
        n = base * 2 ** nlev + 1
        x = np.empty(n ** 3)
        f = self._fine(fine)
        rc = self.lib.pmgref_cycles(base, nlev, ctypes.byref(f), ncycles,
                                    _d(x))
        if rc != 0:
            raise KeyError(f"reference oracle has no ({base}, {nlev}) grid")
        return x

    def hierarchy(self, base, nlev, fine: dict, trilinear=False):
        cap = sum(41 * (base * 2 ** L + 1) ** 3 for L in range(1, nlev))
        out = np.empty(cap)
        f = self._fine(fine)
        got = self.lib.pmgref_hierarchy(base, nlev, ctypes.byref(f),
                                        int(trilinear), _d(out),
                                        ctypes.c_long(cap))
        if got != cap:
            raise KeyError(f"reference oracle has no ({base}, {nlev}) grid")
        return split_hierarchy(out, base, nlev)

    def cg_level1(self, base, nlev, op14, rhs, x):
        rc = self.lib.pmgref_cg_level1(base, nlev, _pp(op14), _d(rhs), _d(x))
        if rc != 0:
            raise KeyError(f"reference oracle has no ({base}, {nlev}) grid")

    def read_pqr(self, path: str, cap: int = 1 << 20) -> np.ndarray:
        """The reference's PQR reader: rows (x, y, z, radius, charge)."""
        atoms = np.empty((cap, 5))
        n = ctypes.c_int()
        rc = self.lib.pmgref_read_pqr(path.encode(), _d(atoms), cap,
                                      ctypes.byref(n))
        if rc != 0:
            raise ValueError("more atoms than cap")
        return atoms[:n.value].copy()

    DX_SHAPES = {0: (4, 5, 6), 1: (7, 7, 7)}

    def write_dx(self, shape: int, values: np.ndarray, origin, box) -> str:
        """The reference's OpenDX text of a grid of DX_SHAPES[shape] interior
        points (slowest axis first) with a one-point padding (oracle/_ref/
        ref_dx, a separate process)."""
        import tempfile
        exe = os.path.join(HERE, "_ref", "ref_dx")
        with tempfile.NamedTemporaryFile(suffix=".bin") as f:
            np.ascontiguousarray(values, dtype="<f8").tofile(f.name)
            r = subprocess.run([exe, str(shape), f.name] +
                               [repr(float(v)) for v in origin] +
                               [repr(float(box))], capture_output=True,
                               check=True)
        return r.stdout.decode()

    def setup(self, base, nlev, atoms, ionic_strength, ion_radius) -> dict:
        n = base * 2 ** nlev + 1
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        out = {k: np.empty(n ** 3) for k in ("oC", "oE", "oN", "uC", "f",
                                             "x0")}
        rc = self.lib.pmgref_setup(
            base, nlev, _d(atoms), int(atoms.shape[0]),
            ctypes.c_double(ionic_strength), ctypes.c_double(ion_radius),
            *[_d(out[k]) for k in ("oC", "oE", "oN", "uC", "f", "x0")])
        if rc != 0:
            raise KeyError(f"reference oracle has no ({base}, {nlev}) grid")
        return out
