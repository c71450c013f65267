"""The pmgc kernels under the reference's names, on torch CUDA tensors.

Each function calls the matching C-ABI entry point of libpmg_b200.so with the
tensors' device pointers and the current torch stream (or `stream`), in the
reference's argument order minus the unused APBS arguments (ipc, rpc) and
with the sycl::queue replaced by a stream. Arrays are flat, n^3 long, with
the reference's layout (x fastest, one-point shell). cc may be None (zero).

  Vgsrb7x        pmgc/gsd.cc:60-111        Vgsrb27x     pmgc/gsd.cc:113-212
  Vmatvec7_1s    pmgc/matvecd.cc:61-90     Vmatvec27_1s pmgc/matvecd.cc:103-176
  Vmresid7_1s    pmgc/matvecd.cc:381-411   Vmresid27_1s pmgc/matvecd.cc:425-495
  Vrestrc2       pmgc/matvecd.cc:695-799   VinterpPMG2  pmgc/matvecd.cc:819-964
  VbuildPb_op7   pmgc/buildPd.cc:172-555   VbuildPb_op27 pmgc/buildPd.cc:578-1091
  VbuildPb_trilin pmgc/buildPd.cc:62-153   VbuildG_7    pmgc/buildGd.cc:437-1361
  VbuildG_27     pmgc/buildGd.cc:1363-3274
  VbuildA_fv     pmgc/buildAd.cc:63-212
  Vmatvec        pmgc/matvecd.cc:244-260   Vmresid      pmgc/matvecd.cc:513-529
  Vcghs          pmgc/cgd.cc:60-125 (packed operators, APBS layer)
  Vmgdriv        pmgc/mgdrvd.cc:60-491 with Vbuildops and Vmvcs (linear)
  Vbuildband     pmgc/buildBd.cc:252-303   Vdpbfa, Vdpbsl pmgc/mlinpckd.cc
  cg_level       CG_Solver.h:45-242 as run by PBE_pmgc_class.h:856-860
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

OP14 = ("oC", "oE", "oN", "uC", "oNE", "oNW", "uE", "uW", "uN", "uS", "uNE",
        "uNW", "uSE", "uSW")
P27 = ("oPC", "oPN", "oPS", "oPE", "oPW", "oPNE", "oPNW", "oPSE", "oPSW",
       "uPC", "uPN", "uPS", "uPE", "uPW", "uPNE", "uPNW", "uPSE", "uPSW",
       "dPC", "dPN", "dPS", "dPE", "dPW", "dPNE", "dPNW", "dPSE", "dPSW")


def _p(t):
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("pmgc kernels take CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("pmgc kernels take contiguous tensors")
    return ctypes.c_void_p(t.data_ptr())


def _s(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(getattr(stream, "cuda_stream", stream))


def _sfx(t):
    if t.dtype == torch.float64:
        return "_d"
    if t.dtype == torch.float32:
        return "_f"
    raise TypeError("float32 or float64 tensors only")


def _pp(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def Vgsrb7x(nx, ny, nz, oC, cc, fc, oE, oN, uC, x, itmax, iadjoint=0,
            zero_init=False, stream=None):
    _lib.call("pmg_Vgsrb7x" + _sfx(x), nx, ny, nz, _p(oC), _p(cc), _p(fc),
              _p(oE), _p(oN), _p(uC), _p(x), int(itmax), int(iadjoint),
              int(zero_init), _s(stream))


def Vgsrb27x(nx, ny, nz, op14, cc, fc, x, itmax, zero_init=False, iadjoint=0,
             stream=None):
    """op14: the 14 diagonals oC..uSW (a sequence of tensors)."""
    a = [_p(t) for t in op14]
    _lib.call("pmg_Vgsrb27x" + _sfx(x), nx, ny, nz, a[0], _p(cc), _p(fc),
              *a[1:], _p(x), int(itmax), int(zero_init), int(iadjoint),
              _s(stream))


def Vmatvec7_1s(nx, ny, nz, oC, cc, oE, oN, uC, x, y, stream=None):
    _lib.call("pmg_Vmatvec7_1s" + _sfx(x), nx, ny, nz, _p(oC), _p(cc),
              _p(oE), _p(oN), _p(uC), _p(x), _p(y), _s(stream))


def Vmatvec27_1s(nx, ny, nz, op14, cc, x, y, stream=None):
    a = [_p(t) for t in op14]
    _lib.call("pmg_Vmatvec27_1s" + _sfx(x), nx, ny, nz, a[0], _p(cc),
              *a[1:], _p(x), _p(y), _s(stream))


def Vmresid7_1s(nx, ny, nz, oC, cc, fc, oE, oN, uC, x, r, stream=None):
    _lib.call("pmg_Vmresid7_1s" + _sfx(x), nx, ny, nz, _p(oC), _p(cc),
              _p(fc), _p(oE), _p(oN), _p(uC), _p(x), _p(r), _s(stream))


def Vmresid27_1s(nx, ny, nz, op14, cc, fc, x, r, stream=None):
    a = [_p(t) for t in op14]
    _lib.call("pmg_Vmresid27_1s" + _sfx(x), nx, ny, nz, a[0], _p(cc),
              _p(fc), *a[1:], _p(x), _p(r), _s(stream))


def Vrestrc2(nxf, nyf, nzf, nxc, nyc, nzc, xin, xout, p27, stream=None):
    _lib.call("pmg_Vrestrc2" + _sfx(xin), nxf, nyf, nzf, nxc, nyc, nzc,
              _p(xin), _p(xout), *[_p(t) for t in p27], _s(stream))


def VinterpPMG2(nxc, nyc, nzc, nxf, nyf, nzf, xin, xout, p27, stream=None):
    _lib.call("pmg_VinterpPMG2" + _sfx(xin), nxc, nyc, nzc, nxf, nyf, nzf,
              _p(xin), _p(xout), *[_p(t) for t in p27], _s(stream))


def VbuildPb_op7(nxf, nyf, nzf, nxc, nyc, nzc, oC, oE, oN, uC, p27,
                 stream=None):
    _lib.call("pmg_VbuildPb_op7_d", nxf, nyf, nzf, nxc, nyc, nzc, _p(oC),
              _p(oE), _p(oN), _p(uC), *[_p(t) for t in p27], _s(stream))


def VbuildPb_op27(nxf, nyf, nzf, nxc, nyc, nzc, op14, p27, stream=None):
    _lib.call("pmg_VbuildPb_op27_d", nxf, nyf, nzf, nxc, nyc, nzc,
              *[_p(t) for t in op14], *[_p(t) for t in p27], _s(stream))


def VbuildPb_trilin(nxf, nyf, nzf, nxc, nyc, nzc, p27, stream=None):
    _lib.call("pmg_VbuildPb_trilin_d", nxf, nyf, nzf, nxc, nyc, nzc,
              *[_p(t) for t in p27], _s(stream))


def VbuildA_fv(nx, ny, nz, ipkey, oC, cc, fc, oE, oN, uC, xf, yf, zf, gxcf,
               gycf, gzcf, a1cf, a2cf, a3cf, ccf, fcf, stream=None):
    """Box-method fine operator (outputs oC..uC written on the interior).
    Returns (ipc, numdia): the 12-int bookkeeping array (ipc[9..11] =
    ipkey, 7, 1) and the stored-diagonal count 4."""
    ipc = (ctypes.c_int * 12)()
    numdia = ctypes.c_int(-1)
    _lib.call("pmg_VbuildA_fv_d", nx, ny, nz, int(ipkey),
              ctypes.byref(numdia), ipc,
              *[_p(t) for t in (oC, cc, fc, oE, oN, uC, xf, yf, zf, gxcf,
                                gycf, gzcf, a1cf, a2cf, a3cf, ccf, fcf)],
              _s(stream))
    return list(ipc), numdia.value


def VbuildG_7(nxf, nyf, nzf, nxc, nyc, nzc, p27, oC, oE, oN, uC, out14,
              stream=None):
    _lib.call("pmg_VbuildG_7_d", nxf, nyf, nzf, nxc, nyc, nzc, _pp(p27),
              _p(oC), _p(oE), _p(oN), _p(uC), _pp(out14), _s(stream))


def VbuildG_27(nxf, nyf, nzf, nxc, nyc, nzc, p27, op14, out14, stream=None):
    _lib.call("pmg_VbuildG_27_d", nxf, nyf, nzf, nxc, nyc, nzc, _pp(p27),
              _pp(op14), _pp(out14), _s(stream))


def _packed(ac):
    """ac: a contiguous (4 or 14, n^3) tensor of diagonals -> ipc, pointer."""
    if ac.dim() != 2 or ac.shape[0] not in (4, 14):
        raise ValueError("ac must have 4 (7-point) or 14 (27-point) rows")
    ipc = (ctypes.c_int * 12)()
    ipc[10] = 7 if ac.shape[0] == 4 else 27
    return ipc, _p(ac)


def Vmatvec(nx, ny, nz, ac, cc, x, y, stream=None):
    """y = A x with the packed operator ac (rows oC oE oN uC [oNE .. uSW])."""
    ipc, a = _packed(ac)
    _lib.call("pmg_Vmatvec_d", nx, ny, nz, ipc, a, _p(cc), _p(x), _p(y),
              _s(stream))


def Vmresid(nx, ny, nz, ac, cc, fc, x, r, stream=None):
    ipc, a = _packed(ac)
    _lib.call("pmg_Vmresid_d", nx, ny, nz, ipc, a, _p(cc), _p(fc), _p(x),
              _p(r), _s(stream))


def Vcghs(nx, ny, nz, ac, cc, fc, x, p, ap, r, itmax, errtol, iresid=0,
          stream=None):
    """APBS conjugate gradient from x (updated); returns the iterations."""
    ipc, a = _packed(ac)
    it = ctypes.c_int(-1)
    _lib.call("pmg_Vcghs_d", nx, ny, nz, ipc, a, _p(cc), _p(fc), _p(x),
              _p(p), _p(ap), _p(r), int(itmax), ctypes.byref(it),
              ctypes.c_double(errtol), int(iresid), _s(stream))
    return it.value


def Vbuildband(nx, ny, nz, ac, acB, stream=None):
    """Band storage and factorisation of the packed operator ac into acB;
    returns (key, [n, m, lda, 1])."""
    ipc, a = _packed(ac)
    key = ctypes.c_int(-1)
    ipcB = (ctypes.c_int * 4)()
    _lib.call("pmg_Vbuildband_d", ctypes.byref(key), nx, ny, nz, ipc, a,
              ipcB, _p(acB), _s(stream))
    return key.value, list(ipcB)


def Vdpbfa(abd, lda, n, m, stream=None):
    info = ctypes.c_int(-1)
    _lib.call("pmg_Vdpbfa_d", _p(abd), lda, n, m, ctypes.byref(info),
              _s(stream))
    return info.value


def Vdpbsl(abd, lda, n, m, b, stream=None):
    _lib.call("pmg_Vdpbsl_d", _p(abd), lda, n, m, _p(b), _s(stream))


def Vmgdriv(iparm, rparm, u, xf, yf, zf, gxcf, gycf, gzcf, a1cf, a2cf, a3cf,
            ccf, fcf, tcf=None, stream=None):
    """APBS driver (linear): iparm / rparm are 0-based sequences in the
    reference's order; u (n^3) gets the solution with its boundary values.
    Returns (cycles, ierror, final stop ratio)."""
    ip = (ctypes.c_int * max(len(iparm), 25))(*iparm)
    rp = (ctypes.c_double * max(len(rparm), 12))(*rparm)
    it, ie, rs = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    _lib.call("pmg_Vmgdriv_d", ip, rp, _p(u),
              *[_p(t) for t in (xf, yf, zf, gxcf, gycf, gzcf, a1cf, a2cf,
                                a3cf, ccf, fcf)],
              _p(tcf) if tcf is not None else None, ctypes.byref(it),
              ctypes.byref(ie), ctypes.byref(rs), _s(stream))
    return it.value, ie.value, rs.value


def Vmvcs(nx, ny, nz, x, iz, w0, w1, w2, w3, istop, itmax, nlev, ipc, pc,
          ac, cc, fc, tru=None, ilev=1, nlev_real=None, mgsolv=0,
          epsiln=0.0, errtol=1e-10, nu1=2, nu2=2, mgsmoo=1, stream=None):
    """APBS V-cycle loop on a packed hierarchy the caller built: iz is the
    Vbuildstr table (50 x nlev_real ints, column-major, 1-based offsets),
    ipc the packed host integer parameters (100 per level); x, w0, pc, ac,
    cc, fc, tru packed device arrays, w1..w3 finest-size work. Returns
    (cycles, ierror)."""
    nlev_real = nlev_real or nlev
    izc = (ctypes.c_int * len(iz))(*[int(v) for v in iz])
    ipcc = (ctypes.c_int * len(ipc))(*[int(v) for v in ipc])
    it, ie = ctypes.c_int(), ctypes.c_int()
    _lib.call("pmg_Vmvcs_d", nx, ny, nz, _p(x), izc, _p(w0), _p(w1), _p(w2),
              _p(w3), int(istop), int(itmax), ctypes.byref(it),
              ctypes.byref(ie), int(nlev), int(ilev), int(nlev_real),
              int(mgsolv), 1, 0, ctypes.c_double(epsiln),
              ctypes.c_double(errtol), ctypes.c_double(1.0), int(nu1),
              int(nu2), int(mgsmoo), ipcc, None,
              _p(pc) if pc is not None else None, _p(ac), _p(cc), _p(fc),
              _p(tru) if tru is not None else None, _s(stream))
    return it.value, ie.value


def cg_level(nx, ny, nz, op14, rhs, x, thresh=1e-8, max_iters=20000,
             stream=None) -> int:
    """Coarsest-level CG of the class; returns the iteration count."""
    it = ctypes.c_int()
    _lib.call("pmg_cg_level_d", nx, ny, nz, _pp(op14), _p(rhs), _p(x),
              float(thresh), int(max_iters), ctypes.byref(it), _s(stream))
    return it.value
