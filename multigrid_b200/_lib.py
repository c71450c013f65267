"""ctypes binding of libpmg_b200.so (the C ABI in include/pmg_b200.h).

The shared library is built in-tree (python -m multigrid_b200.build). There
is no fallback: if it is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmg_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -m multigrid_b200.build`"
    )

lib = ctypes.CDLL(LIB_PATH)

c_int = ctypes.c_int
c_long = ctypes.c_long
c_ll = ctypes.c_longlong
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
PD = ctypes.POINTER(ctypes.c_double)
PF = ctypes.POINTER(ctypes.c_float)
PI = ctypes.POINTER(ctypes.c_int)

PMG_OK = 0
STATUS = {
    0: "PMG_OK", -1: "PMG_ERR_ARG", -2: "PMG_ERR_CUDA", -3: "PMG_ERR_NOMEM",
    -4: "PMG_ERR_DIVERGED", -5: "PMG_ERR_TIMEOUT", -6: "PMG_ERR_BUDGET",
    -7: "PMG_ERR_STATE",
}
globals().update({name: code for code, name in STATUS.items()})
PREC_FP64 = 0
PREC_MIXED = 1
PREC_FP64_FAST = 2


class PmgError(RuntimeError):
    """A pmg_b200 entry point returned a negative status."""

    def __init__(self, func: str, status: int):
        self.status = status
        msg = lib.pmg_last_error().decode(errors="replace")
        super().__init__(f"{func}: {STATUS.get(status, status)}: {msg}")


class PmgPhysics(ctypes.Structure):
    _fields_ = [
        ("eps_in", c_double), ("eps_out", c_double),
        ("ionic_strength", c_double), ("ion_radius", c_double),
        ("temperature", c_double), ("probe_radius", c_double),
    ]


def _sig(name: str, restype, *argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


_sig("pmg_last_error", ctypes.c_char_p)
_sig("pmg_version", ctypes.c_char_p)

_V = c_void_p  # device pointers and streams cross the ABI as void*
_GS7 = [c_int] * 3 + [_V] * 7 + [c_int] * 3 + [_V]
_sig("pmg_Vgsrb7x_d", c_int, *_GS7)
_sig("pmg_Vgsrb7x_f", c_int, *_GS7)
_GS27 = [c_int] * 3 + [_V] * 17 + [c_int] * 3 + [_V]
_sig("pmg_Vgsrb27x_d", c_int, *_GS27)
_sig("pmg_Vgsrb27x_f", c_int, *_GS27)
for _t in ("_d", "_f"):
    _sig("pmg_Vmatvec7_1s" + _t, c_int, *([c_int] * 3 + [_V] * 7 + [_V]))
    _sig("pmg_Vmatvec27_1s" + _t, c_int, *([c_int] * 3 + [_V] * 17 + [_V]))
    _sig("pmg_Vmresid7_1s" + _t, c_int, *([c_int] * 3 + [_V] * 8 + [_V]))
    _sig("pmg_Vmresid27_1s" + _t, c_int, *([c_int] * 3 + [_V] * 18 + [_V]))
    _sig("pmg_Vrestrc2" + _t, c_int, *([c_int] * 6 + [_V] * 29 + [_V]))
    _sig("pmg_VinterpPMG2" + _t, c_int, *([c_int] * 6 + [_V] * 29 + [_V]))
_sig("pmg_VbuildPb_op7_d", c_int, *([c_int] * 6 + [_V] * 31 + [_V]))
_sig("pmg_VbuildPb_op27_d", c_int, *([c_int] * 6 + [_V] * 41 + [_V]))
_sig("pmg_VbuildPb_trilin_d", c_int, *([c_int] * 6 + [_V] * 27 + [_V]))
_sig("pmg_VbuildA_fv_d", c_int, *([c_int] * 4 + [PI, PI] + [_V] * 17 + [_V]))
_sig("pmg_Vmatvec_d", c_int, *([c_int] * 3 + [PI] + [_V] * 4 + [_V]))
_sig("pmg_Vmresid_d", c_int, *([c_int] * 3 + [PI] + [_V] * 5 + [_V]))
_sig("pmg_Vcghs_d", c_int, *([c_int] * 3 + [PI] + [_V] * 7 + [c_int, PI,
                                                               c_double,
                                                               c_int, _V]))
_sig("pmg_Vmgdriv_d", c_int, PI, PD, *([_V] * 13), PI, PI, PD, _V)
_sig("pmg_Vbuildband_d", c_int, PI, c_int, c_int, c_int, PI, _V, PI, _V, _V)
_sig("pmg_Vdpbfa_d", c_int, _V, c_int, c_int, c_int, PI, _V)
_sig("pmg_Vdpbsl_d", c_int, _V, c_int, c_int, c_int, _V, _V)
_PP = ctypes.POINTER(c_void_p)
_sig("pmg_VbuildG_7_d", c_int, *([c_int] * 6 + [_PP, _V, _V, _V, _V, _PP, _V]))
_sig("pmg_VbuildG_27_d", c_int, *([c_int] * 6 + [_PP, _PP, _PP, _V]))
_sig("pmg_cg_level_d", c_int,
     *([c_int] * 3 + [_PP, _V, _V, c_double, c_int, PI, _V]))
_sig("pmg_cg_level_noalloc_d", c_int,
     *([c_int] * 3 + [_PP, _V, _V, c_double, c_int, PI, _V]))

_sig("pmg_kappa", c_int, ctypes.POINTER(PmgPhysics), PD, PD)
_sig("pmg_setup_fine", c_int, c_int, c_double, PD, c_int,
     ctypes.POINTER(PmgPhysics), PD, PD, PD, PD, PD, PD)
_sig("pmg_setup_fine_d", c_int, c_int, c_double, PD, c_int,
     ctypes.POINTER(PmgPhysics), _V, _V, _V, _V, _V, _V, _V)
_sig("pmg_problem_set_atoms", c_int, _V, PD, c_int,
     ctypes.POINTER(PmgPhysics))

_sig("pmg_problem_create", c_int, c_int, c_int, c_double, c_int, _V,
     ctypes.POINTER(c_void_p))
_sig("pmg_problem_destroy", c_int, _V)
_sig("pmg_problem_bytes", c_ll, c_int, c_int, c_int)
_sig("pmg_problem_set_fine", c_int, _V, _V, _V, _V, _V, _V, _V)
_sig("pmg_build_hierarchy", c_int, _V, c_int)
_sig("pmg_vcycle", c_int, _V, c_int)
_sig("pmg_compute_residual_2", c_int, _V, PD)
_sig("pmg_solve", c_int, _V, c_double, c_int, PI, PD, PD)
_sig("pmg_pcg_solve", c_int, _V, c_double, c_int, PI, PD, PD)
_sig("pmg_problem_set_host_loop", c_int, _V, c_int)
_sig("pmg_set_autotune", c_int, c_int)
_sig("pmg_set_tma_staging", c_int, c_int)
_sig("pmg_set_finest_streaming", c_int, c_int)
_sig("pmg_test_tma_short_delivery", c_int, c_int)
_sig("pmg_problem_set_coded_couplings", c_int, _V, c_int)
_sig("pmg_problem_coded_couplings", c_int, _V, PI)
_sig("pmg_problem_finest_streamed", c_int, _V, PI)
_sig("pmg_problem_set_throughput_mode", c_int, _V, c_int)
_sig("pmg_solve_start", c_int, _V, c_double, c_int)
_sig("pmg_solve_poll", c_int, _V, PI)
_sig("pmg_solve_finish", c_int, _V, PI, PD, PD)
_sig("pmg_get_potential", c_int, _V, _V)
_sig("pmg_get_potential_async", c_int, _V, _V)
_sig("pmg_problem_set_stream", c_int, _V, _V)
_sig("pmg_get_level", c_int, _V, c_int, _V)
_sig("pmg_problem_stream", c_void_p, _V)
_sig("pmg_problem_set_coarse_rtol", c_int, _V, c_double)
_sig("pmg_problem_set_profiling", c_int, _V, c_int)
_sig("pmg_problem_launches", c_ll, _V)
_sig("pmg_problem_profile", c_int, _V, PD, ctypes.POINTER(c_ll), c_int, c_int)


def check(func: str, status: int) -> None:
    if status != PMG_OK:
        raise PmgError(func, status)


def call(name: str, *args) -> None:
    """Calls an entry point and raises PmgError on a negative status."""
    check(name, getattr(lib, name)(*args))


def exported_symbols() -> list[str]:
    """Names declared in include/pmg_b200.h that the library must export."""
    import re

    hdr = os.path.join(os.path.dirname(HERE), "include", "pmg_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(pmg_[A-Za-z0-9_]+)\s*\(", text)))
