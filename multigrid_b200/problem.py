"""Host mirror of the reference's PBE_linear_problem (PBE_pmgc_class.h:112-1174).

The reference fixes its grid at compile time as template parameters
<base_length, nlev, box_length>; here they are constructor arguments. The
method names follow the class: initialize_boundary / initialize_epsilons /
set_up_rhs (set-up from atoms), buildmultilevelops, v_cycle,
compute_residual_2, plus solve(), which runs the V-cycle loop the reference's
drivers write by hand (PBE_pmgc_class_test.cc:150-162). All work happens in
libpmg_b200.so on the current CUDA device.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .molecule import REFERENCE_PHYSICS, grid_step, level_n, levels_for


def physics_struct(physics: dict) -> _lib.PmgPhysics:
    return _lib.PmgPhysics(**{k: float(physics[k]) for k in (
        "eps_in", "eps_out", "ionic_strength", "ion_radius", "temperature",
        "probe_radius")})


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_lib.PD)


def setup_fine(n: int, h: float, atoms: np.ndarray, physics: dict) -> dict:
    """Fine-level arrays (oC, oE, oN, uC, f, x0; n^3 doubles each, x fastest)
    from atoms (rows x, y, z, radius, charge in the grid frame)."""
    atoms = np.ascontiguousarray(atoms, dtype=np.float64)
    out = {k: np.empty(n ** 3) for k in ("oC", "oE", "oN", "uC", "f", "x0")}
    ph = physics_struct(physics)
    _lib.check("pmg_setup_fine", _lib.lib.pmg_setup_fine(
        n, h, _dptr(atoms), int(atoms.shape[0]), ctypes.byref(ph),
        *[_dptr(out[k]) for k in ("oC", "oE", "oN", "uC", "f", "x0")]))
    return out


def kappa(physics: dict) -> tuple[float, float]:
    """(kappa [1/A], eps0 [reduced units]) of the physics."""
    k = ctypes.c_double()
    e = ctypes.c_double()
    ph = physics_struct(physics)
    _lib.check("pmg_kappa", _lib.lib.pmg_kappa(ctypes.byref(ph),
                                               ctypes.byref(k),
                                               ctypes.byref(e)))
    return k.value, e.value


def set_tma_staging(on: bool) -> None:
    """Problems created afterwards stage the mixed path's 27-point smoother
    tiles by tensor-memory access (default) or load per point (the same
    bits; pmg_set_tma_staging)."""
    _lib.check("pmg_set_tma_staging", _lib.lib.pmg_set_tma_staging(int(on)))


def set_finest_streaming(on: bool) -> None:
    """Problems created afterwards stream the refinement paths' finest
    colour passes through shared memory by bulk copies (default) or load
    per point (the same bits; pmg_set_finest_streaming)."""
    _lib.check("pmg_set_finest_streaming",
               _lib.lib.pmg_set_finest_streaming(int(on)))


@dataclasses.dataclass
class SolveResult:
    cycles: int
    relres: float
    history: np.ndarray  # residual norm before and after each cycle


PRECISIONS = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED,
              "fp64-fast": _lib.PREC_FP64_FAST}


class PBELinearProblem:
    """PBE_linear_problem<base, nlev, box> with runtime sizes.

    precision: "fp64" (the reference's arithmetic), "mixed" (float
    V-cycles inside double iterative refinement; double residual, norms and
    coarsest CG) or "fp64-fast" (double V-cycles in the mixed path's
    structure: the fastest all-double solve).
    """

    def __init__(self, base: int, nlev: int, box: float,
                 precision: str = "fp64", physics: dict | None = None,
                 stream: int | None = None, hierarchy: str | None = None):
        """hierarchy: "reference" keeps the class's levels (base * 2^L + 1,
        L = 1..nlev); "deep" coarsens the same finest grid as far as a 5^3
        coarsest level allows (levels_for), which makes the coarsest CG
        cheap. Default: "reference" for fp64 (parity with the reference),
        "deep" for mixed and fp64-fast."""
        n = level_n(int(base), int(nlev))
        if hierarchy is None:
            hierarchy = "reference" if precision == "fp64" else "deep"
        if hierarchy == "deep":
            base, nlev = levels_for(n, max_levels=12, min_coarse=5)
        elif hierarchy != "reference":
            raise ValueError(f"unknown hierarchy {hierarchy!r}")
        self.hierarchy = hierarchy
        self.base, self.nlev, self.box = int(base), int(nlev), float(box)
        self.n = level_n(self.base, self.nlev)
        self.grid_step = grid_step(self.base, self.nlev, self.box)
        self.precision = precision
        self.physics = dict(physics or REFERENCE_PHYSICS)
        self._atoms = None
        self._fine = None
        h = ctypes.c_void_p()
        _lib.check("pmg_problem_create", _lib.lib.pmg_problem_create(
            self.base, self.nlev, self.box, PRECISIONS[precision],
            ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self._h = h

    # -- lifetime ----------------------------------------------------------
    def close(self) -> None:
        if self._h:
            _lib.lib.pmg_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def device_bytes(base: int, nlev: int, precision: str = "fp64") -> int:
        return int(_lib.lib.pmg_problem_bytes(base, nlev,
                                              PRECISIONS[precision]))

    @property
    def stream(self) -> int:
        return int(_lib.lib.pmg_problem_stream(self._h) or 0)

    # -- set-up (PBE_pmgc_class.h:191-349) ----------------------------------
    def _setup_from_atoms(self, atoms) -> None:
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        if self._atoms is None or not np.array_equal(self._atoms, atoms):
            self._atoms = atoms
            self._fine = setup_fine(self.n, self.grid_step, atoms,
                                    self.physics)
            self.set_fine(**self._fine)

    def set_atoms(self, atoms, physics: dict | None = None) -> None:
        """Loads the finest level from atoms with the GPU set-up
        (pmg_problem_set_atoms): only the atoms cross PCIe. Equal to the host
        set-up bit for bit except the Debye-Hueckel boundary values (CUDA's
        exp, a few ulp)."""
        atoms = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 5)
        ph = physics_struct(physics or self.physics)
        _lib.check("pmg_problem_set_atoms", _lib.lib.pmg_problem_set_atoms(
            self._h, _dptr(atoms), len(atoms), ctypes.byref(ph)))
        # the atoms are copied before the call returns (pageable source)
        self._atoms = None
        self._fine = None

    def initialize_boundary(self, atoms) -> None:
        """Debye-Hueckel boundary values on the finest shell."""
        self._setup_from_atoms(atoms)

    def initialize_epsilons(self, atoms) -> None:
        """Dielectric, kappa and centre coefficients of the finest level."""
        self._setup_from_atoms(atoms)

    def set_up_rhs(self, atoms) -> None:
        """Trilinear charge distribution on the finest level."""
        self._setup_from_atoms(atoms)

    def set_fine(self, oC, oE, oN, uC, f, x0) -> None:
        """Loads the finest level from host (numpy) or device (torch)
        arrays of n^3 doubles."""
        keep = []

        def ptr(a):
            if hasattr(a, "data_ptr"):
                assert a.dtype.is_floating_point and a.element_size() == 8
                assert a.numel() == self.n ** 3 and a.is_contiguous()
                return ctypes.c_void_p(a.data_ptr())
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
            assert a.size == self.n ** 3
            keep.append(a)
            return ctypes.c_void_p(a.ctypes.data)

        ptrs = [ptr(a) for a in (oC, oE, oN, uC, f, x0)]
        _lib.check("pmg_problem_set_fine",
                   _lib.lib.pmg_problem_set_fine(self._h, *ptrs))
        # pmg_problem_set_fine is stream-ordered; host buffers must live
        # until the copies finish.
        self.synchronize()
        del keep

    def synchronize(self) -> None:
        import torch  # noqa: F401  (CUDA context of the process)
        torch.cuda.current_stream()  # make sure CUDA is initialised
        torch.cuda.ExternalStream(self.stream).synchronize()

    def set_coarse_rtol(self, rtol: float) -> None:
        """Mixed precision: relative stop of the coarsest CG per correction."""
        _lib.check("pmg_problem_set_coarse_rtol",
                   _lib.lib.pmg_problem_set_coarse_rtol(self._h, float(rtol)))

    @property
    def launches(self) -> int:
        """Kernels launched by this problem so far."""
        return int(_lib.lib.pmg_problem_launches(self._h))

    PHASES = ("pre-smooth", "defect", "restrict", "coarse-solve", "damping",
              "interp", "axpy", "post-smooth")
    GLOBAL_PHASES = ("residual", "refine-update")

    def set_host_loop(self, on: bool = True) -> None:
        """Drive solve()'s cycles from the host (one graph launch per cycle)
        instead of one graph with the stop test on the GPU: same results;
        for kernel profilers, which cannot see kernels inside graphs with
        conditional nodes."""
        _lib.check("pmg_problem_set_host_loop",
                   _lib.lib.pmg_problem_set_host_loop(self._h, int(on)))

    def set_throughput_mode(self, on: bool = True) -> None:
        """Choose kernels for many solves sharing the GPU (the serving
        runtime's setting) rather than for this solve's latency; mixed
        results may differ from the default mode in the last bits."""
        _lib.check("pmg_problem_set_throughput_mode",
                   _lib.lib.pmg_problem_set_throughput_mode(self._h, int(on)))

    def set_coded_couplings(self, on: bool = True) -> None:
        """Mixed precision: read the finest couplings as one code byte per
        point when the operator has two values per direction (default on;
        the same bits either way)."""
        _lib.check("pmg_problem_set_coded_couplings",
                   _lib.lib.pmg_problem_set_coded_couplings(self._h, int(on)))

    def coded_couplings(self) -> bool:
        """Whether the built mixed problem's finest couplings are coded."""
        c = ctypes.c_int()
        _lib.check("pmg_problem_coded_couplings",
                   _lib.lib.pmg_problem_coded_couplings(self._h,
                                                        ctypes.byref(c)))
        return bool(c.value)

    def finest_streamed(self) -> bool:
        """Whether the finest colour passes and refinement residual stream
        their rows through shared memory (pmg_problem_finest_streamed)."""
        c = ctypes.c_int()
        _lib.check("pmg_problem_finest_streamed",
                   _lib.lib.pmg_problem_finest_streamed(self._h,
                                                        ctypes.byref(c)))
        return bool(c.value)

    def set_profiling(self, on: bool = True) -> None:
        """Time every cycle phase with CUDA events inside the cycle graph."""
        _lib.check("pmg_problem_set_profiling",
                   _lib.lib.pmg_problem_set_profiling(self._h, int(on)))

    def profile(self, reset: bool = False) -> dict:
        """{(level, phase): (total ms, launches)} accumulated by solve();
        level 0 holds the finest-level residual and refinement update."""
        cap = 8 * 13
        ms = np.zeros(cap)
        cnt = np.zeros(cap, dtype=np.int64)
        n = _lib.lib.pmg_problem_profile(
            self._h, _dptr(ms), cnt.ctypes.data_as(
                ctypes.POINTER(ctypes.c_longlong)), cap, int(reset))
        out = {}
        for q in range(min(n, cap)):
            if cnt[q]:
                L, ph = divmod(q, 8)
                name = (self.GLOBAL_PHASES[ph] if L == 0 and ph < 2
                        else self.PHASES[ph])
                out[(L, name)] = (float(ms[q]), int(cnt[q]))
        return out

    # -- multigrid ------------------------------------------------------------
    def buildmultilevelops(self, trilinear: bool = False) -> None:
        """Galerkin hierarchy (PBE_pmgc_class.h:351-617)."""
        _lib.check("pmg_build_hierarchy",
                   _lib.lib.pmg_build_hierarchy(self._h, int(trilinear)))

    def v_cycle(self, as_preconditioner: bool = False) -> None:
        """One V-cycle (PBE_pmgc_class.h:1070-1114); fp64 problems."""
        _lib.check("pmg_vcycle",
                   _lib.lib.pmg_vcycle(self._h, int(as_preconditioner)))

    def compute_residual_2(self) -> float:
        """sqrt(sum (f - A x)^2 / n^3) on the finest level."""
        out = ctypes.c_double()
        _lib.check("pmg_compute_residual_2",
                   _lib.lib.pmg_compute_residual_2(self._h, ctypes.byref(out)))
        return out.value

    def solve(self, tol: float = 1e-10, max_cycles: int = 100) -> SolveResult:
        """V-cycles (fp64) or refinement steps (mixed) until
        compute_residual_2() / r0 < tol."""
        hist = np.zeros(max_cycles + 1)
        cycles = ctypes.c_int()
        rel = ctypes.c_double()
        _lib.check("pmg_solve", _lib.lib.pmg_solve(
            self._h, tol, max_cycles, ctypes.byref(cycles), ctypes.byref(rel),
            _dptr(hist)))
        return SolveResult(cycles.value, rel.value, hist[:cycles.value + 1])

    def pcg_solve(self, tol: float = 1e-10,
                  max_iters: int = 100) -> SolveResult:
        """MG-preconditioned CG on the finest level (the app's outer solver:
        CG_solver with this class as preconditioner); tol = 0 runs exactly
        max_iters iterations."""
        hist = np.zeros(max_iters + 1)
        iters = ctypes.c_int()
        rel = ctypes.c_double()
        _lib.check("pmg_pcg_solve", _lib.lib.pmg_pcg_solve(
            self._h, tol, max_iters, ctypes.byref(iters), ctypes.byref(rel),
            _dptr(hist)))
        return SolveResult(iters.value, rel.value, hist[:iters.value + 1])

    def solve_start(self, tol: float = 1e-10, max_cycles: int = 100) -> None:
        """Enqueues the whole solve (one graph launch, stop test on the GPU)
        and returns at once; finish with solve_finish()."""
        _lib.check("pmg_solve_start", _lib.lib.pmg_solve_start(
            self._h, tol, max_cycles))
        self._pending_max = max_cycles

    def solve_done(self) -> bool:
        done = ctypes.c_int()
        _lib.check("pmg_solve_poll", _lib.lib.pmg_solve_poll(
            self._h, ctypes.byref(done)))
        return bool(done.value)

    def solve_finish(self) -> SolveResult:
        hist = np.zeros(getattr(self, "_pending_max", 1024) + 1)
        cycles = ctypes.c_int()
        rel = ctypes.c_double()
        _lib.check("pmg_solve_finish", _lib.lib.pmg_solve_finish(
            self._h, ctypes.byref(cycles), ctypes.byref(rel), _dptr(hist)))
        return SolveResult(cycles.value, rel.value, hist[:cycles.value + 1])

    # -- results ----------------------------------------------------------------
    def potential(self) -> np.ndarray:
        """Finest iterate, shape (n, n, n) indexed [k, j, i] (x fastest)."""
        out = np.empty(self.n ** 3)
        _lib.check("pmg_get_potential", _lib.lib.pmg_get_potential(
            self._h, ctypes.c_void_p(out.ctypes.data)))
        return out.reshape(self.n, self.n, self.n)

    def get_level(self, level: int) -> tuple[np.ndarray, np.ndarray]:
        """(P (27, n_L^3), A (14, n_L^3)) of coarse level L in [1, nlev-1]."""
        nl = level_n(self.base, level) ** 3
        out = np.empty(41 * nl)
        _lib.check("pmg_get_level", _lib.lib.pmg_get_level(
            self._h, level, ctypes.c_void_p(out.ctypes.data)))
        out = out.reshape(41, nl)
        return out[:27], out[27:]
