"""Serving and batched solves over the native runtime (pmg_server_* in
include/pmg_b200.h).

A Server admits PB solve requests in arrival order against a device-memory
budget, keeps each admitted solve's hierarchy resident in a problem of its
shape (reused by later requests of the same grid and precision), and runs up
to `max_inflight` solves at once, each as one graph launch on its own stream,
so cycles of different grid sizes overlap on the device. The admission,
pooling and polling loop is the library's worker thread (C++); this module
only marshals requests and keeps their buffers alive until they complete.

The reference has no serving layer: it solves one molecule per process
(PBE_pmgc_class_test.cc:84-146); each request here runs that solve
(set fine level, buildmultilevelops, V-cycles to the relative residual).
"""
from __future__ import annotations

import ctypes
from ctypes import c_char, c_double, c_int, c_longlong, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _lib
from .molecule import level_n
from .problem import PRECISIONS

FINE_KEYS = ("oC", "oE", "oN", "uC", "f", "x0")


class _Request(ctypes.Structure):
    _fields_ = [("base", c_int), ("nlev", c_int), ("box", c_double),
                ("precision", c_int), ("fine", c_void_p * 6),
                ("potential", c_void_p), ("tol", c_double),
                ("max_cycles", c_int), ("tag", c_longlong),
                ("hierarchy", c_int), ("atoms", c_void_p),
                ("natoms", c_int), ("physics", _lib.PmgPhysics)]


class _Completion(ctypes.Structure):
    _fields_ = [("tag", c_longlong), ("status", c_int), ("cycles", c_int),
                ("relres", c_double), ("t_submit", c_double),
                ("t_admit", c_double), ("t_done", c_double),
                ("message", c_char * 160)]


class _Stats(ctypes.Structure):
    _fields_ = [("queued", c_int), ("inflight", c_int),
                ("idle_problems", c_int), ("held_bytes", c_longlong),
                ("peak_bytes", c_longlong), ("budget_bytes", c_longlong),
                ("completed", c_longlong), ("created_problems", c_longlong),
                ("evicted_problems", c_longlong), ("issue_s", c_double),
                ("issue_max_s", c_double), ("retire_s", c_double),
                ("retire_max_s", c_double)]


_V = c_void_p
_lib._sig("pmg_server_create", c_int, c_longlong, c_int,
          ctypes.POINTER(c_void_p))
_lib._sig("pmg_server_submit", c_int, _V, ctypes.POINTER(_Request))
_lib._sig("pmg_server_wait", c_int, _V, ctypes.POINTER(_Completion), c_int,
          ctypes.POINTER(c_int), c_double)
_lib._sig("pmg_server_get_stats", c_int, _V, ctypes.POINTER(_Stats))
_lib._sig("pmg_server_destroy", c_int, _V)
_lib._sig("pmg_levels_for", c_int, c_int, c_int, c_int,
          ctypes.POINTER(c_int), ctypes.POINTER(c_int))
_lib._sig("pmg_batch_solve", c_int, ctypes.POINTER(_Request), c_int,
          c_longlong, c_int, ctypes.POINTER(_Completion))


@dataclass
class Completion:
    tag: int
    status: int
    cycles: int
    relres: float
    t_submit: float  # seconds since the server started
    t_admit: float
    t_done: float
    message: str

    @property
    def ok(self) -> bool:
        return self.status == _lib.PMG_OK

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous float64")
        return a.ctypes.data
    import torch
    if isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("tensors must be contiguous float64")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def _completion(c: _Completion) -> Completion:
    return Completion(int(c.tag), int(c.status), int(c.cycles),
                      float(c.relres), float(c.t_submit), float(c.t_admit),
                      float(c.t_done), c.message.decode(errors="replace"))


def _request(base, nlev, box, precision, fine, out, tol, max_cycles, tag,
             atoms=None, physics=None):
    """fine: dict of the six fine-level arrays, or None with `atoms`
    (rows x y z radius charge, GPU set-up with `physics`)."""
    n3 = level_n(base, nlev) ** 3
    r = _Request()
    r.base, r.nlev, r.box = base, nlev, box
    r.precision = PRECISIONS[precision]
    keep = []
    if atoms is not None:
        from .problem import physics_struct
        from .molecule import REFERENCE_PHYSICS
        a = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 5)
        if not len(a):  # no atoms: any valid non-null pointer
            a = np.zeros(5)
        keep.append(a)
        r.atoms = a.ctypes.data
        r.natoms = len(np.asarray(atoms).reshape(-1, 5))
        r.physics = physics_struct(physics or REFERENCE_PHYSICS)
        fine = None
    for q, k in enumerate(FINE_KEYS if fine is not None else ()):
        a = fine[k]
        if isinstance(a, np.ndarray):
            a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        if (a.size if isinstance(a, np.ndarray) else a.numel()) != n3:
            raise ValueError(f"{k}: expected {n3} values")
        keep.append(a)
        r.fine[q] = _ptr(a)
    if out is not None:
        if (out.size if isinstance(out, np.ndarray) else out.numel()) != n3:
            raise ValueError(f"out: expected {n3} values")
        keep.append(out)
        r.potential = _ptr(out)
    r.tol, r.max_cycles, r.tag = tol, max_cycles, tag
    # same default as PBELinearProblem: the deepest hierarchy except for
    # the reference's FP64 cycle
    r.hierarchy = 0 if precision == "fp64" else 1
    return r, keep


class Server:
    """Continuous-batching PB solve server on the current CUDA device.

    submit() enqueues and returns at once; wait() returns completions as
    the worker retires them. Device inputs must be fully written (their
    producing stream synchronised) before submit()."""

    def __init__(self, budget_bytes: int, max_inflight: int = 32):
        h = c_void_p()
        _lib.check("pmg_server_create", _lib.lib.pmg_server_create(
            int(budget_bytes), int(max_inflight), ctypes.byref(h)))
        self._h = h
        self._keep: dict[int, list] = {}
        self._next = 0

    def submit(self, base: int, nlev: int, box: float, fine: dict | None,
               precision: str = "mixed", out=None, tol: float = 1e-10,
               max_cycles: int = 100, tag: int | None = None, atoms=None,
               physics: dict | None = None) -> int:
        """Enqueues one solve: from the six fine-level arrays (`fine`), or
        from `atoms` with the GPU set-up (fine=None)."""
        if tag is None:
            tag = self._next
        self._next = max(self._next, tag) + 1
        r, keep = _request(base, nlev, box, precision, fine, out, tol,
                           max_cycles, tag, atoms, physics)
        self._keep[tag] = keep
        _lib.check("pmg_server_submit",
                   _lib.lib.pmg_server_submit(self._h, ctypes.byref(r)))
        return tag

    def wait(self, timeout: float = 0.0, cap: int = 256) -> list[Completion]:
        buf = (_Completion * cap)()
        n = c_int()
        _lib.check("pmg_server_wait", _lib.lib.pmg_server_wait(
            self._h, buf, cap, ctypes.byref(n), float(timeout)))
        out = [_completion(buf[i]) for i in range(n.value)]
        for c in out:
            self._keep.pop(c.tag, None)
        return out

    def drain(self, count: int, timeout: float = 600.0) -> list[Completion]:
        """Waits until `count` more completions arrived."""
        import time
        got: list[Completion] = []
        t_end = time.monotonic() + timeout
        while len(got) < count:
            left = t_end - time.monotonic()
            if left <= 0:
                raise TimeoutError(f"{len(got)} of {count} completions")
            got += self.wait(timeout=min(left, 1.0))
        return got

    def stats(self) -> dict:
        st = _Stats()
        _lib.check("pmg_server_get_stats", _lib.lib.pmg_server_get_stats(
            self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _Stats._fields_}

    def close(self) -> None:
        if self._h:
            _lib.lib.pmg_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_solve(items: list[dict], budget_bytes: int, max_inflight: int = 96,
                tol: float = 1e-10, max_cycles: int = 100) -> list[Completion]:
    """Solves every item ({base, nlev, box, fine, precision, out}) through
    one server (pmg_batch_solve); completions come back in item order."""
    reqs = (_Request * len(items))()
    keep = []
    for i, it in enumerate(items):
        r, k = _request(it["base"], it["nlev"], it["box"],
                        it.get("precision", "mixed"), it.get("fine"),
                        it.get("out"), tol, max_cycles, i, it.get("atoms"),
                        it.get("physics"))
        reqs[i] = r
        keep.append(k)
    out = (_Completion * max(1, len(items)))()
    _lib.check("pmg_batch_solve", _lib.lib.pmg_batch_solve(
        reqs, len(items), int(budget_bytes), int(max_inflight), out))
    return [_completion(out[i]) for i in range(len(items))]


# ---------------------------------------------------------------------------
# open-loop load (serving measurements)
# ---------------------------------------------------------------------------
def poisson_arrivals(rate: float, count: int, seed: int = 0) -> np.ndarray:
    """Arrival times (s, from 0) of an open-loop Poisson stream: cumulative
    exponential gaps of mean 1/rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def percentile(values, q: float) -> float:
    """The q-th percentile (0..100) by the nearest-rank rule."""
    v = np.sort(np.asarray(values, dtype=np.float64))
    if not len(v):
        return float("nan")
    k = max(1, int(np.ceil(q / 100.0 * len(v))))
    return float(v[k - 1])


def open_loop(server: Server, arrivals: np.ndarray, submit_one,
              timeout: float = 600.0) -> tuple[list[Completion], float]:
    """Submits request i (submit_one(server, i)) at arrivals[i] seconds after
    the start, collecting completions while it waits; returns every
    completion and the wall time from the first arrival to the last
    completion."""
    import time
    t0 = time.perf_counter()
    done: list[Completion] = []
    for i, t in enumerate(arrivals):
        while True:
            left = t0 + t - time.perf_counter()
            if left <= 0:
                break
            done += server.wait(timeout=min(left, 0.002))
        submit_one(server, i)
    done += server.drain(len(arrivals) - len(done), timeout=timeout)
    return done, time.perf_counter() - t0 - float(arrivals[0])
