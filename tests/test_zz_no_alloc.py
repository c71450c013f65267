"""The allocation-free coarsest-level CG (pmg_cg_level_noalloc_d) against
the allocating entry point (pmg_cg_level_d), through the C ABI.

pmg_cg_level_noalloc_d serves callers that cannot let a library allocate
device memory (applications that own the whole device budget through their
own pool, or that must not meet allocator stalls mid time-step); it keeps its
work vectors in a static device array of the library, limited to 17^3-point
grids. The tests run it several times in a row on different problems — a
call must not see the previous call's leftovers — and compare each result
with the allocating entry point's: golden coarsest levels, a grid of exactly
17^3 points, and a 19 x 13 x 19 grid (more than 17 points along an axis,
fewer than 17^3 in all), which takes the one-CTA kernel and so the static
array's work vectors. This file is collected last so that a failure
here cannot hide any other test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from conftest import load_golden  # noqa: E402
from multigrid_b200 import _lib  # noqa: E402

DEV = torch.device("cuda:0")
TOL = 1e-12  # the CG tolerance of the GPU kernel tests


def _level1(name):
    g = load_golden(name)
    n1 = 2 * int(g["base"]) + 1
    ops = [torch.as_tensor(np.ascontiguousarray(a), device=DEV)
           for a in g["A1"]]
    return n1, ops, g["cg_rhs"]


def _random_level(nx, ny, nz, seed):
    """A symmetric, strictly diagonally dominant 27-point operator (14
    stored diagonals: couplings in [0, 1), oC = 27) on an nx x ny x nz grid,
    a right-hand side and a warm start, both zero on the shell."""
    rng = np.random.default_rng(seed)
    n3 = nx * ny * nz
    ops = [np.full(n3, 27.0)] + [rng.uniform(0.0, 1.0, n3)
                                 for _ in range(13)]
    shell = np.ones((nz, ny, nx), dtype=bool)
    shell[1:-1, 1:-1, 1:-1] = False
    shell = shell.ravel()
    rhs = np.where(shell, 0.0, rng.normal(size=n3))
    x0 = np.where(shell, 0.0, rng.normal(size=n3) * 1e-3)
    return [torch.as_tensor(a, device=DEV) for a in ops], rhs, x0


def _run(entry, n, ops, rhs, x0):
    nx, ny, nz = n if isinstance(n, tuple) else (n, n, n)
    a14 = (ctypes.c_void_p * 14)(*[t.data_ptr() for t in ops])
    b = torch.as_tensor(rhs, device=DEV)
    x = torch.as_tensor(x0, device=DEV).clone()
    it = ctypes.c_int()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = getattr(_lib.lib, entry)(nx, ny, nz, a14,
                                  ctypes.c_void_p(b.data_ptr()),
                                  ctypes.c_void_p(x.data_ptr()), 1e-8, 20000,
                                  ctypes.byref(it), stream)
    _lib.check(entry, rc)
    torch.cuda.synchronize()
    return x.cpu().numpy(), it.value


def test_noalloc_cg_matches_allocating_entry_twice_in_a_row():
    # a 9^3 level-1 problem, then a 5^3 one: the second reuses the static
    # work area with a different layout
    for name, seed in (("problem_b4n3.npz", 1), ("problem_b2n3.npz", 2)):
        n, ops, rhs = _level1(name)
        x0 = np.random.default_rng(seed).normal(size=n ** 3) * 1e-3
        # warm start with a zero shell, as the coarsest level keeps it
        shell = np.ones((n, n, n), dtype=bool)
        shell[1:-1, 1:-1, 1:-1] = False
        x0 = np.where(shell.ravel(), 0.0, x0)
        want, it_want = _run("pmg_cg_level_d", n, ops, rhs, x0)
        got, it_got = _run("pmg_cg_level_noalloc_d", n, ops, rhs, x0)
        assert it_got == it_want
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= TOL, (name, err)


def test_noalloc_cg_at_the_size_limit_and_on_its_work_vectors():
    """A grid of exactly 17^3 points (cluster kernel), a 19 x 13 x 19 grid
    (4693 <= 17^3 points: the one-CTA kernel, which keeps r, p and A p in
    the static array) and both again, one call after the other, each
    against the allocating entry point."""
    for shape, seed in (((17, 17, 17), 3), ((19, 13, 19), 4),
                        ((17, 17, 17), 5), ((19, 13, 19), 6)):
        ops, rhs, x0 = _random_level(*shape, seed)
        want, it_want = _run("pmg_cg_level_d", shape, ops, rhs, x0)
        got, it_got = _run("pmg_cg_level_noalloc_d", shape, ops, rhs, x0)
        assert it_want > 1
        assert it_got == it_want, shape
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= TOL, (shape, err)


def test_noalloc_cg_rejects_grids_beyond_its_work_area():
    n, ops, rhs = _level1("problem_b2n3.npz")
    a14 = (ctypes.c_void_p * 14)(*[t.data_ptr() for t in ops])
    x = torch.zeros(1, dtype=torch.float64, device=DEV)
    rc = _lib.lib.pmg_cg_level_noalloc_d(
        19, 19, 19, a14, ctypes.c_void_p(x.data_ptr()),
        ctypes.c_void_p(x.data_ptr()), 1e-8, 10, None, None)
    assert rc == -1
    assert b"17*17*17" in _lib.lib.pmg_last_error()
