"""Host-side logic that needs no GPU: the C ABI library loads and exports
every declared symbol, argument checks reject bad calls before any CUDA work,
grid-size rules are exact, synthetic molecules are well formed."""
import ctypes
import os
import math

import numpy as np
import pytest

from multigrid_b200 import _lib
from multigrid_b200.molecule import (BATCH_SIZES, WORKLOADS, batch_grid,
                                     batch_workloads, coarsen, grid_step,
                                     level_n, levels_for, synthetic_atoms)


def test_library_exports_header():
    names = _lib.exported_symbols()
    assert len(names) > 25
    missing = [n for n in names if not hasattr(_lib.lib, n)]
    assert not missing, missing


def test_version():
    assert b"sm_100a" in _lib.lib.pmg_version()


V = ctypes.c_void_p


def test_kernel_args_rejected_without_gpu():
    # grid too small / mismatched coarse sizes / null arrays: PMG_ERR_ARG
    p = V(16)  # never dereferenced: the size checks fail first
    assert _lib.lib.pmg_Vgsrb7x_d(2, 9, 9, p, None, p, p, p, p, p, 1, 0, 0,
                                  None) == -1
    assert _lib.lib.pmg_Vgsrb7x_d(9, 9, 9, None, None, p, p, p, p, p, 1, 0, 0,
                                  None) == -1
    assert b"null" in _lib.lib.pmg_last_error()
    args = [9, 9, 9, 4, 4, 4] + [p] * 29 + [None]
    assert _lib.lib.pmg_Vrestrc2_d(*args) == -1
    assert b"2 n_c - 1" in _lib.lib.pmg_last_error()
    assert _lib.lib.pmg_Vgsrb27x_d(*([9, 9, 9] + [p] * 17 + [-1, 0, 0, None])
                                   ) == -1


def test_problem_bytes():
    b = _lib.lib.pmg_problem_bytes(8, 5, 0)
    # 257^3 finest level: 4 coefficients + x, f, r = 7 arrays, and the
    # colour-split copies of the operator, x and f (6 more) the finest
    # smoother and defect run on
    assert b > 13 * 257 ** 3 * 8
    assert b < 4 * 2 ** 30
    mixed = _lib.lib.pmg_problem_bytes(8, 5, 1)
    # double finest level (x, f and the operator) plus float copies
    assert 7 * 257 ** 3 * 8 < mixed < 4 * 2 ** 30
    assert _lib.lib.pmg_problem_bytes(0, 5, 0) == -1
    assert _lib.lib.pmg_problem_bytes(64, 5, 0) == -1  # n > 1025


def test_grid_rules():
    assert level_n(4, 4) == 65 and level_n(5, 5) == 161
    assert level_n(8, 5) == 257
    for n in (9, 17, 65, 161, 257):
        assert coarsen(n) == (n - 1) // 2 + 1
    assert [level_n(8, L) for L in range(5, 0, -1)] == [257, 129, 65, 33, 17]
    assert grid_step(8, 5, 102.4) == pytest.approx(0.4)
    assert {n: levels_for(n) for n in BATCH_SIZES} == {
        65: (2, 5), 97: (3, 5), 129: (2, 6), 161: (5, 5), 193: (3, 6),
        225: (7, 5)}
    assert batch_grid(5.0) == 65 and batch_grid(30.0) == 161
    assert batch_grid(200.0) == 225


def test_workloads():
    w = WORKLOADS["pb257"]
    assert (w.n, w.base, w.nlev) == (257, 8, 5)
    assert w.box == pytest.approx(102.4)
    assert WORKLOADS["pb65"].n == 65 and WORKLOADS["pb161"].n == 161
    ws = batch_workloads(96)
    assert len(ws) == 96
    assert all(4 <= w.nlev <= 6 for w in ws)
    assert all(200 <= w.natoms <= 6000 for w in ws)
    assert {w.n for w in ws} <= set(BATCH_SIZES)


def test_synthetic_atoms():
    a = synthetic_atoms(500, 12.0, 0, (16.0, 16.0, 16.0))
    b = synthetic_atoms(500, 12.0, 0, (16.0, 16.0, 16.0))
    assert np.array_equal(a, b)
    r = np.linalg.norm(a[:, :3] - 16.0, axis=1)
    assert a.shape == (500, 5) and r.max() <= 12.0
    assert a[:, 3].min() >= 1.2 and a[:, 3].max() <= 2.0
    q = a[:, 4].sum()
    assert abs(q - round(q)) < 1e-9
    assert abs(np.std(a[:, 4]) - 0.4) < 0.05


def test_setup_physics():
    from multigrid_b200.problem import kappa
    from multigrid_b200.molecule import DEFAULT_PHYSICS, REFERENCE_PHYSICS
    k, e0 = kappa(REFERENCE_PHYSICS)
    # Debye length of 0.15 M 1:1 salt at 298 K in water: ~7.85 A
    assert 1 / k == pytest.approx(7.85, abs=0.05)
    assert e0 == pytest.approx(1.42e-4, rel=0.01)
    k2, _ = kappa(DEFAULT_PHYSICS)
    assert k2 == pytest.approx(k * math.sqrt(78.4 / 78.54), rel=1e-12)


def test_setup_probe_surface_contains_vdw():
    from multigrid_b200.molecule import DEFAULT_PHYSICS
    from multigrid_b200.problem import setup_fine
    n, h = 33, 0.5
    atoms = synthetic_atoms(30, 3.5, 5, (8.0, 8.0, 8.0))
    vdw = setup_fine(n, h, atoms, dict(DEFAULT_PHYSICS, probe_radius=0.0))
    ses = setup_fine(n, h, atoms, DEFAULT_PHYSICS)
    inside_vdw = vdw["oE"] < DEFAULT_PHYSICS["eps_out"] / h ** 2
    inside_ses = ses["oE"] < DEFAULT_PHYSICS["eps_out"] / h ** 2
    # the molecular surface encloses the van der Waals volume and more
    assert np.all(inside_ses[inside_vdw])
    assert inside_ses.sum() > inside_vdw.sum()
    # the rest of the set-up does not depend on the probe
    for k in ("f", "x0"):
        assert np.array_equal(vdw[k], ses[k])


def test_setup_rejects_atoms_outside():
    from multigrid_b200.molecule import DEFAULT_PHYSICS
    from multigrid_b200.problem import setup_fine
    with pytest.raises(_lib.PmgError):
        setup_fine(9, 0.5, np.array([[10.0, 1.0, 1.0, 1.5, 1.0]]),
                   DEFAULT_PHYSICS)


def test_bench_reads_profiled_traffic():
    """bench.py's roofline takes its DRAM traffic from the committed ncu
    summary of the dominant kernel (bytes per launch x launches per phase)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "bench", os.path.join(os.path.dirname(__file__), "..", "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    t = bench.profiled_traffic("gs7_split_color_kernel", 4, "pb257", "mixed")
    assert t == pytest.approx(4 * 343670000)
    assert bench.profiled_traffic("no_such_kernel", 1, "pb257", "mixed") is None
    assert bench.profiled_traffic(None, 1, "pb257", "mixed") is None


def test_server_rejects_bad_arguments_without_gpu():
    from multigrid_b200.serve import Server
    for budget, inflight in ((0, 4), (1 << 30, 0), (1 << 30, 1000)):
        with pytest.raises(_lib.PmgError) as e:
            Server(budget, inflight)
        assert e.value.status == _lib.PMG_ERR_ARG


def test_native_levels_rule_matches_python():
    """The runtime's hierarchy rule (pmg_levels_for) and levels_for agree."""
    import ctypes
    from multigrid_b200 import serve  # noqa: F401  (declares the symbol)
    from multigrid_b200.molecule import levels_for
    for n in list(range(5, 300, 4)) + [129, 161, 193, 225, 257, 513]:
        try:
            want = levels_for(n, max_levels=12, min_coarse=5)
        except ValueError:
            want = None
        b, L = ctypes.c_int(), ctypes.c_int()
        rc = _lib.lib.pmg_levels_for(n, 12, 5, ctypes.byref(b),
                                     ctypes.byref(L))
        got = (b.value, L.value) if rc == 0 else None
        assert got == want, n


def test_poisson_arrivals_and_percentiles():
    from multigrid_b200.serve import percentile, poisson_arrivals
    t = poisson_arrivals(200.0, 20000, seed=1)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 200.0) < 200.0 * 0.03
    assert percentile([5, 1, 3, 2, 4], 50) == 3
    assert percentile(list(range(1, 101)), 99) == 99
    assert percentile([7.0], 99) == 7.0


def test_pqr_reader(tmp_path):
    """Lines of exactly ten fields other than REMARK are atoms: x y z from
    fields 6-8, charge 9, radius 10; other lines are skipped."""
    from multigrid_b200.fileio import read_pqr
    p = tmp_path / "mol.pqr"
    p.write_text(
        "REMARK   1 generated for a reader test\n"
        "\n"
        "ATOM      1  N   ALA     1      1.000   2.000   3.000 -0.3000 1.8240\n"
        "ATOM      2  CA  ALA     1     -4.500   0.250  10.125  0.1500 1.9080\n"
        "HETATM    3  O   HOH\n"
        "ATOM      4  C   ALA     1      7.000   8.000   9.000  0.5000 1.7000\n"
        "TER\nEND\n")
    a = read_pqr(str(p))
    assert a.shape == (3, 5)
    assert np.array_equal(a[1], [-4.5, 0.25, 10.125, 1.908, 0.15])
    b = read_pqr(str(p), origin=(1.0, 2.0, 3.0))
    assert np.array_equal(b[0], [0.0, 0.0, 0.0, 1.824, -0.3])
    with pytest.raises(_lib.PmgError):
        read_pqr(str(tmp_path / "missing.pqr"))


def test_dx_writer_format(tmp_path):
    """The reference's OpenDX layout: header, three values per line in array
    order formatted as {:<+13e} plus a space, field trailer."""
    from multigrid_b200.fileio import write_dx
    v = np.arange(27, dtype=np.float64).reshape(3, 3, 3) * 0.5 - 3.0
    v[0, 0, 1] = 1.5e-120
    p = tmp_path / "pot.dx"
    write_dx(str(p), v, origin=(-1.0, 2.0, 0.25), box_length=8.0)
    fmt = lambda x: format(x, "<+13e") + " "  # noqa: E731
    lines = [
        "object 1 class gridpositions counts 3 3 3",
        "origin " + fmt(-1.0) + fmt(2.0) + fmt(0.25),
        "delta " + fmt(4.0) + fmt(0.0) + fmt(0.0),
        "delta " + fmt(0.0) + fmt(4.0) + fmt(0.0),
        "delta " + fmt(0.0) + fmt(0.0) + fmt(4.0),
        "object 2 class gridconnections count 3 3 3",
        "object 3 class array type double rank 0 items 27 data follows",
    ]
    flat = v.ravel()
    for r in range(9):
        lines.append("".join(fmt(x) for x in flat[3 * r:3 * r + 3]))
    lines += ['attribute "dep" string "positions"',
              'object "regular positions regular connections" class field',
              'component "positions" value 1',
              'component "connections" value 2',
              'component "data" value 3']
    assert p.read_text() == "\n".join(lines) + "\n"


def test_bench_phase_accounting():
    """bench.py's algorithmic bytes and kernel names per cycle phase: the
    coupling arrays (28 B per point and sweep in float, 7 arrays) or, with
    the operator coded (couplings and oC in one byte), code byte + f + x
    read and written (13 B); the refinement residual 52 B or 21 B per
    point."""
    import importlib
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))))
    bench = importlib.import_module("bench")

    class P:
        base, nlev, n, precision = 2, 7, 257, "mixed"  # 257^3, 7 levels

    p = P()
    n3 = 257.0 ** 3
    assert bench.phase_bytes(p, 7, "pre-smooth", 4) == 2 * 7 * 4 * n3
    assert bench.phase_bytes(p, 7, "pre-smooth", 4, True) == 2 * 13 * n3
    assert bench.phase_bytes(p, 7, "defect", 4, True) == 13 * n3
    assert bench.phase_bytes(p, 0, "residual", 4) == 52 * n3
    assert bench.phase_bytes(p, 0, "residual", 4, True) == 21 * n3
    assert bench.phase_kernel(p, 7, "pre-smooth", True)[0] == \
        "gs7_code_color_kernel"
    assert bench.phase_kernel(p, 7, "pre-smooth")[0] == \
        "gs7_split_color_kernel"
    assert bench.phase_kernel(p, 0, "residual", True)[0] == \
        "defect_norm_code_kernel"
    assert bench.phase_kernel(p, 6, "pre-smooth", True)[0] == \
        "gs27_tma_kernel"
    p.precision = "fp64"
    assert bench.phase_kernel(p, 4, "pre-smooth")[0] == "gs27_phase_kernel"


def test_c_header_compiles_as_c99(tmp_path):
    """include/pmg_b200.h is the C ABI: plain C99, no C++ or CUDA types."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("gcc not found")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "abi.c"
    src.write_text('#include "pmg_b200.h"\nint main(void) { return 0; }\n')
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-pedantic", "-I",
                    os.path.join(root, "include"), "-c", str(src), "-o",
                    str(tmp_path / "abi.o")], check=True)


def test_packed_operator_rows_checked():
    """pmgc's packed-operator entry points take 4 (7-point) or 14 (27-point)
    rows; anything else is refused before any device call."""
    torch = pytest.importorskip("torch")
    from multigrid_b200 import pmgc
    with pytest.raises(ValueError):
        pmgc._packed(torch.zeros(5, 8))
    with pytest.raises(ValueError):
        pmgc._packed(torch.zeros(14))
    with pytest.raises(TypeError):  # host tensors are refused
        pmgc._packed(torch.zeros(4, 8))
