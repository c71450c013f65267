"""Benchmark: linearized PB solves/s with the B200 PMG solver.

A step is one PB solve of the workload from device-resident fine-level
inputs: load the fine level (device copy), build the Galerkin hierarchy,
V-cycles until the relative residual is below 1e-10. The default workload is
the 257^3 grid (5 levels, 0.4 A, synthetic 5000-atom molecule) solved in
mixed precision (float V-cycles inside double iterative refinement); the
same run also times the plain FP64 solve.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--workload pb257|pb161|pb65] [--precision mixed|fp64]

--impl reference times the reference's own PMG class on the host cores
(oracle/_ref, built from the reference sources; the CPU restatement when it
is absent) on bounded samples of the same workload. Under torchrun every rank
solves its own replica (the solve does not shard); value = all ranks'
solves / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PB solves/s at rel. residual 1e-10"
UNIT = "solves/s"
TOL = 1e-10
MAX_CYCLES = 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pb257")
    ap.add_argument("--precision", default="mixed",
                    choices=["mixed", "fp64", "fp64-fast"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # skip the batched (96 molecules) and serving (Poisson load) legs
    ap.add_argument("--no-extras", action="store_true")
    # one precision, no end-to-end or kernel legs, cycles driven from the
    # host: a short run for kernel profilers
    ap.add_argument("--quick", action="store_true")
    # the mixed path's 27-point smoother with per-point loads instead of
    # tiles staged by tensor-memory access (the same bits)
    ap.add_argument("--no-tma", action="store_true")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}",
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(parts)
            except Exception:
                pass
        os.unlink(self.path)
        sm = [float(r[1].split()[0]) for r in rows if r[1].split()[0]
              .replace(".", "").isdigit()]
        mx = [float(r[2].split()[0]) for r in rows if r[2].split()[0]
              .replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(
            seconds=600), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    """The slowest rank's time (every rank gets it): the job is done when
    the last replica is."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world: int, steps: int, ms: float) -> float:
    """Whole-job solves/s of `world` independent replicas that each ran
    `steps` solves, the slowest in `ms` milliseconds."""
    return world * steps / (ms / 1000.0)


# ---------------------------------------------------------------------------
# CPU baseline: reference class (or the restatement) on bounded samples
# ---------------------------------------------------------------------------
def workload_defs():
    """The workload definitions (multigrid_b200/molecule.py: pure Python and
    numpy), loaded by file path so that the reference arm never imports the
    package and so never maps the CUDA library into its process."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "pmg_workloads", os.path.join(ROOT, "multigrid_b200", "molecule.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look the module up
    spec.loader.exec_module(mod)
    return mod


def oracle_fine(w):
    """Fine-level inputs of workload w built by the oracle's own set-up
    (oracle/pmg_oracle_setup.c, bit for bit the product's host set-up)."""
    from oracle.oracle import Restatement
    return Restatement().setup_fine(w.n, w.h, w.atoms(), w.physics)


def cpu_sample(w, fine, fp64_cycles: int, solves: int = 1):
    """Times complete solves of the reference class on the host cores (class
    construction, hierarchy build, V-cycles to rel. residual 1e-10; OpenMP,
    all cores). Without the reference build, the single-threaded restatement
    is timed on hierarchy build + 2 V-cycles and extrapolated to
    fp64_cycles cycles (a full solve would take minutes). The reference's
    potential of the last solve is returned under "x" (not printed)."""
    from oracle.oracle import Reference, Restatement, reference_available
    cores = os.cpu_count() or 1
    if reference_available(omp=True):
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
        ref = Reference(omp=True)
        times, cycles, x = [], None, None
        for _ in range(max(1, solves)):
            t0 = time.perf_counter()
            x, cycles, hist = ref.solve(w.base, w.nlev, fine, tol=TOL,
                                        max_cycles=MAX_CYCLES)
            times.append(time.perf_counter() - t0)
        t = statistics.median(times)
        return {
            "value": 1.0 / t, "unit": UNIT, "cores": cores,
            "kind": "reference",
            "sample": (f"{w.name}: {len(times)} complete reference solve(s) "
                       f"(class set-up, hierarchy build, {cycles} FP64 "
                       f"V-cycles to rel. residual {hist[-1] / hist[0]:.2e}),"
                       f" median {t:.2f} s"),
            "cycles": cycles, "x": x,
        }
    ref = Restatement()
    t0 = time.perf_counter()
    ref.solve(w.base, w.nlev, fine, tol=0.0, max_cycles=0)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.solve(w.base, w.nlev, fine, tol=0.0, max_cycles=2)
    t_cyc = (time.perf_counter() - t0 - t_build) / 2
    t_solve = t_build + fp64_cycles * max(t_cyc, 0.0)
    return {
        "value": 1.0 / t_solve, "unit": UNIT, "cores": 1, "kind": "port",
        "sample": (f"{w.name}: hierarchy build ({t_build:.2f} s) + 2 FP64 "
                   f"V-cycles ({t_cyc:.2f} s each) of the restatement, "
                   f"extrapolated to {fp64_cycles} cycles"),
    }


# A reference solve at 257^3 takes 5-11 s on 16 host cores: the arm times at
# most this many steps after at most this many warm-up solves.
REF_STEP_CAP = 10
REF_WARMUP_CAP = 1


def run_reference(args):
    """The reference's own PMG class on the host cores (rank 0 only): at
    most REF_WARMUP_CAP untimed solves, then at most REF_STEP_CAP timed
    complete solves. The inputs come from the oracle's set-up; nothing of
    the product is loaded in this process."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    WORKLOADS = workload_defs().WORKLOADS
    if args.workload not in WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"{args.workload}: the reference solves one "
                          "molecule per process; its arm is timed on the "
                          "single-solve workloads"}))
        return 0
    w = WORKLOADS[args.workload]
    fine = oracle_fine(w)
    # FP64 cycle count of this workload (used only by the extrapolated
    # restatement fallback)
    cycles = {"pb65": 13, "pb161": 16, "pb257": 24}.get(w.name, 24)
    warm = min(args.warmup, REF_WARMUP_CAP)
    if warm:
        cpu_sample(w, fine, cycles, solves=warm)
    steps = max(1, min(args.steps, REF_STEP_CAP))
    base = cpu_sample(w, fine, cycles, solves=steps)
    base.pop("x", None)
    v = base["value"]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": world, "steps": steps, "warmup": warm,
        "steps_requested": args.steps, "warmup_requested": args.warmup,
        "step_cap": REF_STEP_CAP, "warmup_cap": REF_WARMUP_CAP,
        "ms_per_step": 1000.0 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "precision": "fp64", "levels_used": w.nlev,
        "data": "synthetic", "config": workload_config(w),
        "cpu_baseline": base,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def workload_config(w):
    """The workload (the same dict in both arms; how a solve computes it,
    precision and hierarchy depth, is reported beside the config)."""
    return {
        "workload": (f"{w.name}: {w.n}^3 grid, {w.nlev} levels, h {w.h} A, "
                     f"{w.natoms}-atom synthetic molecule, linearized PBE, "
                     f"Galerkin PMG V-cycles to rel. residual 1e-10"),
        "grid": w.n, "levels": w.nlev, "spacing_A": w.h, "atoms": w.natoms,
        "tol": TOL,
        "l2_flush": "inputs larger than L2 (fine level 4+2 arrays of n^3)",
    }


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def phase_bytes(p, level: int, phase: str, esz: int,
                coded: bool = False) -> float | None:
    """Algorithmic bytes moved by one occurrence of a cycle phase (counted in
    arrays of the level's n^3 points; see the kernel table of the design
    notes)."""
    from multigrid_b200.molecule import level_n
    n3 = float(level_n(p.base, level) ** 3) if level >= 1 else 0.0
    nf3 = float(p.n ** 3)
    fine = level == p.nlev
    nc3 = float(level_n(p.base, level - 1) ** 3) if level >= 2 else 0.0
    if level == 0:
        # the refinement paths' residual reads the code byte and writes the
        # split right-hand side; FP64's stop-test norm reads the arrays
        if phase == "residual" and coded and p.precision != "fp64":
            return nf3 * (2 * 8 + 1 + (4 if p.precision == "mixed" else 8))
        if phase == "residual":  # 4 coefficients + f + x in double
            return nf3 * (6 * 8 + (4 if p.precision == "mixed" else 0))
        if phase == "refine-update":  # x64 read/write, e32 read
            return nf3 * (8 + 4 + 8)
        return None
    if fine and coded and phase in ("pre-smooth", "post-smooth"):
        # per sweep: the code byte (couplings and oC), f, x read once and
        # written once
        return 2 * (3 * esz + 1) * n3
    if fine and coded and phase == "defect":  # code, f, x, r
        return (3 * esz + 1) * n3
    arrays = {"pre-smooth": 2 * (7 if fine else 17),
              "post-smooth": 2 * (7 if fine else 17),
              "defect": 7 if fine else 17}
    if phase in arrays:
        return arrays[phase] * n3 * esz
    if phase == "restrict":  # fine r; coarse 27 P + f
        return (n3 + 28 * nc3) * esz
    if phase == "interp":  # coarse x + 27 P; fine x read and written
        return (2 * n3 + 28 * nc3) * esz
    if phase == "damping":  # on the level below, double accumulators
        return 16 * nc3 * esz
    return None


# kernel launched by a cycle phase, and launches per phase occurrence
def phase_kernel(p, level: int, phase: str, coded: bool = False,
                 streamed: bool = False):
    if phase in ("pre-smooth", "post-smooth"):
        if level < p.nlev:
            # the mixed path's padded float levels stage their tiles by
            # tensor-memory access
            return ("gs27_tma_kernel" if p.precision == "mixed"
                    else "gs27_phase_kernel", 4)
        # the refinement paths' finest level is colour-split (and coded
        # when its couplings have two values per direction); its colour
        # passes stream their rows through shared memory
        if streamed:
            return ("gs7_stream_kernel", 4)
        if coded:
            return ("gs7_code_color_kernel", 4)
        if p.precision != "fp64":
            return ("gs7_split_color_kernel", 4)
        return ("gs7_color_kernel", 4)
    if phase == "defect" and level == p.nlev and coded:
        return ("defect7_code_kernel", 1)
    if phase == "residual" and streamed:
        return ("defect_norm_stream_kernel", 1)
    if phase == "residual" and coded:
        return ("defect_norm_code_kernel", 1)
    return {"residual": ("defect_norm_kernel", 1),
            "defect": ("defect_kernel", 1),
            "restrict": ("restrict_kernel", 1),
            "interp": ("interp_add_kernel", 1)}.get(phase, (None, 0))


def profiled_traffic(kernel: str | None, launches: int, workload: str,
                     precision: str):
    """DRAM bytes (read + write) of one phase occurrence from the committed
    ncu summary profiles/<kernel>_<workload>_<precision>.md (its
    'dram_bytes_per_launch:' line) times the phase's launches; None when no
    capture exists for this kernel and workload."""
    import re
    if not kernel:
        return None
    path = os.path.join(ROOT, "profiles",
                        f"{kernel}_{workload}_{precision}.md")
    try:
        with open(path) as f:
            m = re.search(r"^dram_bytes_per_launch:\s*([0-9.e+]+)", f.read(),
                          re.M)
    except OSError:
        return None
    return float(m.group(1)) * launches if m else None


def profile_solve(p, step, dev, esz, coded=False):
    """One extra solve with CUDA events recorded around every cycle phase
    inside the cycle graph; returns per-phase averages and bandwidths
    (coded: the finest couplings are read as code bytes)."""
    p.set_profiling(True)
    p.profile(reset=True)
    step(p, dev)
    prof = p.profile(reset=True)
    p.set_profiling(False)
    rows = []
    for (L, ph), (ms, cnt) in prof.items():
        avg_ms = ms / cnt
        b = phase_bytes(p, L, ph, esz if L != 1 else 8, coded)
        rows.append({"level": L, "phase": ph, "ms_total": ms, "count": cnt,
                     "us_avg": 1000 * avg_ms,
                     "gbs": (b / (avg_ms / 1000) / 1e9) if b else None,
                     "bytes": b})
    rows.sort(key=lambda r: -r["ms_total"])
    return rows


def run_e2e_pipelined(w, precision, host, steps, world):
    """End to end through the C ABI from pinned host buffers: every step
    copies the six fine-level arrays in (pmg_problem_set_fine), builds the
    hierarchy, solves (pmg_solve_start / pmg_solve_finish) and copies the
    potential out (pmg_get_potential_async). Three problem handles on three
    streams take the steps in turn, so a step's copies overlap the others'
    solves (with two, a step's copies waited behind the solve in flight:
    28.0 against 30.5 solves/s at pb257). Timed with CUDA events on the
    first handle's stream, which waits for the others' last events."""
    import ctypes
    import torch
    from multigrid_b200 import PBELinearProblem, _lib
    keys = ("oC", "oE", "oN", "uC", "f", "x0")
    n3 = w.n ** 3
    nh = 3
    probs = [PBELinearProblem(w.base, w.nlev, w.box, precision, w.physics)
             for _ in range(nh)]
    outs = [torch.empty(n3, dtype=torch.float64).pin_memory()
            for _ in range(nh)]
    streams = [torch.cuda.ExternalStream(p.stream) for p in probs]
    ptrs = [ctypes.c_void_p(host[k].data_ptr()) for k in keys]
    pending = [False] * nh

    def issue(q):
        p = probs[q]
        if pending[q]:
            _lib.check("pmg_solve_finish", _lib.lib.pmg_solve_finish(
                p._h, None, None, None))
        _lib.check("pmg_problem_set_fine",
                   _lib.lib.pmg_problem_set_fine(p._h, *ptrs))
        _lib.check("pmg_build_hierarchy",
                   _lib.lib.pmg_build_hierarchy(p._h, 0))
        _lib.check("pmg_solve_start",
                   _lib.lib.pmg_solve_start(p._h, TOL, MAX_CYCLES))
        _lib.check("pmg_get_potential_async",
                   _lib.lib.pmg_get_potential_async(
                       p._h, ctypes.c_void_p(outs[q].data_ptr())))
        pending[q] = True

    def drain():
        for q in range(nh):
            if pending[q]:
                _lib.check("pmg_solve_finish", _lib.lib.pmg_solve_finish(
                    probs[q]._h, None, None, None))
                pending[q] = False

    for q in range(2 * nh):  # warm-up: builds, tuning, graph captures
        issue(q % nh)
    drain()
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(streams[0])
    for st in streams[1:]:
        st.wait_event(e0)
    for i in range(steps):
        issue(i % nh)
    for st in streams[1:]:
        mid = torch.cuda.Event()
        mid.record(st)
        streams[0].wait_event(mid)
    e1.record(streams[0])
    drain()
    torch.cuda.synchronize()
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    for p in probs:
        p.close()
    return {"value": world * steps / (ms / 1000.0), "unit": UNIT,
            "h2d_bytes_per_step": 6 * n3 * 8, "d2h_bytes_per_step": n3 * 8,
            "steps": steps,
            "path": "fine-level arrays from pinned host memory "
                    "(pmg_problem_set_fine), build, solve, potential to "
                    "pinned host memory (pmg_get_potential_async); three "
                    "handles on three streams, copies overlapping the "
                    "other handles' solves"}


# ---------------------------------------------------------------------------
# batched solves and serving (molecules of the batched set)
# ---------------------------------------------------------------------------
def batch_molecules(count: int):
    from multigrid_b200.molecule import batch_workloads
    return [(w, w.atoms()) for w in batch_workloads(count)]


def run_batch(count: int = 96, reps: int = 2, warm: int = 1) -> dict:
    """`count` molecules of the batched set (97^3-161^3 grids, 200-6000
    atoms), each a full solve from its atoms (GPU set-up, hierarchy,
    V-cycles to 1e-10, potential copied out): all in flight at once through
    the serving runtime (mixed and FP64), against the same solves one after
    another through the problem handle (plain FP64). Wall time between
    device synchronisations (the work spans many streams)."""
    import ctypes
    import torch
    from multigrid_b200 import PBELinearProblem, _lib
    from multigrid_b200.serve import Server
    mols = batch_molecules(count)
    outs = [torch.empty(w.n ** 3, dtype=torch.float64, device="cuda")
            for w, _ in mols]
    out = {"molecules": count,
           "grids": sorted({w.n for w, _ in mols}),
           "levels": sorted({w.nlev for w, _ in mols})}
    for prec in ("mixed", "fp64"):
        times, cycles = [], []
        with Server(120 << 30, max_inflight=count) as srv:
            for rep in range(warm + reps):
                torch.cuda.synchronize()
                t = time.perf_counter()
                for i, (w, at) in enumerate(mols):
                    srv.submit(w.base, w.nlev, w.box, None, prec,
                               out=outs[i], tag=rep * count + i, atoms=at,
                               physics=w.physics)
                done = srv.drain(count)
                torch.cuda.synchronize()
                if rep >= warm:
                    times.append(time.perf_counter() - t)
                bad = [c.message for c in done if not c.ok]
                if bad:
                    raise RuntimeError(f"batched {prec} solve failed: {bad[0]}")
                cycles = [c.cycles for c in done]
            st = srv.stats()
        t = statistics.median(times)
        out[f"concurrent_{prec}"] = {
            "solves_per_s": count / t, "ms": 1000 * t,
            "cycles_min": min(cycles), "cycles_max": max(cycles),
            "peak_device_gib": st["peak_bytes"] / 2 ** 30}
    # the same solves one after another through the problem handle (the
    # mixed ones with the mixed path's deeper hierarchy, as the server runs
    # them), for the gain of running them concurrently
    from multigrid_b200.molecule import level_n, levels_for
    for prec in ("fp64", "mixed"):
        probs = {}
        times = []
        for rep in range(warm + reps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            for i, (w, at) in enumerate(mols):
                b, nl = w.base, w.nlev
                if prec == "mixed":
                    b, nl = levels_for(level_n(b, nl), max_levels=12,
                                       min_coarse=5)
                if (b, nl) not in probs:
                    probs[b, nl] = PBELinearProblem(b, nl, w.box, prec,
                                                    w.physics)
                p = probs[b, nl]
                p.set_atoms(at)
                p.buildmultilevelops()
                p.solve(TOL, MAX_CYCLES)
                _lib.check("pmg_get_potential", _lib.lib.pmg_get_potential(
                    p._h, ctypes.c_void_p(outs[i].data_ptr())))
            torch.cuda.synchronize()
            if rep >= warm:
                times.append(time.perf_counter() - t)
        for p in probs.values():
            p.close()
        t = statistics.median(times)
        out[f"sequential_{prec}"] = {"solves_per_s": count / t, "ms": 1000 * t}
    t = out["sequential_fp64"]["ms"] / 1000
    out["speedup_concurrent_mixed_vs_sequential_fp64"] = (
        out["concurrent_mixed"]["solves_per_s"] / (count / t))
    out["speedup_concurrent_vs_sequential_mixed"] = (
        out["concurrent_mixed"]["solves_per_s"] /
        out["sequential_mixed"]["solves_per_s"])
    return out


def run_serving(count: int = 128,
                loads=(0.25, 0.5, 0.75, 0.9, 1.1)) -> dict:
    """Open-loop Poisson arrivals of PB solve requests (molecules of the
    batched set, from atoms) at rates swept up to past saturation, through
    the serving runtime with a 120 GB budget; p50/p99 latency (submit to
    potential on the device) and achieved solves/s per rate, mixed and
    FP64. Saturation = the closed-loop rate with every request in flight."""
    import torch
    from multigrid_b200.serve import Server, open_loop, percentile
    from multigrid_b200.serve import poisson_arrivals
    mols = batch_molecules(count)
    outs = [torch.empty(w.n ** 3, dtype=torch.float64, device="cuda")
            for w, _ in mols]
    res = {"requests_per_rate": count, "budget_gb": 120}
    for prec in ("mixed", "fp64"):
        with Server(120 << 30, max_inflight=32) as srv:
            def submit_one(s, i, prec=prec):
                w, at = mols[i]
                s.submit(w.base, w.nlev, w.box, None, prec, out=outs[i],
                         tag=i, atoms=at, physics=w.physics)
            # warm-up + capacity: everything in flight at once
            for _ in range(2):
                torch.cuda.synchronize()
                t = time.perf_counter()
                for i in range(count):
                    submit_one(srv, i)
                srv.drain(count)
                cap = count / (time.perf_counter() - t)
            rows = []
            for k, f in enumerate(loads):
                rate = f * cap
                arr = poisson_arrivals(rate, count, seed=100 + k)
                done, wall = open_loop(srv, arr, submit_one)
                bad = [c.message for c in done if not c.ok]
                if bad:
                    raise RuntimeError(f"served {prec} solve failed: {bad[0]}")
                lat = [1000 * c.latency for c in done]
                rows.append({"offered_per_s": rate,
                             "achieved_per_s": count / wall,
                             "p50_ms": percentile(lat, 50),
                             "p99_ms": percentile(lat, 99)})
        res[prec] = {"saturation_per_s": cap, "rates": rows}
    return res


def run_mode(args, world: int, rank: int) -> int:
    """--workload batch96 / serve: the batched or serving measurement alone
    (every rank runs its own replica; rank 0 reports)."""
    if args.workload == "batch96":
        res = run_batch(96, reps=max(1, args.steps), warm=max(1, args.warmup))
        value = res["concurrent_mixed"]["solves_per_s"]
        line = {"metric": METRIC + " (batched)", "value": world * value,
                "unit": UNIT, "n_gpus": world, "steps": max(1, args.steps),
                "warmup": max(1, args.warmup),
                "ms_per_step": res["concurrent_mixed"]["ms"],
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic",
                "config": {"workload": "batch96: 96 synthetic molecules, "
                           "200-6000 atoms, 0.5 A, grids 97-161^3, mixed, "
                           "from atoms (GPU set-up), all in flight"},
                "batch": res}
    else:
        res = run_serving(128)
        value = res["mixed"]["saturation_per_s"]
        line = {"metric": "PB solves/s at saturation; p50/p99 latency",
                "value": world * value, "unit": UNIT, "n_gpus": world,
                "steps": 1, "warmup": 2, "ms_per_step": 1000.0 / value,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic",
                "config": {"workload": "serve: open-loop Poisson arrivals "
                           "of batched-set molecules, 120 GB budget"},
                "serving": res}
    if rank == 0:
        print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    # concurrent solves run on many streams: give them hardware queues
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    import torch

    world, rank, local = dist_setup(args)
    if args.workload in ("batch96", "serve"):
        return run_mode(args, world, rank)
    from multigrid_b200 import PBELinearProblem
    from multigrid_b200.molecule import WORKLOADS
    from multigrid_b200.problem import setup_fine

    w = WORKLOADS[args.workload]
    atoms = w.atoms()
    fine = setup_fine(w.n, w.h, atoms, w.physics)
    keys = ("oC", "oE", "oN", "uC", "f", "x0")
    dev = {k: torch.from_numpy(fine[k]).cuda() for k in keys}
    n3 = w.n ** 3

    def step(p, inputs):
        p.set_fine(*[inputs[k] for k in keys])
        p.buildmultilevelops()
        return p.solve(TOL, MAX_CYCLES)

    if args.no_tma:
        from multigrid_b200.problem import set_tma_staging
        set_tma_staging(False)
    if args.quick:
        # profiler runs: launches are serialised and replayed there, so the
        # smoother's tile timings would mean nothing; use the size rule
        from multigrid_b200 import _lib
        _lib.check("pmg_set_autotune", _lib.lib.pmg_set_autotune(0))
    results = {}
    precisions = [args.precision]
    if not args.quick:
        precisions += [q for q in ("mixed", "fp64", "fp64-fast")
                       if q != args.precision]
    for precision in precisions:
        p = PBELinearProblem(w.base, w.nlev, w.box, precision, w.physics)
        if args.quick:
            # profiler runs: kernel profilers do not see kernels inside
            # graphs with conditional nodes, so drive the cycles from the host
            p.set_host_loop(True)
        stream = torch.cuda.ExternalStream(p.stream)
        for _ in range(args.warmup):
            res = step(p, dev)
        torch.cuda.synchronize()
        barrier(world)
        clocks = ClockSampler(torch.cuda.current_device())
        if precision == args.precision:
            clocks.start()
            time.sleep(0.3)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        cyc = []
        l0 = p.launches
        e0.record(stream)
        for _ in range(args.steps):
            res = step(p, dev)
            cyc.append(res.cycles)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = p.launches - l0
        ms = e0.elapsed_time(e1)
        ck = clocks.stop() if precision == args.precision else None
        barrier(world)
        ms = max_over_ranks(world, ms)
        x = p.potential().ravel()
        # the set-up share of a step: fine-level copy and hierarchy build
        build_ms = None
        if not args.quick:
            b0 = torch.cuda.Event(enable_timing=True)
            b1 = torch.cuda.Event(enable_timing=True)
            b0.record(stream)
            for _ in range(3):
                p.set_fine(*[dev[k] for k in keys])
                p.buildmultilevelops()
            b1.record(stream)
            torch.cuda.synchronize()
            build_ms = b0.elapsed_time(b1) / 3
        results[precision] = dict(ms=ms, cycles=cyc, relres=res.relres,
                                  x=x, clocks=ck, p=p, stream=stream,
                                  launches=launches, build_ms=build_ms)

    prim = results[args.precision]
    value = replicas_value(world, args.steps, prim["ms"])
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT,
                              "quick": True, "cycles": prim["cycles"][-1],
                              "ms_per_step": prim["ms"] / args.steps}))
        for r in results.values():
            r["p"].close()
        return 0

    # end to end through the public API from pinned host buffers
    import ctypes
    from multigrid_b200 import _lib
    p = prim["p"]
    stream = prim["stream"]
    host = {k: torch.from_numpy(fine[k]).pin_memory() for k in keys}
    out_host = torch.empty(n3, dtype=torch.float64).pin_memory()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    k_e2e = max(1, min(args.steps, 5))
    barrier(world)
    e0.record(stream)
    for _ in range(k_e2e):
        step(p, host)
        _lib.check("pmg_get_potential", _lib.lib.pmg_get_potential(
            p._h, ctypes.c_void_p(out_host.data_ptr())))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1))
    e2e_serial = {"value": world * k_e2e / (e2e_ms / 1000.0), "unit": UNIT,
                  "h2d_bytes_per_step": 6 * n3 * 8,
                  "d2h_bytes_per_step": n3 * 8,
                  "path": "fine-level arrays from pinned host memory "
                          "(pmg_problem_set_fine), potential to host, one "
                          "step after the other"}
    e2e = run_e2e_pipelined(w, args.precision, host, 3 * k_e2e, world)
    # the class's own entry: atoms in (GPU set-up), potential out
    atoms_host = np.ascontiguousarray(atoms)
    barrier(world)
    e0.record(stream)
    for _ in range(k_e2e):
        p.set_atoms(atoms_host)
        p.buildmultilevelops()
        p.solve(TOL, MAX_CYCLES)
        _lib.check("pmg_get_potential", _lib.lib.pmg_get_potential(
            p._h, ctypes.c_void_p(out_host.data_ptr())))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1))
    e2e_atoms = {"value": world * k_e2e / (e2e_ms / 1000.0), "unit": UNIT,
                 "h2d_bytes_per_step": int(atoms_host.nbytes),
                 "d2h_bytes_per_step": n3 * 8,
                 "path": "atoms from host (pmg_problem_set_atoms: GPU "
                         "set-up), hierarchy build, solve, potential to "
                         "pinned host memory; the set-up is extra work the "
                         "device-resident value excludes"}

    # per-phase timing of one more solve (CUDA events inside the cycle graph,
    # on the solver's stream); the dominant bandwidth-bound phase gives the
    # roofline
    peak, peak_kind = peaks()
    esz = 4 if args.precision == "mixed" else 8
    coded = p.coded_couplings()
    phases = profile_solve(p, step, dev, esz, coded)
    dom = next(r for r in phases if r["gbs"])
    streamed = p.finest_streamed()
    kname, klaunches = phase_kernel(p, dom["level"], dom["phase"], coded,
                                    streamed)
    roofline = {"bound": "hbm",
                "kernel": (f"{kname} x{klaunches}: level {dom['level']} "
                           f"{dom['phase']}"),
                "achieved": dom["gbs"], "peak": peak, "unit": "GB/s",
                "frac": dom["gbs"] / peak,
                "traffic": profiled_traffic(kname, klaunches, w.name,
                                            args.precision),
                "traffic_unit": "bytes per phase occurrence (ncu capture)",
                "peak_source": peak_kind,
                "bytes_basis": (
                    "coded operator: per point one code byte (couplings and "
                    "oC), f, x"
                    if coded and kname and ("code" in kname or
                                            "stream" in kname) else
                    "coefficient arrays as stored (kernel table)"),
                "algorithmic_bytes_per_launch": dom["bytes"],
                "avg_launch_us": dom["us_avg"]}

    def error(x, ref):
        return {"rel_l2": float(np.linalg.norm(x - ref) /
                                np.linalg.norm(ref)),
                "max_norm": float(np.abs(x - ref).max() /
                                  np.abs(ref).max())}

    xm, xd = results["mixed"]["x"], results["fp64"]["x"]
    err = error(xm, xd)

    # the MG-preconditioned CG on the same problems (pmg_pcg_solve: the
    # reference app's outer solver, CG_Solver.h:45-242, with the V-cycle of
    # each precision as preconditioner), to the same relative residual; a
    # reported alternative, not the headline
    pcg = {}
    for precision, r in results.items():
        q, qs = r["p"], r["stream"]

        def pcg_step():
            q.set_fine(*[dev[k] for k in keys])
            q.buildmultilevelops()
            return q.pcg_solve(TOL, MAX_CYCLES)

        for _ in range(args.warmup):
            pr = pcg_step()
        torch.cuda.synchronize()
        barrier(world)
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(qs)
        for _ in range(args.steps):
            pr = pcg_step()
        p1.record(qs)
        torch.cuda.synchronize()
        pms = max_over_ranks(world, p0.elapsed_time(p1))
        pcg[precision] = dict(value=world * args.steps / (pms / 1000.0),
                              ms_per_step=pms / args.steps,
                              iterations=pr.cycles, relres=pr.relres,
                              x=q.potential().ravel().copy())

    cpu = None
    err_oracle = {}
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        try:
            cpu_sample(w, fine, results["fp64"]["cycles"][-1])  # warm-up
            cpu = cpu_sample(w, fine, results["fp64"]["cycles"][-1])
            # the reference's own FP64 potential of the same inputs
            xr = cpu.pop("x", None)
            if xr is not None:
                err_oracle = {prec: error(r["x"], xr)
                              for prec, r in results.items()}
                for prec, r in pcg.items():
                    r["error_vs_oracle"] = error(r["x"], xr)
        except Exception as e:  # reported, never silently replaced
            cpu = {"error": str(e)}

    fp64_value = world * args.steps / (results["fp64"]["ms"] / 1000.0)
    mixed_value = world * args.steps / (results["mixed"]["ms"] / 1000.0)
    fast_value = world * args.steps / (results["fp64-fast"]["ms"] / 1000.0)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": prim["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": workload_config(w),
            "precision": args.precision,
            "levels_used": results[args.precision]["p"].nlev,
            "parallelism": f"replicas x{world}",
            "cycles": prim["cycles"][-1],
            "relres": prim["relres"],
            "fp64": {"value": fp64_value, "cycles":
                     results["fp64"]["cycles"][-1],
                     "ms_per_step": results["fp64"]["ms"] / args.steps,
                     "build_ms": results["fp64"]["build_ms"],
                     "levels": results["fp64"]["p"].nlev,
                     "error_vs_oracle": err_oracle.get("fp64")},
            "mixed": {"value": mixed_value, "cycles":
                      results["mixed"]["cycles"][-1],
                      "ms_per_step": results["mixed"]["ms"] / args.steps,
                      "build_ms": results["mixed"]["build_ms"],
                      "levels": results["mixed"]["p"].nlev,
                      "error_vs_fp64": err,
                      "error_vs_oracle": err_oracle.get("mixed")},
            # the fastest all-double solve: double V-cycles with the mixed
            # path's hierarchy, refinement loop and coded split finest level
            "fp64_fast": {"value": fast_value, "cycles":
                          results["fp64-fast"]["cycles"][-1],
                          "ms_per_step": results["fp64-fast"]["ms"] /
                          args.steps,
                          "build_ms": results["fp64-fast"]["build_ms"],
                          "levels": results["fp64-fast"]["p"].nlev,
                          "error_vs_fp64": error(results["fp64-fast"]["x"],
                                                 xd),
                          "error_vs_oracle": err_oracle.get("fp64-fast")},
            "pcg": {prec.replace("-", "_"): {
                        k: v for k, v in r.items() if k != "x"}
                    for prec, r in pcg.items()},
            "mixed_speedup_vs_fp64": mixed_value / fp64_value,
            "mixed_speedup_vs_best_fp64": mixed_value / max(fp64_value,
                                                            fast_value),
            # against the reference class timed in this run (cpu_baseline):
            # the FP64 GPU solve has the reference's hierarchy and arithmetic
            "speedup_vs_cpu_baseline": (
                {"mixed": mixed_value / cpu["value"],
                 "fp64_same_hierarchy": fp64_value / cpu["value"],
                 "fp64_fast": fast_value / cpu["value"]}
                if cpu and "value" in cpu else None),
            "fine_unknowns_x_cycles_per_s": value * (w.n - 2) ** 3 *
            prim["cycles"][-1],
            "gpu_launches": prim["launches"],
            "e2e": e2e, "e2e_one_at_a_time": e2e_serial,
            "e2e_from_atoms": e2e_atoms,
            "roofline": roofline,
            "phases_top": [{k: (round(v, 3) if isinstance(v, float) else v)
                            for k, v in r.items() if k != "bytes"}
                           for r in phases[:8]],
            "cpu_baseline": cpu,
            "clocks": prim["clocks"],
        }
        if world == 1 and not args.no_extras:
            line["batch"] = run_batch(96)
            line["serving"] = run_serving(128)
        print(json.dumps(line))
    for r in results.values():
        r["p"].close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
