"""Synthetic molecules, grid-size rules and the workloads of the PB solves.

Stands in for molecular input (the reference reads PQR files,
fileio.cc:10-53): atoms uniform in a ball, radii U[1.2, 2.0] A, charges
N(0, 0.4) e shifted so the net charge is an integer. The PRNG is numpy's
PCG64 (np.random.default_rng) with seed = 1000 * config index + molecule id.

Atom rows are (x, y, z, radius, charge) in the grid frame: grid point
(i0, i1, i2) sits at (i0 h, i1 h, i2 h), coordinate 0 on the slowest array
axis, as the reference's Atom::Position (PBE_pmgc_class.h:179-186).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# Physics of the PB workloads: dielectric 2 inside / 78.54 outside with a
# 1.4 A probe, 0.15 M 1:1 salt, ion radius 2.0 A, 298.15 K.
DEFAULT_PHYSICS = dict(eps_in=2.0, eps_out=78.54, ionic_strength=0.15,
                       ion_radius=2.0, temperature=298.15, probe_radius=1.4)
# The reference's compiled-in constants (scientific_quantities.h:9-15) and
# van der Waals marking (no probe).
REFERENCE_PHYSICS = dict(eps_in=4.0, eps_out=78.4, ionic_strength=0.15,
                         ion_radius=2.0, temperature=298.15, probe_radius=0.0)

BATCH_SIZES = (65, 97, 129, 161, 193, 225)


def level_n(base: int, level: int) -> int:
    """Points per axis of level L: base * 2^L + 1 (the class's
    length = base*2^L - 1 plus the shell, MultigridDomain.h:136-141,
    PBE_pmgc_class.h:1166-1173)."""
    return base * (1 << level) + 1


def coarsen(n: int) -> int:
    """Coarse size of an n-point axis, n_c = (n - 1)/2 + 1 (Vcorsr,
    pmgc/mgsubd.cc:395-413)."""
    return (n - 1) // 2 + 1


def grid_step(base: int, nlev: int, box: float) -> float:
    """box / (base * 2^nlev) (PBE_pmgc_class.h:1157-1159)."""
    return box / (base * (1 << nlev))


def levels_for(n: int, max_levels: int = 6, min_coarse: int = 5):
    """(base, nlev) for an n-point axis: the largest nlev <= max_levels with
    n = base * 2^nlev + 1 and a coarsest grid of at least min_coarse
    points."""
    for L in range(max_levels, 1, -1):
        if (n - 1) % (1 << L) == 0 and (n - 1) >> L >= 1:
            base = (n - 1) >> L
            if 2 * base + 1 >= min_coarse:
                return base, L
    raise ValueError(f"no multigrid hierarchy for n = {n}")


def batch_grid(radius: float, h: float = 0.5, margin: float = 10.0) -> int:
    """Smallest n in BATCH_SIZES with (n-1) h >= 2 (R + 2) + margin."""
    need = 2 * (radius + 2.0) + margin
    for n in BATCH_SIZES:
        if (n - 1) * h >= need:
            return n
    return BATCH_SIZES[-1]


def synthetic_atoms(natoms: int, ball_radius: float, seed: int,
                    center: tuple[float, float, float]) -> np.ndarray:
    """natoms x 5 array (x, y, z, radius, charge), uniform in a ball."""
    rng = np.random.default_rng(seed)
    pts = np.empty((0, 3))
    while len(pts) < natoms:
        cand = rng.uniform(-ball_radius, ball_radius, size=(2 * natoms, 3))
        cand = cand[np.einsum("ij,ij->i", cand, cand) <= ball_radius ** 2]
        pts = np.concatenate([pts, cand])
    pts = pts[:natoms] + np.asarray(center, dtype=np.float64)
    radii = rng.uniform(1.2, 2.0, size=natoms)
    q = rng.normal(0.0, 0.4, size=natoms)
    q += (np.round(q.sum()) - q.sum()) / natoms
    return np.column_stack([pts, radii, q]).astype(np.float64)


@dataclasses.dataclass(frozen=True)
class Workload:
    """One PB solve: grid, molecule and physics."""
    name: str
    base: int
    nlev: int
    h: float
    natoms: int
    ball_radius: float
    seed: int
    physics: dict = dataclasses.field(default_factory=lambda: dict(
        DEFAULT_PHYSICS))

    @property
    def n(self) -> int:
        return level_n(self.base, self.nlev)

    @property
    def box(self) -> float:
        return self.h * (self.n - 1)

    def atoms(self) -> np.ndarray:
        c = self.box / 2
        return synthetic_atoms(self.natoms, self.ball_radius, self.seed,
                               (c, c, c))


# The single-solve workloads: 65^3 (4 levels, 0.5 A, 400 atoms in 12 A);
# 161^3 and 257^3 (5 levels, 0.4 A, 5000 atoms in 30 A, one molecule).
WORKLOADS = {
    "pb65": Workload("pb65", 4, 4, 0.5, 400, 12.0, 0),
    "pb161": Workload("pb161", 5, 5, 0.4, 5000, 30.0, 1000),
    "pb257": Workload("pb257", 8, 5, 0.4, 5000, 30.0, 1000),
}


def batch_workloads(count: int = 96, seed0: int = 3000,
                    h: float = 0.5) -> list[Workload]:
    """The batched set: atom counts log-uniform in [200, 6000], ball radius
    30 (N/5000)^(1/3) A, grid from batch_grid, levels from levels_for."""
    rng = np.random.default_rng(seed0)
    out = []
    for m in range(count):
        natoms = int(round(math.exp(rng.uniform(math.log(200),
                                                math.log(6000)))))
        radius = 30.0 * (natoms / 5000.0) ** (1.0 / 3.0)
        n = batch_grid(radius, h)
        base, nlev = levels_for(n)
        out.append(Workload(f"batch{m}", base, nlev, h, natoms, radius,
                            seed0 + m))
    return out
