"""Seeded synthetic scenes for the MPM workloads.

No public dataset is involved: the reference only uses procedural scenes.
Every generator takes a seed and uses numpy's PCG64 generator
(``numpy.random.default_rng(seed)``), so a scene is a pure function of its
arguments.

* ``cube_scene``      — one jittered cube on a 2x2x2-per-cell sub-lattice
                        (64^3 grid, dx = 1/64, cube [0.3, 0.7]^3 → 51^3 =
                        132,651 particles; or its 128^3 / 1M-particle scale-up).
* ``boxes_scene``     — several seeded random boxes at 8 particles per cell,
                        each with its own material (elastic with a per-box
                        Young's modulus, or snow).  The 256^3 / 16M-particle
                        single large scene is ``boxes_scene(256, 16_000_000)``.
* ``batch_scenes``    — many independent scenes of uneven grid and particle
                        size (log-uniform 32^3..128^3 grids, 10k..2M
                        particles), half elastic, half snow.
* ``fill_box_lcg``    — the jittered-lattice box fill with the 64-bit LCG used
                        by molla's MPM tests (crates/molla-solvers/tests/mpm_gpu.rs:174-199).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Elastic material: the reference has no pure-elastic rheology; Viscous with
# zero damping leaves the fixed-corotated stress and F unprojected apart from
# the [0.05, 20] singular-value safety clamp.
ELASTIC = {"kind": 2, "velocity_damping": 0.0, "affine_damping": 0.0}
SNOW = {"kind": 1, "theta_c": 2.5e-2, "theta_s": 7.5e-3, "hardening": 10.0}


@dataclass
class Scene:
    """Positions, material table and stepping constants of one scene."""

    grid_size: int
    cell_size: float
    origin: tuple
    positions: np.ndarray          # (n, 3) float32
    rows: list                     # material rows (dicts)
    ids: np.ndarray                # (n,) uint32 material row per particle
    particle_mass: float
    particle_volume: float
    youngs: float
    poisson: float
    dt: float
    gravity_y: float = -9.8
    boundary_friction: float = 0.0
    walls: int = 0                 # 0 reference walls, 1 sticky
    boundary_pad: int = 0          # 0 -> 2 (reference)
    steps: int = 1000
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])


def _lattice(lo, count, h, rng, jitter=0.5):
    """Points lo + (i + 0.5) h on a count^3 lattice with uniform jitter of
    +/- jitter*h per axis."""
    idx = np.arange(count, dtype=np.float64)
    g = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), axis=-1).reshape(-1, 3)
    pts = np.asarray(lo, np.float64) + (g + 0.5) * h
    pts += rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    return pts.astype(np.float32)


def cube_scene(grid_size: int = 64, per_axis: int | None = None, seed: int = 0, walls: int = 0,
               youngs: float = 1.0e4, poisson: float = 0.2, rho: float = 1.0, dt: float | None = None,
               steps: int = 1000) -> Scene:
    """Elastic cube [0.3, 0.7]^3 in the unit box on a 2x2x2-per-cell lattice.

    64^3 → 51 particles per axis (132,651); 128^3 defaults to 100 per axis
    (1,000,000).  dt defaults to 1e-4 at 64^3 (CFL number c_p dt / dx = 0.67
    for E = 1e4, nu = 0.2, rho = 1) and scales with dx, keeping the same CFL
    number on finer grids (5e-5 at 128^3)."""
    dx = 1.0 / grid_size
    if dt is None:
        dt = 1.0e-4 * 64.0 / grid_size
    if per_axis is None:
        per_axis = 51 if grid_size == 64 else (100 if grid_size == 128 else int(0.4 * grid_size * 2))
    h = 0.4 / per_axis
    rng = np.random.default_rng(seed)
    pos = _lattice((0.3, 0.3, 0.3), per_axis, h, rng)
    vol = dx ** 3 / 8.0
    return Scene(grid_size=grid_size, cell_size=dx, origin=(0.0, 0.0, 0.0), positions=pos, rows=[dict(ELASTIC)],
                 ids=np.zeros(pos.shape[0], np.uint32), particle_mass=rho * vol, particle_volume=vol,
                 youngs=youngs, poisson=poisson, dt=dt, walls=walls, boundary_pad=3 if walls == 1 else 0,
                 steps=steps, meta={"kind": "cube", "seed": seed, "rho": rho})


def cfl_dt(youngs: float, poisson: float, rho: float, dx: float, cfl: float = 0.5) -> float:
    """dt = cfl * dx / c_p with c_p = sqrt((lambda + 2 mu) / rho)."""
    mu = youngs / (2 * (1 + poisson))
    lam = youngs * poisson / ((1 + poisson) * (1 - 2 * poisson))
    return cfl * dx / math.sqrt((lam + 2 * mu) / rho)


def _random_boxes(rng, grid_size, n_boxes, cells_total, margin_cells):
    """Non-overlapping axis-aligned boxes (in cells) whose volumes sum to
    about cells_total."""
    lo_lim, hi_lim = margin_cells, grid_size - margin_cells
    weights = rng.uniform(0.5, 1.5, size=n_boxes)
    vols = weights / weights.sum() * cells_total
    boxes = []
    for v in vols:
        for _ in range(2000):
            aspect = rng.uniform(0.6, 1.6, size=3)
            aspect /= aspect.prod() ** (1 / 3)
            ext = np.maximum(np.round(aspect * v ** (1 / 3)).astype(int), 2)
            ext = np.minimum(ext, hi_lim - lo_lim)
            lo = np.array([rng.integers(lo_lim, hi_lim - e + 1) for e in ext])
            hi = lo + ext
            if all(np.any(hi <= b[0]) or np.any(lo >= b[1]) for b in boxes):
                boxes.append((lo, hi))
                break
        else:
            raise RuntimeError("could not place non-overlapping boxes")
    return boxes


def boxes_scene(grid_size: int = 256, n_particles: int = 16_000_000, n_boxes: int = 4, seed: int = 1,
                rho: float = 16.0, poisson: float = 0.2, e_range=(1.0e4, 1.0e5), dt: float = 2.0e-5,
                steps: int = 500, snow_fraction: float = 0.5, margin_cells: int = 4) -> Scene:
    """Seeded random boxes at 8 particles per cell (2x2x2 jittered sub-lattice).

    Each box is elastic (Viscous{0,0} with its own Young's modulus drawn
    log-uniform in e_range — the per-row modulus extension) or snow
    (theta_c 2.5e-2, theta_s 7.5e-3, hardening 10) with the same draw.
    rho = 16 keeps dt = 2e-5 below half the CFL limit at E = 1e5 on
    dx = 1/256 (c_p ≈ 83 m/s, dt c_p / dx ≈ 0.43)."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / grid_size
    cells_total = n_particles / 8.0
    boxes = _random_boxes(rng, grid_size, n_boxes, cells_total, margin_cells)
    rows, pos_list, id_list = [], [], []
    for b, (lo, hi) in enumerate(boxes):
        e = float(math.exp(rng.uniform(math.log(e_range[0]), math.log(e_range[1]))))
        row = dict(SNOW) if rng.uniform() < snow_fraction else dict(ELASTIC)
        row["youngs"] = e
        row["poisson"] = poisson
        rows.append(row)
        ext = (hi - lo) * 2  # sub-lattice points per axis
        h = dx / 2
        idx = [np.arange(k, dtype=np.float64) for k in ext]
        g = np.stack(np.meshgrid(*idx, indexing="ij"), axis=-1).reshape(-1, 3)
        p = lo * dx + (g + 0.5) * h
        p += rng.uniform(-0.5 * h, 0.5 * h, size=p.shape)
        pos_list.append(p.astype(np.float32))
        id_list.append(np.full(p.shape[0], b, np.uint32))
    pos = np.concatenate(pos_list)
    ids = np.concatenate(id_list)
    vol = dx ** 3 / 8.0
    return Scene(grid_size=grid_size, cell_size=dx, origin=(0.0, 0.0, 0.0), positions=pos, rows=rows, ids=ids,
                 particle_mass=rho * vol, particle_volume=vol, youngs=float(e_range[1]), poisson=poisson, dt=dt,
                 steps=steps, meta={"kind": "boxes", "seed": seed, "rho": rho,
                                    "boxes": [(lo.tolist(), hi.tolist()) for lo, hi in boxes]})


def batch_scenes(count: int = 64, seed: int = 3, n_range=(1.0e4, 2.0e6), grid_range=(32, 128),
                 rho: float = 16.0, poisson: float = 0.2, max_fill: float = 0.25) -> list:
    """Independent scenes of uneven size: grid N log-uniform in grid_range,
    particle count log-uniform in n_range (capped at 8 ppc over max_fill of
    the grid), one or two boxes, elastic or snow 50/50, dt at CFL 0.4."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n_grid = int(round(math.exp(rng.uniform(math.log(grid_range[0]), math.log(grid_range[1])))))
        n_part = int(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1]))))
        n_part = int(min(n_part, 8 * max_fill * n_grid ** 3))
        e = float(math.exp(rng.uniform(math.log(1.0e4), math.log(1.0e5))))
        s = boxes_scene(grid_size=n_grid, n_particles=n_part, n_boxes=1, seed=int(rng.integers(1 << 31)), rho=rho,
                        poisson=poisson, e_range=(e, e * 1.0000001), dt=1.0, steps=0,
                        snow_fraction=0.5, margin_cells=3)
        s.dt = cfl_dt(e, poisson, rho, 1.0 / n_grid, cfl=0.4)
        s.meta["index"] = i
        out.append(s)
    return out


def fill_box_lcg(lo, hi, per_axis: int, seed: int) -> np.ndarray:
    """Jittered lattice box with the 64-bit LCG of molla's MPM tests
    (s = s * 6364136223846793005 + 1442695040888963407, jitter 5% of the
    spacing; crates/molla-solvers/tests/mpm_gpu.rs:174-199)."""
    mask = (1 << 64) - 1
    s = seed & mask

    def nxt():
        nonlocal s
        s = (s * 6364136223846793005 + 1442695040888963407) & mask
        return float(np.float32(np.float32(s >> 32) / np.float32(4294967295.0)) * np.float32(2.0) - np.float32(1.0))

    lo = [np.float32(v) for v in lo]
    hi = [np.float32(v) for v in hi]
    d = [np.float32((hi[a] - lo[a]) / np.float32(per_axis)) for a in range(3)]
    out = []
    for ix in range(per_axis):
        for iy in range(per_axis):
            for iz in range(per_axis):
                p = []
                for a, i in enumerate((ix, iy, iz)):
                    j = np.float32(nxt())
                    p.append(np.float32(lo[a] + (np.float32(i) + np.float32(0.5)) * d[a]
                                        + np.float32(0.05) * d[a] * j))
                out.append(p)
    return np.asarray(out, np.float32)
