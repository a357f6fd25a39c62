"""GPU tests of sparse grid storage (MpmSimulation::new_sparse,
crates/molla-solvers/src/mpm.rs:846-853): a scene whose grid holds only a
fixed number of 4^3-node tiles gives the dense storage's results (within the
1e-5 of the atomic accumulation order), reports its active tiles, and
latches the tile-overflow bit, without a GPU fault, when its particles need
more tiles than it holds (MpmActiveGridStats::overflow, mpm.rs:257-283)."""

import numpy as np
import pytest

import molla_b200 as m
from molla_b200 import scenes

pytestmark = pytest.mark.gpu

TOL = 1e-5


def scene():
    return scenes.boxes_scene(grid_size=64, n_particles=30_000, n_boxes=2, seed=5)


def stencil_tiles(s, pos):
    """Distinct 4^3 tiles the particles' quadratic stencils touch."""
    n = s.grid_size
    base = np.floor((pos.astype(np.float64) - np.asarray(s.origin)) / s.cell_size - 0.5).astype(np.int64)
    tiles = set()
    w = (n + 3) // 4
    for off in np.array(np.meshgrid([0, 2], [0, 2], [0, 2], indexing="ij")).reshape(3, -1).T:
        c = np.clip(base + off, 0, n - 1) >> 2
        tiles.update((c[:, 0] + w * (c[:, 1] + w * c[:, 2])).tolist())
    return len(tiles)


def run(engine, s, steps, tile_capacity=None):
    cfg = m.config_for_scene(s)
    sim = m.MpmSimulation(engine, cfg, tile_capacity)
    sim.set_particles(s.positions)
    sim.set_materials(s.rows, s.ids)
    sim.set_sort_interval(8)
    sim.step_n(s.dt, steps)
    out = sim.read_positions(), sim.read_grid_mass_momentum(), sim.read_active_grid_status(), sim.conservation_totals()
    sim.close()
    return out


def test_sparse_matches_dense(engine):
    s = scene()
    w = (s.grid_size + 3) // 4
    need = stencil_tiles(s, s.positions)
    cap = 3 * need
    assert cap < w ** 3 // 4  # the sparse grid is a small part of the dense one
    pos_d, (gm_d, gp_d), st_d, tot_d = run(engine, s, 40)
    pos_s, (gm_s, gp_s), st_s, tot_s = run(engine, s, 40, tile_capacity=cap)
    assert not st_s.faulted() and st_s.completed_substeps == 40
    assert np.abs(pos_s - pos_d).max() < TOL
    # the grid read back through the tile map equals the dense grid
    assert np.abs(gm_s - gm_d).max() <= 1e-5 * gm_d.max()
    assert np.abs(gp_s - gp_d).max() <= 1e-5 * np.abs(gp_d).max()
    assert abs(tot_s[0] / tot_d[0] - 1.0) < 1e-6
    # the active tiles are those of the last deposit's stencils
    assert need // 2 < st_s.active_tiles <= cap and st_d.active_tiles == 0


def test_sparse_overflow_latches_and_freezes(engine):
    s = scene()
    need = stencil_tiles(s, s.positions)
    cfg = m.config_for_scene(s)
    sim = m.MpmSimulation.new_sparse(engine, cfg, max(1, need // 2))
    sim.set_particles(s.positions)
    sim.set_materials(s.rows, s.ids)
    sim.step_n(s.dt, 3)
    st = sim.read_active_grid_status()
    assert st.overflow and st.faulted() and not st.numerical_fault
    frozen = sim.read_positions()
    sim.step_n(s.dt, 5)
    assert np.array_equal(sim.read_positions(), frozen)
    engine.check_device()  # the engine is still healthy
    sim.close()


def test_sparse_capacity_and_unsupported_modes(engine):
    s = scene()
    cfg = m.config_for_scene(s)
    w = (s.grid_size + 3) // 4
    with pytest.raises(m.SolverError):
        m.MpmSimulation.new_sparse(engine, cfg, w ** 3 + 1)
    with pytest.raises(m.SolverError):
        m.MpmSimulation.new_sparse(engine, cfg, 0)
    sim = m.MpmSimulation.new_sparse(engine, cfg, 64)
    sim.set_particles(s.positions[:100])
    with pytest.raises(m.MollaError):
        sim.set_rigid_spheres([([0.5, 0.5, 0.5], 0.1, [0.0, 0.0, 0.0])])
    sim.close()


def test_group_mixes_sparse_and_dense_scenes(engine):
    ss = scenes.batch_scenes(count=4, seed=21, n_range=(5e3, 3e4), grid_range=(48, 64))
    total = sum(s.n for s in ss)
    caps = [0 if k % 2 else 3 * stencil_tiles(s, s.positions) for k, s in enumerate(ss)]
    cells = sum((c * 64 if c else s.grid_size ** 3) + 256 for s, c in zip(ss, caps))
    g = m.MpmGroup(engine, 8, total, cells)
    ids = [g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt, tile_capacity=c)
           for s, c in zip(ss, caps)]
    g.step(16)
    g.step_graph(8, 2)
    for sid, s in zip(ids, ss):
        pos, _, st, _ = run(engine, s, 32)
        assert np.abs(g.read_positions(sid) - pos).max() < TOL, sid
        assert not g.read_status(sid).faulted()
    g.close()
