"""Fused gather + scatter (k_g2p2g) against the separate gather and scatter.

The two paths compute the same substep; only the order of the float atomics
in the grid accumulation differs, so the particle state agrees to float
rounding noise over a few dozen substeps (checked against the oracle's
tolerances by the parity tests, which run the fused path by default).  The
separate path is selected with MOLLA_MPM_FUSED=0 at construction.
"""

import numpy as np
import pytest

import molla_b200 as m
from molla_b200 import scenes

pytestmark = pytest.mark.gpu


def run(engine, scene, svd, steps, interval, chunks=(1,)):
    cfg = m.config_for_scene(scene, svd_precision=svd)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(scene.positions)
    sim.set_materials(scene.rows, scene.ids)
    sim.set_sort_interval(interval)
    for c in chunks:
        sim.step_n(scene.dt, steps // len(chunks))
    C, F, jp = sim.read_particle_state()
    out = dict(pos=sim.read_positions(), vel=sim.read_velocities(), C=C, F=F, jp=jp,
               status=sim.read_active_grid_status(), totals=sim.conservation_totals())
    sim.close()
    return out


@pytest.mark.parametrize("svd,interval", [(1, 4), (0, 3), (1, 1)])
def test_fused_matches_separate_launches(engine, monkeypatch, svd, interval):
    scene = scenes.boxes_scene(grid_size=64, n_particles=120_000, n_boxes=3, seed=5, dt=1.6e-4)
    monkeypatch.setenv("MOLLA_MPM_FUSED", "1")
    fused = run(engine, scene, svd, 24, interval, chunks=(1, 2))
    monkeypatch.setenv("MOLLA_MPM_FUSED", "0")
    split = run(engine, scene, svd, 24, interval, chunks=(1, 2))
    assert fused["status"].fault_bits == 0 and split["status"].fault_bits == 0
    assert fused["status"].completed_substeps == split["status"].completed_substeps == 24
    scale = np.abs(scene.positions).max()
    assert np.abs(fused["pos"] - split["pos"]).max() <= 1e-5 * scale
    vmax = max(np.abs(split["vel"]).max(), 1e-3)
    assert np.abs(fused["vel"] - split["vel"]).max() <= 1e-3 * vmax
    assert np.abs(fused["F"] - split["F"]).max() <= 1e-4
    # the grid mass of the last scatter is the particle mass in both
    np.testing.assert_allclose(fused["totals"][0], split["totals"][0], rtol=1e-6)


def test_fused_deposits_particles_that_left_their_tile(engine, monkeypatch):
    """A fast, never-regrouped block: most particles leave the 6^3 local cells
    of their item and deposit through the global path of the fused kernel;
    grid mass still equals particle mass."""
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    cfg.max_particles = 20_000
    monkeypatch.setenv("MOLLA_MPM_FUSED", "1")
    sim = m.MpmSimulation.new(engine, cfg)
    rng = np.random.default_rng(11)
    pts = rng.uniform(-0.2, 0.2, size=(20_000, 3)).astype(np.float32)
    pts[:, 1] += 0.6
    vel = np.tile(np.array([[30.0, 0.0, 0.0]], np.float32), (len(pts), 1))
    sim.set_particles(pts, vel)
    sim.set_sort_interval(1000)
    sim.step_n(1e-4, 16)
    t = sim.conservation_totals()
    assert not sim.read_active_grid_status().faulted()
    np.testing.assert_allclose(t[0], t[4], rtol=1e-5)
    sim.close()
