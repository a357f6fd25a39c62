"""Parity at the benchmark's own configurations, against the oracle.

* The elastic cube (64^3 grid, 132,651 jittered particles, sticky walls 3
  cells, FP32, dt 1e-4): 1000 substeps in both SVD forms against the FP64
  oracle (FP64 state, FP64 Jacobi SVD to 1e-14), with the grid mass and
  momentum of the last substep.
* The single large scene (256^3 grid, 16M particles in 4 boxes, FP32 +
  FP64 SVD, dt 2e-5): 3 substeps against the oracle's FP32 + FP64-SVD step,
  particle by particle.
* The precision study's cube at 128^3 with 1M particles: 1000 substeps in
  all three modes (FP32, FP32 + FP64 SVD, all-FP64) against the FP64
  oracle.

The reference's own gates are mass to 1e-4 relative with zero momentum at
rest (crates/molla-solvers/tests/mpm_gpu.rs:839-884) and momentum drift
below 1% (mpm_gpu.rs:780-837); the benchmark asks for positions within
1e-4 relative of the FP64 oracle after 1000 substeps.
"""

import numpy as np
import pytest

import molla_b200 as m
from molla_b200 import scenes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_run(engine, scene, svd, steps, grid=True):
    cfg = m.config_for_scene(scene, svd_precision=svd)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(scene.positions)
    sim.set_materials(scene.rows, scene.ids)
    sim.step_n(scene.dt, steps)
    out = {"pos": sim.read_positions().astype(np.float64), "status": sim.read_active_grid_status(),
           "totals": sim.conservation_totals()}
    if grid:
        gm, gp = sim.read_grid_mass_momentum()
        out["grid_mass"] = gm.astype(np.float64)
        out["grid_mom"] = gp.astype(np.float64)
    Cg, Fg, jpg = sim.read_particle_state()
    out["F"] = Fg.astype(np.float64)
    out["jp"] = jpg.astype(np.float64)
    out["vel"] = sim.read_velocities().astype(np.float64)
    sim.close()
    return out, cfg


def fp64_oracle(scene, cfg, steps):
    osc = O.make_scene(cfg, scene.rows, scene.dt, svd_tol=1e-14, svd_sweeps=30)
    st = O.cast_state(O.init_state(scene.positions, mass=cfg.particle_mass, volume=cfg.particle_volume,
                                   ids=scene.ids), np.float64)
    gm, gp = O.step(osc, st, steps, precision="f64", nthreads=O.max_threads(), want_grid=True)
    return st, gm, gp


def rel_max(a, ref):
    return float((np.abs(a - ref) / np.maximum(np.abs(ref), 1e-30)).max())


def check_conservation(g, scene, cfg, ref_gm, ref_gp):
    mass0 = float(np.float32(cfg.particle_mass)) * scene.n
    tot = g["totals"]
    # grid mass of the last substep equals the particle mass (the
    # reference's mass gate, relative 1e-4; here to FP32 summation noise)
    assert abs(tot[0] / mass0 - 1.0) < 1e-6, tot[0] / mass0 - 1.0
    assert abs(g["grid_mass"].sum() / ref_gm.sum() - 1.0) < 1e-6
    # grid momentum against the oracle's grid of the same substep
    mom = g["grid_mom"].reshape(-1, 3).sum(axis=0)
    ref = ref_gp.reshape(-1, 3).sum(axis=0)
    return float(np.linalg.norm(mom - ref) / np.linalg.norm(ref))


@pytest.fixture(scope="module")
def cube64():
    scene = scenes.cube_scene(grid_size=64, seed=0, walls=1)
    assert scene.n == 132651 and scene.grid_size == 64 and scene.dt == 1e-4
    cfg = m.config_for_scene(scene, svd_precision=1)
    st, gm, gp = fp64_oracle(scene, cfg, 1000)
    return scene, st, gm, gp


@pytest.mark.parametrize("svd", [0, 1])
def test_cube64_1000_substeps_vs_fp64_oracle(engine, cube64, svd):
    scene, st, ref_gm, ref_gp = cube64
    g, cfg = gpu_run(engine, scene, svd, 1000)
    assert not g["status"].numerical_fault and g["status"].completed_substeps == 1000
    err = rel_max(g["pos"], st["pos"])
    assert err < 1e-4, err
    mom_err = check_conservation(g, scene, cfg, ref_gm, ref_gp)
    # momentum of the grid against the FP64 oracle's (gravity adds momentum;
    # the reference bounds its drift at 1%)
    assert mom_err < 1e-4, mom_err
    print(f"cube64 svd={svd}: pos rel max {err:.2e}, grid momentum rel {mom_err:.2e}")


def test_large_scene_3_substeps_vs_oracle(engine):
    """The benchmark's 16M-particle scene, particle by particle against the
    oracle's FP32 + FP64-SVD step (same precision, the oracle's FP64 SVD
    converged to 1e-14)."""
    scene = scenes.boxes_scene(grid_size=256, n_particles=16_000_000, n_boxes=4, seed=1)
    g, cfg = gpu_run(engine, scene, 1, 3)
    assert not g["status"].numerical_fault and g["status"].completed_substeps == 3
    osc = O.make_scene(cfg, scene.rows, scene.dt, svd_tol=1e-14, svd_sweeps=30)
    st = O.init_state(scene.positions, mass=cfg.particle_mass, volume=cfg.particle_volume, ids=scene.ids)
    gm, gp = O.step(osc, st, 3, precision="f32_svd64", nthreads=O.max_threads(), want_grid=True)
    dx = np.abs(g["pos"] - st["pos"]).max()
    dv = np.abs(g["vel"] - st["vel"]).max()
    dF = (np.abs(g["F"] - st["F"]) / np.maximum(np.abs(st["F"]), 1.0)).max()
    assert dx < 1e-6, dx
    assert dv < 1e-4 * max(1.0, np.abs(st["vel"]).max()), dv
    assert dF < 1e-5, dF
    assert abs(g["grid_mass"].sum() / gm.astype(np.float64).sum() - 1.0) < 1e-6
    mom = g["grid_mom"].reshape(-1, 3).sum(axis=0)
    ref = gp.astype(np.float64).reshape(-1, 3).sum(axis=0)
    assert np.linalg.norm(mom - ref) / np.linalg.norm(ref) < 1e-4
    print(f"large: |dx| {dx:.2e}, |dv| {dv:.2e}, F rel {dF:.2e}")


def test_precision_study_cube128_1000_substeps(engine):
    """The precision study's scene: all three GPU modes against the FP64
    oracle after 1000 substeps (the benchmark's 1e-4 position gate)."""
    scene = scenes.cube_scene(grid_size=128, seed=0, walls=1)
    assert scene.n == 1_000_000
    steps = 1000
    cfg = m.config_for_scene(scene, svd_precision=1)
    st, ref_gm, ref_gp = fp64_oracle(scene, cfg, steps)
    errs = {}
    for svd in (0, 1):
        g, _ = gpu_run(engine, scene, svd, steps)
        assert not g["status"].faulted() and g["status"].completed_substeps == steps
        errs[svd] = rel_max(g["pos"], st["pos"])
        mom = check_conservation(g, scene, cfg, ref_gm, ref_gp)
        errs[f"mom{svd}"] = mom
    sim64 = m.MpmSimulation64(engine, cfg)
    sim64.set_particles(scene.positions.astype(np.float64))
    sim64.set_materials(scene.rows, scene.ids)
    sim64.step_n(float(np.float32(scene.dt)), steps)
    pos64, _, _ = sim64.read_state()
    sim64.close()
    errs[64] = rel_max(pos64, st["pos"])
    print(f"precision study {steps} substeps:", errs)
    assert errs[0] < 1e-4 and errs[1] < 1e-4
    assert errs["mom1"] < 1e-4 and errs["mom0"] < 1e-4
    assert errs[64] < 1e-9
