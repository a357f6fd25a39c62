"""GPU parity tests: the CUDA path (through the C ABI) against the oracle, the
reference's known-answer tests and the golden fixtures.

Tolerances (FP32 state; atomic accumulation order on the GPU differs from
the oracle's particle-index order, and the GPU path reuses the return
mapping's SVD for the next stress):
  * sort keys / permutations: bit-exact;
  * one substep: |dx| <= 1e-6, |dv| <= 1e-5 * max(1, |v|), F/C/jp within
    2e-5 normalised by max(|a|, 1) (the reference's own `close` bound,
    crates/molla-solvers/src/mpm_particle_order_tests.rs:44-65);
  * many substeps: positions within 1e-4 (absolute, unit box) of the FP32
    oracle and within 1e-4 relative of the FP64 oracle.
"""

import math

import numpy as np
import pytest

import molla_b200 as m
from molla_b200 import scenes
from oracle import oracle as O
from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu
GOLD = G.HERE


def norm_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float((np.abs(a - b) / np.maximum(np.abs(a), 1.0)).max()) if a.size else 0.0


def run_both(engine, cfg, rows, pts, ids, dt, steps, vel=None, precision="f32", chunked=None, sort_interval=None):
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(pts, vel)
    if rows is not None:
        sim.set_materials(rows, ids)
    if sort_interval is not None:
        sim.set_sort_interval(sort_interval)
    if chunked:
        for c in chunked:
            sim.step_n(dt, c)
    else:
        sim.step_n(dt, steps)
    Cg, Fg, jpg = sim.read_particle_state()
    gpu = {"pos": sim.read_positions(), "vel": sim.read_velocities(), "C": Cg, "F": Fg, "jp": jpg,
           "status": sim.read_active_grid_status()}
    eff_rows = rows if rows is not None else [cfg.rheology]
    sc = O.make_scene(cfg, eff_rows, dt)
    st = O.init_state(pts, vel, mass=cfg.particle_mass, volume=cfg.particle_volume, ids=ids)
    O.step(sc, st, steps, precision=precision)
    return sim, gpu, st


# ---- sort: bit-exact permutation ----------------------------------------------

@pytest.mark.parametrize("size", [35, 1536])
def test_sort_permutation_bit_exact(engine, size):
    """mpm_particle_order_tests.rs:67-165: exact keys and identities for
    counts {513, 257, 1, 0, 63} at capacity 513, out-of-grid points clamped."""
    cfg = m.MpmConfig.sand()
    cfg.grid_size = size
    cfg.grid_origin = (-1.0, -1.0, -1.0)
    cfg.cell_size = 0.0625
    cfg.max_particles = 513
    sim = m.MpmSimulation.new(engine, cfg)
    with pytest.raises(m.SolverError):
        sim.set_particle_tile_ordering(True)
    with pytest.raises(m.SolverError):
        sim.prepare_particle_tile_ordering(0)
    with pytest.raises(m.SolverError):
        sim.prepare_particle_tile_ordering(514)
    for count in (513, 257, 1, 0, 63, 513):
        g = np.load(GOLD / f"particle_order_{size}_{count}.npz")
        sim.set_particles(g["positions"][:count])
        keys, ids = sim.read_sort_permutation(513)
        assert np.array_equal(keys, g["keys"]), count
        assert np.array_equal(ids, g["ids"]), count


def test_sort_permutation_capacity_rules(engine):
    """Preparing for 31 then seeding 32 makes step_n fail without moving
    particles (mpm_particle_order_tests.rs:147-156)."""
    cfg = m.MpmConfig.sand()
    cfg.max_particles = 513
    sim = m.MpmSimulation.new(engine, cfg)
    pts = G.points(32) * np.float32(0.5)
    sim.set_particles(pts[:31])
    sim.prepare_particle_tile_ordering(31)
    sim.set_particle_tile_ordering(True)
    sim.set_particles(pts)
    before = sim.read_positions()
    with pytest.raises(m.SolverError):
        sim.step_n(1e-4, 1)
    assert np.array_equal(before, sim.read_positions())
    sim.prepare_particle_tile_ordering(64)
    sim.set_particle_tile_ordering(False)


@pytest.mark.parametrize("name", ["random_1k", "all_equal", "sorted", "reverse", "paired", "high_byte"])
def test_radix_sort_suite(engine, name):
    """radix_sort_gpu.rs:395-520 (stable-sort bit-exactness)."""
    g = np.load(GOLD / f"radix_{name}.npz")
    k, v = m.radix_sort_pairs(engine, g["keys"], g["values"], 32)
    assert np.array_equal(k, g["sorted_keys"]) and np.array_equal(v, g["sorted_values"])


def test_radix_sort_random_100k(engine):
    r = G.lcg(0xBADC0FFEE0DDF00D)
    keys = np.array([r() for _ in range(100_000)], np.uint32)
    vals = np.arange(keys.shape[0], dtype=np.uint32)
    k, v = m.radix_sort_pairs(engine, keys, vals, 32)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])


@pytest.mark.parametrize("n,bits", [(1, 8), (4097, 12), (300_000, 18), (2_000_003, 24)])
def test_radix_sort_sizes_and_widths(engine, n, bits):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = m.radix_sort_pairs(engine, keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])


# ---- known-answer tests on the CUDA path ------------------------------------------

def test_free_fall_exact(engine):
    """mpm_freefall_regression_gpu.rs:76-111."""
    cfg = m.MpmConfig.snow()
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles([[0.013, 0.2, 0.017]])
    dt = 1.0 / 480.0
    for step in range(20):
        sim.step(dt)
        pos = sim.read_positions()
        vel = sim.read_velocities()
        assert abs(vel[0, 1] - (-9.81 * dt * (step + 1))) < 1e-4
        assert abs(vel[0, 0]) < 1e-5 and abs(vel[0, 2]) < 1e-5
        assert abs(pos[0, 0] - 0.013) < 1e-5 and abs(pos[0, 2] - 0.017) < 1e-5
    assert sim.read_active_grid_status().completed_substeps == 20


def test_grid_mass_matches_particle_mass(engine):
    """mpm_gpu.rs:839-884, plus per-cell parity with the oracle's grid."""
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    cfg.grid_origin = (-1.6, -1.6, -1.6)
    cfg.grid_size = 32
    cfg.cell_size = 0.1
    cfg.particle_mass = 2.5e-3
    cfg.boundary_friction = 1.0
    pts = scenes.fill_box_lcg([-0.35] * 3, [0.35] * 3, 7, 19)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(pts)
    sim.step(1.0 / 240)
    gm, gp = sim.read_grid_mass_momentum()
    exp = cfg.particle_mass * len(pts)
    assert (gm > 0).sum() > 0
    assert abs(gm.sum(dtype=np.float64) - exp) / exp < 1e-4
    assert np.abs(gp).max() < 1e-6
    sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 240)
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    om, op = O.step(sc, st, 1, want_grid=True)
    # mpm_perf.rs:364-477 tolerances: per-cell |dm| < 1e-4 or rel < 1e-3
    dm = np.abs(gm - om)
    assert np.all((dm < 1e-4) | (dm / np.maximum(om, 1e-30) < 1e-3))
    assert np.abs(gp - op).max() < 1e-3
    tot = sim.conservation_totals()
    assert abs(tot[0] - exp) / exp < 1e-6 and abs(tot[4] - exp) / exp < 1e-6


def jittered_block_1k():
    """The 10x10x10 block of mpm_perf.rs:377-398: spacing 0.04 from
    (-0.2, 0.2, -0.2), each coordinate jittered by 0.005 * u, u in [-1, 1]
    from a 64-bit LCG (multiplier 6364136223846793005, increment
    1442695040888963407, seed 0xdeadbeef, high 32 bits / u32::MAX)."""
    s = 0xDEADBEEF
    mask = (1 << 64) - 1

    def nxt():
        nonlocal s
        s = (s * 6364136223846793005 + 1442695040888963407) & mask
        return float(np.float32(np.float32(s >> 32) / np.float32(0xFFFFFFFF))) * 2.0 - 1.0

    pts = []
    for ix in range(10):
        for iy in range(10):
            for iz in range(10):
                pts.append([np.float32(-0.2 + 0.04 * ix + 0.005 * nxt()),
                            np.float32(0.2 + 0.04 * iy + 0.005 * nxt()),
                            np.float32(-0.2 + 0.04 * iz + 0.005 * nxt())])
    return np.asarray(pts, np.float32)


def test_p2g_modes_agree_with_each_other_and_the_oracle(engine):
    """mpm_perf.rs:364-477 (legacy vs two-pass P2G): one sand substep of the
    jittered 1k block on a 32^3 grid, grid mass and momentum compared with
    the reference's tolerances.  Both reference modes map to the one tiled
    scatter here, so each is also held to the oracle's grid; the switch
    turns deterministic P2G off and makes prepared steps stale
    (mpm.rs:1642-1650)."""
    cfg = m.MpmConfig.sand()
    cfg.grid_size = 32
    cfg.cell_size = 0.05
    cfg.grid_origin = (-0.8, 0.0, -0.8)
    cfg.max_particles = 4096
    pts = jittered_block_1k()
    dt = 1.0 / 240
    sim = m.MpmSimulation.new(engine, cfg)
    grids = []
    for two_pass in (False, True):
        sim.set_p2g_mode(two_pass)
        sim.set_particles(pts)
        sim.step(dt)
        grids.append(sim.read_grid_mass_momentum())
    (m0, p0), (m1, p1) = grids
    tot0 = m0.sum(dtype=np.float64)
    assert abs(m1.sum(dtype=np.float64) - tot0) / tot0 < 1e-4
    dm = np.abs(m1 - m0)
    assert dm.max() < 1e-4 or (dm / np.maximum(np.abs(m0), 1e-12)).max() < 1e-3
    assert np.abs(p1 - p0).max() < 1e-3
    sc = O.make_scene(cfg, [cfg.rheology], dt)
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    om, op = O.step(sc, st, 1, want_grid=True)
    for gm, gp in grids:
        d = np.abs(gm - om)
        assert np.all((d < 1e-4) | (d / np.maximum(om, 1e-30) < 1e-3))
        assert np.abs(gp - op).max() < 1e-3
    # the switch turns deterministic P2G off and makes prepared steps stale;
    # the getters follow mpm.rs:1245-1252,1689-1694
    assert sim.uses_two_pass_p2g() and not sim.deterministic_p2g_enabled()
    sim.prepare_particle_tile_ordering(cfg.max_particles)
    sim.set_particle_tile_ordering(True)
    sim.prepare_deterministic_p2g()
    sim.set_deterministic_p2g(True)
    assert sim.deterministic_p2g_enabled() and not sim.uses_two_pass_p2g()
    with pytest.raises(m.SolverError):
        sim.release_deterministic_p2g()
    prepared = sim.prepare_step(dt, 1)
    sim.set_p2g_mode(False)
    assert not sim.deterministic_p2g_enabled() and not sim.uses_two_pass_p2g()
    assert sim.particle_tile_ordering_enabled()
    batch = sim.begin_command_batch()
    with pytest.raises(m.StaleError):
        batch.encode_step(prepared)
    sim.release_deterministic_p2g()
    with pytest.raises(m.SolverError):
        sim.set_deterministic_p2g(True)  # released: needs a new prepare call
    sim.set_p2g_mode(True)
    assert sim.uses_two_pass_p2g()
    sim.set_rheology(m.MpmRheology.Snow())
    got = sim.config()
    assert got.grid_size == 32 and got.max_particles == 4096 and got.rheology.kind == m.MpmRheology.Snow().kind


def test_momentum_drift_closed_system(engine):
    """mpm_gpu.rs:780-837."""
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    cfg.grid_origin = (-1.6, -1.6, -1.6)
    cfg.grid_size = 32
    cfg.cell_size = 0.1
    cfg.boundary_friction = 1.0
    pts = scenes.fill_box_lcg([-0.4] * 3, [0.4] * 3, 8, 7)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(pts)
    for _ in range(60):
        sim.step(1.0 / 240)
    vel = sim.read_velocities()
    p = np.linalg.norm(vel.sum(0)) * cfg.particle_mass
    assert p < 0.01 * cfg.particle_mass * len(pts)


def test_sand_block_smoke(engine):
    """mpm_gpu.rs:201-241."""
    cfg = m.MpmConfig.sand()
    pts = scenes.fill_box_lcg([-0.2, 0.6, -0.2], [0.2, 1.0, 0.2], 8, 42)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(pts)
    for _ in range(60):
        sim.step(1.0 / 240)
    pos, vel = sim.read_positions(), sim.read_velocities()
    assert np.isfinite(pos).all() and np.isfinite(vel).all()
    assert pos[:, 1].min() < 0.95 and np.linalg.norm(vel, axis=1).max() < 50


@pytest.mark.parametrize("preset", ["sand", "snow", "viscous"])
def test_dropped_block_settles(engine, preset):
    """mpm_freefall_regression_gpu.rs:113-130 (snow), extended to each rheology."""
    cfg = getattr(m.MpmConfig, preset)()
    pts = scenes.fill_box_lcg([-0.075, 0.12, -0.075], [0.075, 0.27, 0.075], 6, 22)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(pts)
    sim.step_n(1.0 / 480, 300)
    pos = sim.read_positions()
    assert pos[:, 1].max() < 0.35 and np.abs(pos[:, 0]).max() < 0.25
    assert not sim.read_active_grid_status().numerical_fault


# ---- step parity against the oracle ------------------------------------------------

@pytest.mark.parametrize("preset", ["sand", "snow", "viscous"])
def test_one_substep_parity(engine, preset):
    cfg = getattr(m.MpmConfig, preset)()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 8, 42)
    rng = np.random.default_rng(1)
    vel = rng.uniform(-0.5, 0.5, size=pts.shape).astype(np.float32)
    _, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 240, 1, vel=vel)
    assert np.abs(gpu["pos"] - st["pos"]).max() < 1e-6
    assert np.abs(gpu["vel"] - st["vel"]).max() < 1e-5
    assert norm_err(gpu["C"], st["C"]) < 2e-5 * 10
    assert norm_err(gpu["F"], st["F"]) < 2e-5
    assert norm_err(gpu["jp"], st["jp"]) < 2e-5


@pytest.mark.parametrize("preset", ["sand", "snow", "viscous"])
def test_many_substeps_parity(engine, preset):
    cfg = getattr(m.MpmConfig, preset)()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 8, 42)
    _, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 480, 120)
    assert np.abs(gpu["pos"] - st["pos"]).max() < 1e-4
    assert np.abs(gpu["vel"] - st["vel"]).max() < 1e-2
    assert gpu["status"].completed_substeps == 120 and not gpu["status"].numerical_fault


def ordering_config(size=35):
    # mpm_particle_order_tests.rs:7-18
    cfg = m.MpmConfig.sand()
    cfg.grid_size = size
    cfg.grid_origin = (-1.0, -1.0, -1.0)
    cfg.cell_size = 0.0625
    cfg.max_particles = 513
    cfg.youngs = 3000.0
    cfg.particle_volume = float(np.float32(0.021) ** 3)
    cfg.particle_mass = float(np.float32(cfg.particle_volume) * np.float32(1600.0))
    return cfg


MIXED_ROWS = [m.MpmRheology.Sand(0.5), m.MpmRheology.Snow(0.025, 0.0075, 10.0), m.MpmRheology.Viscous(0.1, 0.2)]


@pytest.mark.parametrize("count", [257, 63])
def test_mixed_materials_parity(engine, count):
    """ordered_transfer_preserves_material_state (mpm_particle_order_tests.rs:167-285):
    three rheologies, initial velocity, 6 substeps in windows of 2, the
    reference's `close` tolerance (2e-5)."""
    cfg = ordering_config()
    pts = G.points(count)
    ids = (np.arange(count) % 3).astype(np.uint32)
    vel = np.tile(np.array([0.1, -0.02, 0.03], np.float32), (count, 1))
    _, gpu, st = run_both(engine, cfg, MIXED_ROWS, pts, ids, 1e-4, 6, vel=vel, chunked=[2, 2, 2])
    assert np.abs(gpu["pos"] - st["pos"]).max() <= 2e-5
    assert np.abs(gpu["vel"] - st["vel"]).max() <= 2e-5
    assert norm_err(gpu["C"], st["C"]) <= 2e-5
    assert norm_err(gpu["F"], st["F"]) <= 2e-5
    assert norm_err(gpu["jp"], st["jp"]) <= 2e-5


@pytest.mark.parametrize("interval", [1, 4, 64])
def test_regroup_interval_does_not_change_results(engine, interval):
    cfg = m.MpmConfig.snow()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 10, 3)
    _, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 480, 40, sort_interval=interval)
    assert np.abs(gpu["pos"] - st["pos"]).max() < 2e-5


def test_fp64_svd_mode_parity(engine):
    cfg = m.MpmConfig.snow()
    cfg.svd_precision = 1
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 8, 42)
    _, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 480, 60, precision="f32_svd64")
    assert np.abs(gpu["pos"] - st["pos"]).max() < 1e-4


def test_cube_positions_vs_fp64_oracle(engine):
    """Accuracy gate on a reduced cube scene: positions within 1e-4 relative
    of the FP64 oracle after 1000 substeps."""
    sc_ = scenes.cube_scene(grid_size=16, per_axis=12, seed=0, dt=1e-4)
    cfg = m.config_for_scene(sc_, svd_precision=1)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(sc_.positions)
    sim.set_materials(sc_.rows, sc_.ids)
    sim.step_n(sc_.dt, 1000)
    pos = sim.read_positions().astype(np.float64)
    osc = O.make_scene(cfg, sc_.rows, sc_.dt, svd_tol=1e-14, svd_sweeps=30)
    st = O.cast_state(O.init_state(sc_.positions, mass=cfg.particle_mass, volume=cfg.particle_volume, ids=sc_.ids),
                      np.float64)
    O.step(osc, st, 1000, precision="f64")
    rel = np.abs(pos - st["pos"]) / np.abs(st["pos"])
    assert rel.max() < 1e-4, rel.max()


@pytest.mark.parametrize("preset", ["snow", "sand"])
def test_all_fp64_gpu_matches_fp64_oracle(engine, preset):
    """The all-FP64 GPU mode (precision studies) against the FP64 oracle:
    both run the reference substep in FP64 with the FP64 Jacobi SVD (tol
    1e-14, 30 sweeps); only the order of the grid atomics and FMA
    contraction differ."""
    cfg = getattr(m.MpmConfig, preset)()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 8, 7).astype(np.float64)
    sim = m.MpmSimulation64(engine, cfg)
    sim.set_particles(pts)
    rows = [cfg.rheology]
    sim.set_materials(rows, np.zeros(len(pts), np.uint32))
    dt = float(np.float32(1.0 / 480))  # the oracle's scene holds dt in FP32
    sim.step_n(dt, 40)
    pos, vel, F = sim.read_state()
    assert not sim.read_active_grid_status().numerical_fault
    sc = O.make_scene(cfg, rows, dt, svd_tol=1e-14, svd_sweeps=30)
    st = O.cast_state(O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume), np.float64)
    O.step(sc, st, 40, precision="f64")
    assert np.abs(pos - st["pos"]).max() < 1e-9
    assert np.abs(vel - st["vel"]).max() < 1e-7
    assert np.abs(F - st["F"]).max() < 1e-8
    mass, mom = sim.grid_totals()
    assert abs(mass - cfg.particle_mass * len(pts)) / (cfg.particle_mass * len(pts)) < 1e-12


def test_semi_implicit_preset_matches_oracle(engine):
    """MpmConfig::sand_calibrated (Implicit { jacobi_iters: 3 }) against the
    oracle's semi-implicit sweeps (mpm.wgsl:1060-1173); and switching an
    existing simulation to an even sweep count through set_time_step."""
    cfg = m.MpmConfig.sand_calibrated()
    assert cfg.time_step == 1 and cfg.jacobi_iters == 3
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 10, 9)
    _, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 480, 30)
    assert np.abs(gpu["pos"] - st["pos"]).max() < 2e-5
    assert np.abs(gpu["vel"] - st["vel"]).max() < 2e-3
    sim = m.MpmSimulation.new(engine, m.MpmConfig.sand())
    sim.set_particles(pts)
    sim.set_time_step(1, 2)
    sim.step_n(1.0 / 480, 30)
    c2 = m.MpmConfig.sand()
    c2.time_step, c2.jacobi_iters = 1, 2
    sc = O.make_scene(c2, [c2.rheology], 1.0 / 480)
    st2 = O.init_state(pts, mass=c2.particle_mass, volume=c2.particle_volume)
    O.step(sc, st2, 30)
    assert np.abs(sim.read_positions() - st2["pos"]).max() < 2e-5


def test_rigid_spheres_match_oracle(engine):
    """set_rigid_spheres / read_rigid_wrenches (mpm.rs:1521-1565, 2809) with
    the imprint and shell reaction (mpm.wgsl:939-1003, 1175-1228) against the
    oracle: positions and the last substep's wrench."""
    cfg = m.MpmConfig.sand()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.5, 0.2], 10, 2)
    spheres = [((0.0, 0.55, 0.0), 0.12, (0.0, -1.0, 0.0)), ((0.12, 0.42, 0.1), 0.06, (0.3, 0.0, -0.2))]
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_rigid_spheres(spheres)
    sim.set_particles(pts)  # the spheres are kept across set_particles
    sim.step_n(1.0 / 480, 10)
    got = sim.read_rigid_wrenches()
    sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 480)
    O.set_rigid_spheres(sc, spheres)
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    O.step(sc, st, 10)
    ref = O.rigid_wrenches(sc)
    assert np.abs(sim.read_positions() - st["pos"]).max() < 2e-5
    assert len(got) == 2
    for (gf, gt), (rf, rt) in zip(got, ref):
        scale = max(np.abs(rf).max(), 1e-6)
        assert np.abs(gf - rf).max() < 2e-3 * scale
        assert np.abs(gt - rt).max() < 2e-3 * scale
    with pytest.raises(m.MollaError):
        sim.set_rigid_spheres([((0, 0, 0), 0.1, (0, 0, 0))] * (cfg.max_rigid + 1))


def test_soil_checkpoint_round_trip_and_continuation(engine):
    """archive_drop_reload_preserves_all_history (mpm_checkpoint_tests.rs:176-257):
    a checkpoint of an evolved state restores bit for bit into a fresh
    simulation, re-encodes identically, and both continue alike."""
    cfg = m.MpmConfig.sand()
    cfg.max_particles = 4096
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 10, 5)
    rows = [m.MpmRheology.Sand(0.5), m.MpmRheology.Snow(), m.MpmRheology.Viscous(3.0, 5.0)]
    ids = (np.arange(len(pts)) % 3).astype(np.uint32)
    a = m.MpmSimulation.new(engine, cfg)
    a.set_particles(pts)
    a.set_materials(rows, ids)
    a.step_n(1.0 / 480, 20)
    data = a.checkpoint_soil()
    assert len(data) == 44 + 4 * (21 + 1 + 12 + 1) + 160 * len(pts)
    assert m.checkpoint_reencode(data, cfg.max_particles) == (data, len(pts))
    b = m.MpmSimulation.new(engine, cfg)
    b.restore_soil(data)
    for f in ("read_positions", "read_velocities"):
        assert np.array_equal(getattr(a, f)(), getattr(b, f)())
    sa, sb = a.read_particle_state(), b.read_particle_state()
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    assert b.checkpoint_soil() == data
    a.step_n(1.0 / 480, 10)
    b.step_n(1.0 / 480, 10)
    assert np.abs(a.read_positions() - b.read_positions()).max() < 1e-5


def test_soil_checkpoint_rejects_incompatible_or_faulted_state(engine):
    cfg = m.MpmConfig.sand()
    cfg.max_particles = 256
    pts = scenes.fill_box_lcg([-0.1, 0.3, -0.1], [0.1, 0.5, 0.1], 4, 1)
    a = m.MpmSimulation.new(engine, cfg)
    a.set_particles(pts)
    a.step_n(1.0 / 480, 2)
    data = a.checkpoint_soil()
    other = m.MpmConfig.sand()
    other.max_particles = 256
    other.youngs = cfg.youngs * 2
    b = m.MpmSimulation.new(engine, other)
    with pytest.raises(m.MollaError):
        b.restore_soil(data)
    small = m.MpmConfig.sand()
    small.max_particles = len(pts) - 1
    c = m.MpmSimulation.new(engine, small)
    with pytest.raises(m.MollaError):
        c.restore_soil(data)
    # a latched numerical fault cannot be archived
    pos = a.read_positions()
    pos[0, 0] = np.nan
    a.set_particles(pos)
    a.step_n(1.0 / 480, 1)
    assert a.read_active_grid_status().numerical_fault
    with pytest.raises(m.MollaError):
        a.checkpoint_soil()


# ---- fault latch (mpm_numerical_fault_tests.rs:19-100) -----------------------------

def test_bounded_device_wait_reports_and_keeps_the_engine(engine):
    """The scatter's stage wait, run on a barrier that nothing completes,
    gives up after about a second, latches the device-wait bit (8) and
    leaves the context usable: a simulation still steps afterwards."""
    bits, waited_ms = engine.selftest_device_wait()
    assert bits == 8
    assert 900.0 <= waited_ms <= 5000.0
    cfg = m.MpmConfig.snow()
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles([[0.013, 0.2, 0.017]])
    sim.step_n(1.0 / 480, 4)
    st = sim.read_active_grid_status()
    assert st.completed_substeps == 4 and not st.numerical_fault


@pytest.mark.parametrize("bits", [np.nan, np.inf, -np.inf])
def test_fault_latches_without_repair(engine, bits):
    cfg = m.MpmConfig.sand()
    cfg.max_particles = 4
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles([[0.0, 0.3, 0.0], [0.1, 0.3, 0.0]])
    sim.step_n(1e-4, 1)
    C0, F0, jp0 = sim.read_particle_state()
    F = F0.copy()
    F[0, 4] = bits
    sim.write_particle_state(F=F)
    sim.step_n(1e-4, 1)
    s = sim.read_active_grid_status()
    assert s.numerical_fault and s.faulted()
    before = (sim.read_positions(), sim.read_velocities(), *sim.read_particle_state())
    sim.step_n(1e-4, 3)
    after = (sim.read_positions(), sim.read_velocities(), *sim.read_particle_state())
    for a, b in zip(before, after):
        assert np.array_equal(a, b, equal_nan=True)
    assert sim.read_active_grid_status().numerical_fault
    # restore + reset recovers
    sim.write_particle_state(C_=C0, F=F0, jp=jp0)
    sim.reset_active_grid()
    sim.step_n(1e-4, 1)
    assert not sim.read_active_grid_status().faulted()


# ---- prepared steps / command batches (mpm_command_batch.rs) ---------------------

def test_prepared_batch_matches_step_n_and_goes_stale(engine):
    cfg = m.MpmConfig.snow()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.7, 0.2], 8, 5)
    a = m.MpmSimulation.new(engine, cfg)
    b = m.MpmSimulation.new(engine, cfg)
    a.set_particles(pts)
    b.set_particles(pts)
    a.set_sort_interval(8)
    b.set_sort_interval(8)
    rec = b.prepare_step(1.0 / 480, 10)
    for _ in range(3):
        a.step_n(1.0 / 480, 10)
        batch = b.begin_command_batch()
        batch.encode_step(rec)
        batch.submit()
    pa, pb = a.read_positions(), b.read_positions()
    assert np.abs(pa - pb).max() < 1e-5
    assert b.read_active_grid_status().completed_substeps == 30
    # a dropped batch does nothing
    batch = b.begin_command_batch()
    batch.encode_step(rec)
    del batch
    assert np.array_equal(pb, b.read_positions())
    # another simulation's record / a stale record is rejected
    batch = a.begin_command_batch()
    with pytest.raises(m.StaleError):
        batch.encode_step(rec)
    b.set_rheology(m.MpmRheology.Snow())
    batch = b.begin_command_batch()
    with pytest.raises(m.StaleError):
        batch.encode_step(rec)


# ---- multi-material equivalence (mpm_multimaterial_gpu.rs:129-191) ---------------

def test_disjoint_blocks_mixed_equal_separate_runs(engine):
    cfg = m.MpmConfig.sand()
    cfg.max_particles = 4096
    a = scenes.fill_box_lcg([-0.5, 0.2, -0.1], [-0.3, 0.4, 0.1], 6, 1)
    b = scenes.fill_box_lcg([0.3, 0.2, -0.1], [0.5, 0.4, 0.1], 6, 2)
    rows = [m.MpmRheology.Sand(math.radians(30)), m.MpmRheology.Snow()]
    mixed = m.MpmSimulation.new(engine, cfg)
    mixed.set_particles(np.concatenate([a, b]))
    mixed.set_materials(rows, np.r_[np.zeros(len(a)), np.ones(len(b))].astype(np.uint32))
    mixed.step_n(1.0 / 480, 60)
    pm = mixed.read_positions()
    outs = []
    for pts, rid in ((a, 0), (b, 1)):
        s = m.MpmSimulation.new(engine, cfg)
        s.set_particles(pts)
        s.set_materials(rows, np.full(len(pts), rid, np.uint32))
        s.step_n(1.0 / 480, 60)
        outs.append(s.read_positions())
    assert np.abs(pm - np.concatenate(outs)).max() < 1e-5


def test_deterministic_p2g_lifecycle_and_repeatability(engine):
    """mpm_fixed_order_runtime.rs:65-159: preconditions, then two simulations
    stepped identically are byte-equal; results match the oracle."""
    cfg = ordering_config()
    pts = G.points(257)
    ids = (np.arange(257) % 3).astype(np.uint32)
    vel = np.tile(np.array([0.1, -0.02, 0.03], np.float32), (257, 1))
    sims = []
    for _ in range(2):
        sim = m.MpmSimulation.new(engine, cfg)
        sim.set_particles(pts, vel)
        sim.set_materials(MIXED_ROWS, ids)
        with pytest.raises(m.SolverError):
            sim.set_deterministic_p2g(True)  # not prepared, no ordering
        sim.prepare_deterministic_p2g()
        with pytest.raises(m.SolverError):
            sim.set_deterministic_p2g(True)  # ordering not enabled
        sim.prepare_particle_tile_ordering(257)
        sim.set_particle_tile_ordering(True)
        sim.set_deterministic_p2g(True)
        with pytest.raises(m.SolverError):
            sim.set_particle_tile_ordering(False)
        for _ in range(3):
            sim.step_n(1e-4, 2)
        sims.append(sim)
    a = [sims[0].read_positions(), sims[0].read_velocities(), *sims[0].read_particle_state()]
    b = [sims[1].read_positions(), sims[1].read_velocities(), *sims[1].read_particle_state()]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert sims[0].read_active_grid_status().fault_bits == 0
    sc = O.make_scene(cfg, MIXED_ROWS, 1e-4)
    st = O.init_state(pts, vel, mass=cfg.particle_mass, volume=cfg.particle_volume, ids=ids)
    O.step(sc, st, 6)
    assert np.abs(a[0] - st["pos"]).max() <= 2e-5
    assert norm_err(a[3], st["F"]) <= 2e-5


def test_simulation_outlives_its_engine_handle():
    """Destroying the engine handle first is allowed: the simulation keeps the
    device stream until it is destroyed itself (the order the interpreter
    may pick at exit)."""
    e = m.Engine(0)
    cfg = m.MpmConfig.sand()
    sim = m.MpmSimulation.new(e, cfg)
    sim.set_particles([[0.0, 0.3, 0.0], [0.05, 0.3, 0.0]])
    e.close()
    sim.step_n(1e-4, 3)
    assert sim.read_active_grid_status().completed_substeps == 3
    sim.close()


@pytest.mark.parametrize("preset,window", [("sand", (3, -2, 1)), ("snow", (-5, 4, 0))])
def test_grid_window_parity(engine, preset, window):
    """A shifted lattice (grid_window_cells, mpm.wgsl:513-516: base cell minus
    the window, node position o + (index + window) dx): the block sits in the
    shifted domain, falls against its floor, and matches the oracle; the tile
    keys of the sort subtract the window too."""
    cfg = getattr(m.MpmConfig, preset)()
    cfg.grid_window_cells = window
    dx, n = cfg.cell_size, cfg.grid_size
    lo = [cfg.grid_origin[a] + (window[a] + 0.35 * n) * dx for a in range(3)]
    hi = [cfg.grid_origin[a] + (window[a] + 0.65 * n) * dx for a in range(3)]
    lo[1] = cfg.grid_origin[1] + (window[1] + 6) * dx  # near the shifted floor
    hi[1] = lo[1] + 0.25 * n * dx
    pts = scenes.fill_box_lcg(lo, hi, 8, 7)
    sim, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 480, 60)
    assert gpu["status"].completed_substeps == 60 and not gpu["status"].numerical_fault
    assert np.abs(gpu["pos"] - st["pos"]).max() < 1e-4
    assert np.abs(gpu["vel"] - st["vel"]).max() < 1e-2
    # the block fell (gravity) and stayed inside the shifted walls
    assert gpu["pos"][:, 1].mean() < pts[:, 1].mean()
    floor = cfg.grid_origin[1] + (window[1] + 2) * dx
    assert gpu["pos"][:, 1].min() >= floor - 1e-6
    keys, ids = sim.read_sort_permutation()
    ok, oi = O.particle_order(O.make_scene(cfg, [cfg.rheology], 1.0 / 480), gpu["pos"], len(pts), len(pts))
    assert np.array_equal(keys, ok) and np.array_equal(ids, oi)


@pytest.mark.parametrize("pad,walls", [(3, 0), (4, 1)])
def test_wall_extensions_parity(engine, pad, walls):
    """boundary_pad (the reference's fixed 2 made a parameter) and the sticky
    no-slip walls extension: a block thrown at the -x wall and dropped onto
    the floor matches the oracle, and no particle crosses the pad layer."""
    cfg = m.MpmConfig.sand()
    cfg.boundary_pad = pad
    cfg.walls = walls
    dx, o = cfg.cell_size, cfg.grid_origin
    lo = [o[0] + (pad + 2) * dx, o[1] + (pad + 3) * dx, o[2] + 0.4 * cfg.grid_size * dx]
    hi = [lo[0] + 8 * dx, lo[1] + 8 * dx, lo[2] + 8 * dx]
    pts = scenes.fill_box_lcg(lo, hi, 8, 3)
    vel = np.tile(np.array([[-2.0, 0.0, 0.0]], np.float32), (len(pts), 1))
    _, gpu, st = run_both(engine, cfg, None, pts, None, 1.0 / 960, 80, vel=vel)
    assert gpu["status"].completed_substeps == 80 and not gpu["status"].numerical_fault
    assert np.abs(gpu["pos"] - st["pos"]).max() < 1e-4
    assert np.abs(gpu["vel"] - st["vel"]).max() < 1e-2
    for a in (0, 1):
        assert gpu["pos"][:, a].min() >= o[a] + pad * dx - 1e-6


def test_stage_profile_counts_launches(engine):
    """MpmProfileStage timing (mpm_profile.rs:8-80): per-stage launch counts
    and device times of a profiled step_n, nothing while disabled, zero after
    a reset."""
    cfg = m.MpmConfig.snow()
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(scenes.fill_box_lcg([-0.1, 0.2, -0.1], [0.1, 0.4, 0.1], 8, 5))
    sim.set_sort_interval(4)
    sim.step_n(1.0 / 480, 2)
    engine.synchronize()
    engine.reset_profile()
    engine.profile(True)
    sim.step_n(1.0 / 480, 10)
    engine.synchronize()
    engine.profile(False)
    prof = engine.read_profile()
    assert set(prof) == set(m.Engine.STAGES)
    # no record-only gather: the previous call's last gather left the records
    # and no regrouping opens this call
    assert prof["GridUpdate"][0] == 10 and prof["StressRecord"][0] == 0
    # gathers: every substep; scatters: once per call when fused, else every substep but the last
    assert prof["GridToParticle"][0] == 10
    assert prof["ParticleToGrid"][0] in (1, 10)
    assert prof["ParticleOrdering"][0] >= 2  # one every 4 substeps of the cadence
    assert all(ms > 0.0 for cnt, ms in prof.values() if cnt)
    sim.step_n(1.0 / 480, 3)
    engine.synchronize()
    assert engine.read_profile() == prof  # disabled: nothing added
    engine.reset_profile()
    assert all(v == (0, 0.0) for v in engine.read_profile().values())
    sim.close()
