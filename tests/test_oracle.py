"""CPU tests of the oracle against the reference's known-answer tests.

These pin the CPU restatement (oracle/) before it is trusted as the checker
of the CUDA path.  Each test names the reference test it reproduces.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import make_golden as G

import molla_b200 as m
from molla_b200 import scenes

GOLD = G.HERE


# ---- material oracles: crates/molla-solvers/tests/mpm_material_oracles.rs ----

def sand(s, jp, E, nu, phi):
    out_s = np.empty(3)
    out_jp = np.empty(1)
    O.lib().orc_sand_project_f64(np.asarray(s, np.float64), jp, E, nu, phi, out_s, out_jp)
    return out_s, out_jp[0]


def snow(s, jp, tc, ts):
    out_s = np.empty(3)
    out_jp = np.empty(1)
    O.lib().orc_snow_clamp_f64(np.asarray(s, np.float64), jp, tc, ts, out_s, out_jp)
    return out_s, out_jp[0]


def test_dp_alpha_matches_shader_formula():  # :19-28
    L = O.lib()
    phi = math.radians(30.0)
    exp = math.sqrt(2 / 3) * (2 * math.sin(phi)) / (3 - math.sin(phi))
    assert abs(L.orc_dp_alpha_f64(phi) - exp) < 1e-15
    assert L.orc_dp_alpha_f64(math.radians(-10.0)) == L.orc_dp_alpha_f64(math.radians(1.0))


def test_sand_resets_tensile_volume_expansion():  # :30-39
    s, jp = sand([1.2, 1.1, 1.0], 0.0, 1e5, 0.3, 0.5)
    assert np.array_equal(s, [1.0, 1.0, 1.0])
    assert jp > 0


def test_sand_keeps_elastic_state_inside_cone():  # :41-48
    s, jp = sand([0.95] * 3, 0.2, 1e5, 0.3, math.radians(30))
    assert np.array_equal(s, [0.95] * 3) and jp == 0.2


def test_sand_projects_shear_outside_cone():  # :50-64
    s0 = np.array([0.5, 0.9, 1.1])
    s, jp = sand(s0, 0.0, 1e5, 0.3, math.radians(5))
    assert np.linalg.norm(s - s0) > 1e-3 and jp > 0 and s[0] > s0[0]


def test_sand_friction_angle_monotone():  # :66-111
    s0 = np.array([0.42, 0.82, 1.05])
    lo, jlo = sand(s0, 0.0, 1e5, 0.3, math.radians(5))
    hi, jhi = sand(s0, 0.0, 1e5, 0.3, math.radians(35))
    dev = lambda s: np.linalg.norm(s - s.mean())
    assert dev(hi) > dev(lo) and dev(hi) <= dev(s0) + 1e-12
    assert np.linalg.norm(hi - s0) < np.linalg.norm(lo - s0) and jhi < jlo


def test_sand_bounds_plastic_flow():  # :113-117
    assert sand([20.0] * 3, 4.9, 1e5, 0.3, 0.5)[1] == 5.0


def test_snow_clamps_to_envelope():  # :242-252
    s, jp = snow([0.8, 1.2, 1.0], 0.0, 0.025, 0.0075)
    assert abs(s[0] - 0.975) < 1e-15 and abs(s[1] - 1.0075) < 1e-15 and s[2] == 1.0 and np.isfinite(jp)


def test_snow_tracks_log_plastic_volume():  # :254-267
    s0 = np.array([0.5, 1.5, 1.1])
    s, jp = snow(s0, 0.25, 0.025, 0.0075)
    exp = 0.25 + math.log(max(s0.prod(), 1e-6)) - math.log(max(s.prod(), 1e-6))
    assert abs(jp - min(max(exp, -5), 5)) < 1e-15


def test_snow_repeated_compression_bounded():  # :269-307
    jp, prev = 0.0, 0.0
    for _ in range(12):
        s, jp = snow([0.82, 0.94, 1.06], jp, 0.025, 0.0075)
        assert np.all((s >= 0.975) & (s <= 1.0075)) and jp <= prev and -5 <= jp <= 5
        prev = jp
    assert jp < -0.5


def test_snow_bounds_hardening():  # :309-316
    assert snow([20.0] * 3, 4.9, 0.025, 0.0075)[1] == 5.0
    assert snow([1e-3] * 3, -4.9, 0.025, 0.0075)[1] == -5.0


def test_viscous_damping_factors():  # :119-150
    v = np.array([0.4, -0.2, 0.1])
    Cm = np.arange(9, dtype=np.float64) / 10
    ov, oc, f = np.empty(3), np.empty(9), np.empty(2)
    O.lib().orc_viscous_damping_f64(v, Cm, 0.01, 4.0, 8.0, ov, oc, f)
    assert abs(f[0] - math.exp(-0.04)) < 1e-15 and abs(f[1] - math.exp(-0.08)) < 1e-15
    assert np.abs(ov - v * f[0]).max() < 1e-15 and np.abs(oc - Cm * f[1]).max() < 1e-15
    O.lib().orc_viscous_damping_f64(v, Cm, -1.0, -4.0, -8.0, ov, oc, f)
    assert f[0] == 1.0 and f[1] == 1.0 and np.array_equal(ov, v)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_step_plasticity_matches_material_twins(kind):
    """The step's own plasticity body (mpm.wgsl:1366-1479) agrees with the f64
    twins (mpm_oracle.rs) on diagonal deformation gradients."""
    cfg = {"grid_size": 8, "cell_size": 0.1, "youngs": 1e5, "poisson": 0.3}
    row = [{"kind": 0, "friction_angle": math.radians(5)},
           {"kind": 1, "theta_c": 0.025, "theta_s": 0.0075, "hardening": 10.0},
           {"kind": 2, "velocity_damping": 1.0, "affine_damping": 1.0}][kind]
    sc = O.make_scene(cfg, [row], 1e-4)
    for s0 in ([0.5, 0.9, 1.1], [0.95, 0.96, 0.97], [1.2, 1.1, 1.0], [0.82, 0.94, 1.06]):
        F = np.zeros(9)
        F[0], F[4], F[8] = s0
        jp = np.array([0.1])
        assert O.lib().orc_plasticity_f64(C_byref(sc), F, jp, 0) == 1
        got = np.sort(np.array([F[0], F[4], F[8]]))
        if kind == 0:
            alpha = float(sc.materials[0].dp_alpha)
            # the step uses the row's f32 alpha; the twin recomputes it from phi
            exp, ejp = sand_with_alpha(s0, 0.1, 1e5, 0.3, alpha)
        elif kind == 1:
            exp, ejp = snow(s0, 0.1, 0.025, 0.0075)
        else:
            exp, ejp = np.array(s0), 0.0
        exp = np.clip(np.sort(exp), 0.05, 20)
        assert np.abs(got - exp).max() < 1e-6, (kind, s0, got, exp)
        assert abs(jp[0] - ejp) < 1e-6


def C_byref(sc):
    import ctypes
    return ctypes.byref(sc)


def sand_with_alpha(s, jp, E, nu, alpha):
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    eps = np.log(np.maximum(s, 1e-6))
    tr = eps.sum()
    dev = eps - tr / 3
    dn = np.linalg.norm(dev)
    kappa = (3 * lam + 2 * mu) / (2 * mu)
    if tr > 0:
        return np.ones(3), min(max(jp + np.linalg.norm(eps), 0), 5)
    if dn == 0:
        return np.array(s), jp
    fy = dn + kappa * tr * alpha
    if fy <= 0:
        return np.array(s), jp
    rc = max(0.0, -alpha * kappa * tr)
    return np.exp(dev * (rc / dn) + tr / 3), min(max(jp + fy, 0), 5)


# ---- SVD (mpm.wgsl:365-468) ----

@pytest.mark.parametrize("prec,tol", [("f32", 2e-5), ("f64", 1e-12)])
def test_svd_reconstructs_and_is_proper(prec, tol):
    rng = np.random.default_rng(5)
    for _ in range(200):
        A = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if rng.uniform() < 0.2:
            A[:, 0] *= -1  # det < 0
        F = A.T.reshape(9)  # column-major
        U, s, V = O.svd3(F, prec, tol=1e-7 if prec == "f32" else 1e-14, sweeps=16)
        Um = U.reshape(3, 3).T
        Vm = V.reshape(3, 3).T
        R = Um @ np.diag(s) @ Vm.T
        assert np.abs(R - A).max() < tol * 10
        assert np.linalg.det(Um) > 0 and np.linalg.det(Vm) > 0


# ---- gather exactness: crates/molla-solvers/src/mpm_gather_oracle.rs:53-90 ----

def test_gather_reproduces_affine_fields():
    import ctypes
    cfg = {"grid_size": 8, "cell_size": 0.125, "grid_origin": (-0.5, -0.5, -0.5)}
    sc = O.make_scene(cfg, [{"kind": 0}], 1e-4)
    pos = np.array([-0.03125, 0.09375, 0.0])
    tr = np.array([0.2, -0.3, 0.1])
    for grad in (np.zeros((3, 3)), np.array([[1, 0.5, 0], [0, 1, -0.25], [0.25, 0, 1]], float)):
        grid = np.zeros((512, 4))
        for i in range(512):
            node = np.array([-0.5, -0.5, -0.5]) + 0.125 * np.array([i % 8, i // 8 % 8, i // 64])
            grid[i, :3] = tr + grad @ node
        v = np.empty(3)
        Cm = np.empty(9)
        O.lib().orc_gather_f64(ctypes.byref(sc), pos, np.ascontiguousarray(grid.reshape(-1)), v, Cm)
        assert np.abs(v - tr - grad @ pos).max() < 1e-14
        assert np.abs(Cm.reshape(3, 3).T - grad).max() < 1e-14


# ---- free fall: crates/molla-solvers/tests/mpm_freefall_regression_gpu.rs:76-111 ----

def test_single_particle_free_fall_is_exact():
    cfg = m.MpmConfig.snow()
    dt = 1.0 / 480.0
    sc = O.make_scene(cfg, [cfg.rheology], dt)
    st = O.init_state([[0.013, 0.2, 0.017]], mass=cfg.particle_mass, volume=cfg.particle_volume)
    for step in range(20):
        O.step(sc, st, 1)
        vy = -9.81 * dt * (step + 1)
        assert abs(st["vel"][0, 1] - vy) < 1e-4
        assert abs(st["vel"][0, 0]) < 1e-5 and abs(st["vel"][0, 2]) < 1e-5
        assert abs(st["pos"][0, 0] - 0.013) < 1e-5 and abs(st["pos"][0, 2] - 0.017) < 1e-5


# ---- grid mass: crates/molla-solvers/tests/mpm_gpu.rs:839-884 ----

def test_grid_mass_matches_particle_mass():
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    cfg.grid_origin = (-1.6, -1.6, -1.6)
    cfg.grid_size = 32
    cfg.cell_size = 0.1
    cfg.particle_mass = 2.5e-3
    cfg.boundary_friction = 1.0
    pts = scenes.fill_box_lcg([-0.35] * 3, [0.35] * 3, 7, 19)
    sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 240)
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    gm, gp = O.step(sc, st, 1, want_grid=True)
    exp = cfg.particle_mass * len(pts)
    assert (gm > 0).sum() > 0
    assert abs(gm.sum(dtype=np.float64) - exp) / exp < 1e-4
    assert np.abs(gp).max() < 1e-6


# ---- closed-system momentum: crates/molla-solvers/tests/mpm_gpu.rs:780-837 ----

def test_momentum_drift_closed_system():
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    cfg.grid_origin = (-1.6, -1.6, -1.6)
    cfg.grid_size = 32
    cfg.cell_size = 0.1
    cfg.boundary_friction = 1.0
    pts = scenes.fill_box_lcg([-0.4] * 3, [0.4] * 3, 8, 7)
    sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 240)
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    O.step(sc, st, 60)
    p = np.linalg.norm(st["vel"].sum(0)) * cfg.particle_mass
    assert p < 0.01 * cfg.particle_mass * len(pts)


# ---- smoke: crates/molla-solvers/tests/mpm_gpu.rs:201-241 ----

def test_sand_block_falls_without_exploding():
    cfg = m.MpmConfig.sand()
    pts = scenes.fill_box_lcg([-0.2, 0.6, -0.2], [0.2, 1.0, 0.2], 8, 42)
    sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 240)
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    O.step(sc, st, 60)
    assert np.isfinite(st["pos"]).all() and np.isfinite(st["vel"]).all()
    assert st["pos"][:, 1].min() < 0.95
    assert np.linalg.norm(st["vel"], axis=1).max() < 50
    assert st["status"][0] == 0 and st["status"][1] == 60


# ---- particle order: crates/molla-solvers/src/mpm_particle_order_tests.rs:67-165 ----

@pytest.mark.parametrize("size", [35, 1536])
@pytest.mark.parametrize("count", [513, 257, 1, 0, 63])
def test_particle_order_matches_reference_golden(size, count):
    g = np.load(GOLD / f"particle_order_{size}_{count}.npz")
    cfg = {"grid_size": size, "cell_size": 0.0625, "grid_origin": (-1.0, -1.0, -1.0)}
    sc = O.make_scene(cfg, [{"kind": 0}], 1e-4)
    keys, ids = O.particle_order(sc, g["positions"], count, 513)
    assert np.array_equal(keys, g["keys"])
    assert np.array_equal(ids, g["ids"])


def test_golden_fixtures_are_current():
    for (size, count), (pos, keys, ids) in G.particle_order_cases().items():
        g = np.load(GOLD / f"particle_order_{size}_{count}.npz")
        assert np.array_equal(g["keys"], keys) and np.array_equal(g["ids"], ids)
        assert np.array_equal(g["positions"], pos)


@pytest.mark.parametrize("name", ["random_1k", "all_equal", "sorted", "reverse", "paired", "high_byte"])
def test_stable_sort_reference(name):
    g = np.load(GOLD / f"radix_{name}.npz")
    k, v = O.sort_pairs(g["keys"], g["values"])
    assert np.array_equal(k, g["sorted_keys"]) and np.array_equal(v, g["sorted_values"])


def test_fault_latches_and_freezes_state():
    """mpm_numerical_fault_tests.rs:19-100 (host-injected NaN)."""
    cfg = m.MpmConfig.sand()
    sc = O.make_scene(cfg, [cfg.rheology], 1e-4)
    st = O.init_state([[0.0, 0.3, 0.0]], mass=cfg.particle_mass, volume=cfg.particle_volume)
    O.step(sc, st, 1)
    st["F"][0, 4] = np.nan
    O.step(sc, st, 1)
    assert st["status"][0] & 2
    before = {k: v.copy() for k, v in st.items()}
    O.step(sc, st, 3)
    for k in ("pos", "vel", "C", "jp"):
        assert np.array_equal(before[k], st[k], equal_nan=True)


# ---- semi-implicit Jacobi relaxation (mpm.wgsl:1060-1173) ----

def test_implicit_sweeps_keep_a_uniform_velocity_field():
    """Every node of a block in uniform translation has the same velocity,
    so the neighbour mean equals it and the relaxation changes nothing."""
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    pts = scenes.fill_box_lcg([-0.15, 0.3, -0.15], [0.15, 0.6, 0.15], 8, 4)
    vel = np.tile(np.array([[0.3, -0.2, 0.1]], np.float32), (len(pts), 1))
    runs = []
    for kind, iters in ((0, 0), (1, 3)):
        cfg.time_step, cfg.jacobi_iters = kind, iters
        sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 480)
        st = O.cast_state(O.init_state(pts, vel, mass=cfg.particle_mass, volume=cfg.particle_volume), np.float64)
        O.step(sc, st, 1, precision="f64")
        runs.append(st)
    assert np.abs(runs[0]["vel"] - runs[1]["vel"]).max() < 1e-12
    assert np.abs(runs[0]["pos"] - runs[1]["pos"]).max() < 1e-14


def test_implicit_sweeps_relax_a_velocity_jump():
    """Two halves sliding past each other: the semi-implicit sweeps pull the
    grid velocities toward their neighbour means, so the particle velocity
    jump across the interface after one substep is smaller than explicit."""
    cfg = m.MpmConfig.sand_calibrated()
    cfg.gravity_y = 0.0
    pts = scenes.fill_box_lcg([-0.15, 0.3, -0.15], [0.15, 0.6, 0.15], 10, 6)
    vel = np.zeros_like(pts)
    vel[:, 0] = np.where(pts[:, 1] > 0.45, 1.0, -1.0)
    jumps = {}
    for kind, iters in ((0, 0), (1, 3)):
        cfg.time_step, cfg.jacobi_iters = kind, iters
        sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 480)
        st = O.init_state(pts, vel, mass=cfg.particle_mass, volume=cfg.particle_volume)
        O.step(sc, st, 1)
        v = st["vel"][:, 0]
        jumps[iters] = v[pts[:, 1] > 0.45].mean() - v[pts[:, 1] <= 0.45].mean()
    assert 0.0 < jumps[3] < jumps[0]


# ---- legacy rigid spheres (mpm.wgsl:939-1003, 1175-1228; mpm_oracle.rs:59-118) ----

def test_rigid_imprint_wrench_of_a_particle_at_rest():
    """rigid_cell_imprint_wrench: a sphere that covers the whole stencil of
    a particle at rest takes its mass at the sphere velocity, so the force
    on the sphere is -m v / dt and the particle leaves with v."""
    cfg = m.MpmConfig.sand()
    cfg.gravity_y = 0.0
    dt = 1.0 / 480
    sc = O.make_scene(cfg, [cfg.rheology], dt)
    x = np.array([[0.013, 0.2, 0.017]], np.float32)
    v = (0.4, -0.3, 0.2)
    O.set_rigid_spheres(sc, [((0.013, 0.2, 0.017), 0.35, v)])
    st = O.init_state(x, mass=cfg.particle_mass, volume=cfg.particle_volume)
    O.step(sc, st, 1)
    (force, torque), = O.rigid_wrenches(sc)
    exp = -np.array(v) * np.float32(cfg.particle_mass) / np.float32(dt)
    assert np.abs(force - exp).max() < 1e-4 * np.abs(exp).max()
    assert np.abs(st["vel"][0] - np.array(v)).max() < 1e-5
    # nodes symmetric about the particle within the sphere: torque small
    assert np.abs(torque).max() < 0.05 * np.abs(exp).max()


def test_rigid_sphere_pushes_sand_and_feels_it():
    cfg = m.MpmConfig.sand()
    pts = scenes.fill_box_lcg([-0.2, 0.3, -0.2], [0.2, 0.5, 0.2], 10, 2)
    sc = O.make_scene(cfg, [cfg.rheology], 1.0 / 480)
    O.set_rigid_spheres(sc, [((0.0, 0.55, 0.0), 0.12, (0.0, -1.0, 0.0))])
    st = O.init_state(pts, mass=cfg.particle_mass, volume=cfg.particle_volume)
    O.step(sc, st, 10)
    (force, _), = O.rigid_wrenches(sc)
    assert force[1] > 0.0  # sand resists the downward push
    near = np.linalg.norm(st["pos"] - np.array([0.0, 0.55, 0.0]), axis=1) < 0.14
    assert near.any() and st["vel"][near, 1].mean() < -0.1
