"""ctypes wrapper of the CPU oracle (oracle/mpm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module as the checker.  The product library never
imports it.

State arrays use the product's host conventions: positions/velocities (n, 3),
C/F (n, 9) column-major per particle, jp/mass/volume (n,), material ids (n,).
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libmpm_oracle.so"


class orc_material(C.Structure):
    _fields_ = [
        ("rheology", C.c_uint32),
        ("dp_alpha", C.c_float),
        ("theta_c", C.c_float),
        ("theta_s", C.c_float),
        ("hardening", C.c_float),
        ("velocity_damping", C.c_float),
        ("affine_damping", C.c_float),
        ("youngs", C.c_float),
        ("poisson", C.c_float),
    ]


class orc_scene(C.Structure):
    _fields_ = [
        ("grid_size", C.c_uint32),
        ("cell_size", C.c_float),
        ("inv_cell_size", C.c_float),
        ("origin", C.c_float * 3),
        ("window", C.c_int32 * 3),
        ("dt", C.c_float),
        ("gravity_y", C.c_float),
        ("youngs", C.c_float),
        ("poisson", C.c_float),
        ("boundary_friction", C.c_float),
        ("boundary_pad", C.c_uint32),
        ("sticky", C.c_uint32),
        ("n_materials", C.c_uint32),
        ("materials", orc_material * 8),
        ("svd_tol", C.c_double),
        ("svd_sweeps", C.c_uint32),
        ("jacobi_iters", C.c_uint32),
        ("n_rigid", C.c_uint32),
        ("rigid", (C.c_float * 7) * 8),
        ("wrench", (C.c_double * 6) * 8),
    ]


_lib = None


def _nullable(dtype):
    base = np.ctypeslib.ndpointer(dtype, flags="C_CONTIGUOUS")

    def from_param(cls, obj):
        if obj is None:
            return None
        return base.from_param(obj)

    return type(f"nullable_{np.dtype(dtype).name}", (base,), {"from_param": classmethod(from_param)})


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        f32p = _nullable(np.float32)
        f64p = _nullable(np.float64)
        u32p = _nullable(np.uint32)
        S = C.POINTER(orc_scene)
        L.orc_step_f32.argtypes = [S, C.c_int, f32p, f32p, f32p, f32p, f32p, f32p, f32p, u32p, f32p, f32p, u32p,
                                   C.c_int, C.c_int, C.c_int]
        L.orc_step_f64.argtypes = [S, C.c_int, f64p, f64p, f64p, f64p, f64p, f64p, f64p, u32p, f64p, f64p, u32p,
                                   C.c_int, C.c_int]
        L.orc_svd3_f32.argtypes = [f32p, f32p, f32p, f32p, C.c_double, C.c_int]
        L.orc_svd3_f64.argtypes = [f64p, f64p, f64p, f64p, C.c_double, C.c_int]
        L.orc_plasticity_f64.argtypes = [S, f64p, f64p, C.c_uint32]
        L.orc_gather_f64.argtypes = [S, f64p, f64p, f64p, f64p]
        L.orc_particle_order.argtypes = [S, C.c_uint32, C.c_uint32, f32p, u32p, u32p]
        L.orc_sort_pairs.argtypes = [C.c_uint32, u32p, u32p]
        L.orc_dp_alpha_f64.argtypes = [C.c_double]
        L.orc_dp_alpha_f64.restype = C.c_double
        L.orc_dp_alpha_f32.argtypes = [C.c_float]
        L.orc_dp_alpha_f32.restype = C.c_float
        L.orc_snow_clamp_f64.argtypes = [f64p, C.c_double, C.c_double, C.c_double, f64p, f64p]
        L.orc_sand_project_f64.argtypes = [f64p, C.c_double, C.c_double, C.c_double, C.c_double, f64p, f64p]
        L.orc_viscous_damping_f64.argtypes = [f64p, f64p, C.c_double, C.c_double, C.c_double, f64p, f64p, f64p]
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _get(obj, k, default=0.0):
    if isinstance(obj, dict):
        return obj.get(k, default)
    return getattr(obj, k, default)


def make_scene(cfg, rows, dt: float, svd_tol: float = 1e-7, svd_sweeps: int = 16) -> orc_scene:
    """orc_scene from an MpmConfig-like object (attributes or dict) and
    material rows (MpmRheology or dicts)."""
    s = orc_scene()
    s.grid_size = int(_get(cfg, "grid_size"))
    s.cell_size = float(_get(cfg, "cell_size"))
    s.inv_cell_size = float(np.float32(1.0) / np.float32(s.cell_size))
    org = _get(cfg, "grid_origin", (0.0, 0.0, 0.0))
    win = _get(cfg, "grid_window_cells", (0, 0, 0))
    for i in range(3):
        s.origin[i] = float(org[i])
        s.window[i] = int(win[i])
    s.dt = float(dt)
    s.gravity_y = float(_get(cfg, "gravity_y"))
    s.youngs = float(_get(cfg, "youngs"))
    s.poisson = float(_get(cfg, "poisson"))
    s.boundary_friction = float(_get(cfg, "boundary_friction"))
    s.boundary_pad = int(_get(cfg, "boundary_pad", 0))
    s.sticky = 1 if int(_get(cfg, "walls", 0)) == 1 else 0
    s.n_materials = len(rows)
    L = lib()
    for i, r in enumerate(rows):
        m = s.materials[i]
        kind = int(_get(r, "kind"))
        m.rheology = kind
        m.dp_alpha = L.orc_dp_alpha_f32(float(_get(r, "friction_angle"))) if kind == 0 else 0.0
        if kind == 1:
            m.theta_c = float(_get(r, "theta_c"))
            m.theta_s = float(_get(r, "theta_s"))
            m.hardening = float(_get(r, "hardening"))
        if kind == 2:
            m.velocity_damping = float(_get(r, "velocity_damping"))
            m.affine_damping = float(_get(r, "affine_damping"))
        m.youngs = float(_get(r, "youngs"))
        m.poisson = float(_get(r, "poisson"))
    s.svd_tol = svd_tol
    s.svd_sweeps = svd_sweeps
    s.jacobi_iters = int(_get(cfg, "jacobi_iters", 0)) if int(_get(cfg, "time_step", 0)) == 1 else 0
    return s


def init_state(positions, velocities=None, mass=1e-3, volume=1e-6, ids=None, dtype=np.float32) -> dict:
    """set_particles_with_velocity (mpm.rs:1458-1519): F = I, C = 0, jp = 0."""
    pos = np.ascontiguousarray(np.asarray(positions, dtype).reshape(-1, 3))
    n = pos.shape[0]
    vel = np.zeros((n, 3), dtype) if velocities is None else np.ascontiguousarray(np.asarray(velocities, dtype))
    F = np.zeros((n, 9), dtype)
    F[:, 0] = F[:, 4] = F[:, 8] = 1
    return {
        "pos": pos.copy(), "vel": vel.reshape(n, 3).copy(), "C": np.zeros((n, 9), dtype), "F": F,
        "mass": np.full(n, mass, dtype) if np.isscalar(mass) else np.asarray(mass, dtype).copy(),
        "vol": np.full(n, volume, dtype) if np.isscalar(volume) else np.asarray(volume, dtype).copy(),
        "jp": np.zeros(n, dtype),
        "mat": np.zeros(n, np.uint32) if ids is None else np.ascontiguousarray(np.asarray(ids, np.uint32)),
        "status": np.zeros(2, np.uint32),
    }


def cast_state(st: dict, dtype) -> dict:
    out = {k: (np.ascontiguousarray(v.astype(dtype)) if k not in ("mat", "status") else v.copy())
           for k, v in st.items()}
    return out


def step(scene: orc_scene, st: dict, substeps: int, precision: str = "f32", nthreads: int = 1,
         want_grid: bool = False):
    """Runs `substeps` reference substeps in place on `st`.  precision:
    "f32" (FP32), "f32_svd64" (FP32 state, FP64 SVD), "f64" (FP64).
    Returns (grid_mass, grid_momentum) of the last substep if want_grid."""
    L = lib()
    n3 = scene.grid_size ** 3
    n = st["pos"].shape[0]
    if precision == "f64":
        dt = np.float64
        gm = np.zeros(n3 if want_grid else 1, dt)
        gp = np.zeros(3 * n3 if want_grid else 1, dt)
        L.orc_step_f64(C.byref(scene), n, st["pos"], st["vel"], st["C"], st["F"], st["mass"], st["vol"], st["jp"],
                       st["mat"], gm if want_grid else None, gp if want_grid else None, st["status"], substeps,
                       nthreads)
    else:
        dt = np.float32
        gm = np.zeros(n3 if want_grid else 1, dt)
        gp = np.zeros(3 * n3 if want_grid else 1, dt)
        L.orc_step_f32(C.byref(scene), n, st["pos"], st["vel"], st["C"], st["F"], st["mass"], st["vol"], st["jp"],
                       st["mat"], gm if want_grid else None, gp if want_grid else None, st["status"], substeps,
                       1 if precision == "f32_svd64" else 0, nthreads)
    if want_grid:
        return gm, gp
    return None


def set_rigid_spheres(scene: orc_scene, spheres):
    """[(center_xyz, radius, velocity_xyz)] on the scene (at most 8)."""
    scene.n_rigid = len(spheres)
    for i, (c, r, v) in enumerate(spheres):
        vals = [*c, r, *v]
        for k in range(7):
            scene.rigid[i][k] = float(vals[k])


def rigid_wrenches(scene: orc_scene):
    """[(force_xyz, torque_xyz)] of the last substep."""
    return [(np.array(scene.wrench[i][:3]), np.array(scene.wrench[i][3:])) for i in range(scene.n_rigid)]


def particle_order(scene: orc_scene, positions, count: int, capacity: int):
    pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
    if pos.shape[0] == 0:
        pos = np.zeros((1, 3), np.float32)
    keys = np.empty(capacity, np.uint32)
    ids = np.empty(capacity, np.uint32)
    lib().orc_particle_order(C.byref(scene), count, capacity, pos, keys, ids)
    return keys, ids


def sort_pairs(keys, values):
    k = np.ascontiguousarray(np.asarray(keys, np.uint32)).copy()
    v = np.ascontiguousarray(np.asarray(values, np.uint32)).copy()
    lib().orc_sort_pairs(k.shape[0], k, v)
    return k, v


def svd3(F, precision="f32", tol=1e-7, sweeps=16):
    dt = np.float32 if precision == "f32" else np.float64
    f = np.ascontiguousarray(np.asarray(F, dt).reshape(9))
    U = np.empty(9, dt)
    s = np.empty(3, dt)
    V = np.empty(9, dt)
    (lib().orc_svd3_f32 if dt == np.float32 else lib().orc_svd3_f64)(f, U, s, V, tol, sweeps)
    return U, s, V


def max_threads() -> int:
    return int(lib().orc_max_threads())
