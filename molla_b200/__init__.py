"""molla_b200 — B200-native explicit MLS-MPM step with molla's solver interface.

Python mirror of molla's ``MpmSimulation`` API (crates/molla-solvers/src/mpm.rs,
re-exported at crates/molla-solvers/src/lib.rs:180-199) over the C ABI of
``include/molla_mpm.h``.  Names, argument meaning and error behaviour follow
the reference: ``MpmConfig.sand()``, ``MpmSimulation.new(engine, cfg)``,
``set_particles``, ``set_materials``, ``step`` / ``step_n``,
``prepare_step`` + ``begin_command_batch``, ``read_positions``,
``read_velocities``, ``read_grid_mass_momentum``,
``read_active_grid_status``.  Errors raise ``SolverError`` (Error::Solver) or
``GpuError`` (Error::Gpu).

Every call runs the CUDA library; there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from ._ffi import (MPM_ERR_BUSY, MPM_ERR_FAULT, MPM_ERR_GPU, MPM_ERR_INVALID, MPM_ERR_NOMEM, MPM_ERR_STALE,
                   MPM_ERR_UNSUPPORTED, MPM_OK)

__all__ = [
    "Engine", "MpmConfig", "MpmRheology", "MpmTimeStep", "MpmSimulation", "PreparedMpmStep", "MpmCommandBatch",
    "MpmActiveGridStats", "MpmParticleRenderView", "MpmParticleRenderSource", "MpmGroup", "MpmServer", "MpmSimulation64", "MollaError", "SolverError", "GpuError",
    "radix_sort_pairs", "blake3", "checkpoint_reencode",
    "MAX_MPM_MATERIALS", "library_path",
]

MAX_MPM_MATERIALS = 8  # crates/molla-solvers/src/mpm.rs:660


def library_path() -> str:
    return str(_ffi.LIB_PATH)


class MollaError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class SolverError(MollaError):
    """Error::Solver (invalid input or state)."""


class GpuError(MollaError):
    """Error::Gpu (device problems)."""


class StaleError(SolverError):
    """A prepared step belongs to another simulation or configuration."""


def _check(rc: int):
    if rc == MPM_OK:
        return
    msg = _ffi.last_error()
    if rc == MPM_ERR_GPU:
        raise GpuError(rc, msg)
    if rc == MPM_ERR_STALE:
        raise StaleError(rc, msg)
    raise SolverError(rc, msg)


def _f32(a, cols=None):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if cols is not None:
        arr = arr.reshape(-1, cols)
    return arr


def _fp(arr):
    return arr.ctypes.data_as(_ffi.F32P) if arr is not None else None


def _up(arr):
    return arr.ctypes.data_as(_ffi.U32P) if arr is not None else None


# ---------------------------------------------------------------------------

@dataclass
class MpmRheology:
    """MpmRheology (crates/molla-solvers/src/mpm.rs:320-370).

    ``youngs``/``poisson`` > 0 give a material row its own elastic moduli (an
    extension; 0 keeps the simulation-wide values as the reference does)."""

    kind: int
    friction_angle: float = 0.0
    theta_c: float = 0.0
    theta_s: float = 0.0
    hardening: float = 0.0
    velocity_damping: float = 0.0
    affine_damping: float = 0.0
    youngs: float = 0.0
    poisson: float = 0.0

    SAND = 0
    SNOW = 1
    VISCOUS = 2

    @classmethod
    def Sand(cls, friction_angle: float = math.radians(30.0), **kw):
        return cls(kind=0, friction_angle=friction_angle, **kw)

    @classmethod
    def Snow(cls, theta_c: float = 2.5e-2, theta_s: float = 7.5e-3, hardening: float = 10.0, **kw):
        return cls(kind=1, theta_c=theta_c, theta_s=theta_s, hardening=hardening, **kw)

    @classmethod
    def Viscous(cls, velocity_damping: float = 0.0, affine_damping: float = 0.0, **kw):
        return cls(kind=2, velocity_damping=velocity_damping, affine_damping=affine_damping, **kw)

    @classmethod
    def from_dict(cls, d: dict):
        return cls(**d)

    def to_c(self) -> _ffi.mpm_rheology:
        r = _ffi.mpm_rheology()
        for k in ("kind", "friction_angle", "theta_c", "theta_s", "hardening", "velocity_damping",
                  "affine_damping", "youngs", "poisson"):
            setattr(r, k, getattr(self, k))
        return r


class MpmTimeStep:
    """MpmTimeStep (mpm.rs:372-398); only Explicit is built."""

    EXPLICIT = 0
    IMPLICIT = 1


@dataclass
class MpmConfig:
    """MpmConfig (crates/molla-solvers/src/mpm.rs:400-433) plus extensions
    (boundary_pad, walls, svd_precision, grid_window_cells)."""

    grid_size: int = 32
    cell_size: float = 0.05
    grid_origin: tuple = (-0.8, 0.0, -0.8)
    gravity_y: float = -9.81
    youngs: float = 5.0e3
    poisson: float = 0.3
    friction_angle: float = math.radians(30.0)
    cohesion: float = 0.0
    boundary_friction: float = 0.5
    particle_mass: float = 1.0e-3
    particle_volume: float = 1.0e-6
    max_particles: int = 16384
    max_rigid: int = 8
    rheology: MpmRheology = field(default_factory=MpmRheology.Sand)
    time_step: int = MpmTimeStep.EXPLICIT
    jacobi_iters: int = 0
    boundary_pad: int = 0
    walls: int = 0
    svd_precision: int = 0
    grid_window_cells: tuple = (0, 0, 0)

    @classmethod
    def _preset(cls, idx: int) -> "MpmConfig":
        c = _ffi.mpm_config()
        _check(_ffi.lib().mpm_config_preset(idx, C.byref(c)))
        return cls.from_c(c)

    @classmethod
    def sand(cls):
        return cls._preset(0)

    @classmethod
    def sand_calibrated(cls):
        return cls._preset(1)

    @classmethod
    def snow(cls):
        return cls._preset(2)

    @classmethod
    def viscous(cls):
        return cls._preset(3)

    @classmethod
    def from_c(cls, c: _ffi.mpm_config) -> "MpmConfig":
        r = c.rheology
        rh = MpmRheology(kind=r.kind, friction_angle=r.friction_angle, theta_c=r.theta_c, theta_s=r.theta_s,
                         hardening=r.hardening, velocity_damping=r.velocity_damping,
                         affine_damping=r.affine_damping, youngs=r.youngs, poisson=r.poisson)
        return cls(grid_size=c.grid_size, cell_size=c.cell_size, grid_origin=tuple(c.grid_origin),
                   gravity_y=c.gravity_y, youngs=c.youngs, poisson=c.poisson, friction_angle=c.friction_angle,
                   cohesion=c.cohesion, boundary_friction=c.boundary_friction, particle_mass=c.particle_mass,
                   particle_volume=c.particle_volume, max_particles=c.max_particles, max_rigid=c.max_rigid,
                   rheology=rh, time_step=c.time_step, jacobi_iters=c.jacobi_iters, boundary_pad=c.boundary_pad,
                   walls=c.walls, svd_precision=c.svd_precision, grid_window_cells=tuple(c.grid_window_cells))

    def to_c(self) -> _ffi.mpm_config:
        c = _ffi.mpm_config()
        c.grid_size = self.grid_size
        c.cell_size = self.cell_size
        for i in range(3):
            c.grid_origin[i] = self.grid_origin[i]
            c.grid_window_cells[i] = self.grid_window_cells[i]
        for k in ("gravity_y", "youngs", "poisson", "friction_angle", "cohesion", "boundary_friction",
                  "particle_mass", "particle_volume", "max_particles", "max_rigid", "time_step", "jacobi_iters",
                  "boundary_pad", "walls", "svd_precision"):
            setattr(c, k, getattr(self, k))
        c.rheology = self.rheology.to_c()
        return c


@dataclass
class MpmActiveGridStats:
    """MpmActiveGridStats (mpm.rs:257-283).  active_tiles / overflow concern
    sparse grid storage (MpmSimulation.new_sparse)."""

    numerical_fault: bool
    completed_substeps: int
    fault_bits: int
    active_tiles: int = 0
    tile_capacity: int = 0

    @property
    def overflow(self) -> bool:
        return bool(self.fault_bits & 16)

    def faulted(self) -> bool:
        return self.numerical_fault or self.overflow


class Engine:
    """Engine::new_gpu (crates/molla-compute/src/engine.rs:140): a CUDA device
    and the engine's stream."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(_ffi.lib().mpm_engine_create(device, C.byref(h)))
        self._h = h

    @classmethod
    def new_gpu(cls, device: int = 0) -> "Engine":
        return cls(device)

    def check_device(self):
        _check(_ffi.lib().mpm_engine_check(self._h))

    def synchronize(self):
        _check(_ffi.lib().mpm_engine_synchronize(self._h))

    @property
    def stream_handle(self) -> int:
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(_ffi.lib().mpm_engine_stream(self._h) or 0)

    @property
    def launch_count(self) -> int:
        return int(_ffi.lib().mpm_engine_launch_count(self._h))

    def selftest_device_wait(self):
        """Runs the scatter's bounded-wait timeout path on a barrier nothing
        completes (about one second).  Returns (fault_bits, waited_ms)."""
        bits = C.c_uint32()
        ms = C.c_double()
        _check(_ffi.lib().mpm_selftest_device_wait(self._h, C.byref(bits), C.byref(ms)))
        return int(bits.value), float(ms.value)

    STAGES = ("ParticleOrdering", "StressRecord", "GridUpdate", "GridToParticle", "ParticleToGrid")

    def profile(self, enabled: bool = True):
        _check(_ffi.lib().mpm_profile_enable(self._h, int(bool(enabled))))

    def read_profile(self) -> dict:
        arr = (_ffi.mpm_profile_stage * 5)()
        _check(_ffi.lib().mpm_profile_read(self._h, arr, 5))
        return {name: (int(arr[i].launches), float(arr[i].total_ms)) for i, name in enumerate(self.STAGES)}

    def reset_profile(self):
        _check(_ffi.lib().mpm_profile_reset(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().mpm_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PreparedMpmStep:
    """PreparedMpmStep (crates/molla-solvers/src/mpm_command_batch.rs:9-16)."""

    def __init__(self, h, sim):
        self._h = h
        self._sim = sim

    def __del__(self):
        try:
            if self._h:
                _ffi.lib().mpm_prepared_destroy(self._h)
        except Exception:
            pass


class MpmCommandBatch:
    """MpmCommandBatch (mpm_command_batch.rs:18-27, 142-235): encode prepared
    steps, then submit; dropping it without submit discards the work."""

    def __init__(self, sim, stream=None):
        h = C.c_void_p()
        _check(_ffi.lib().mpm_batch_begin(sim._h, C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h
        self._sim = sim

    def encode_step(self, record: PreparedMpmStep):
        _check(_ffi.lib().mpm_batch_encode_step(self._h, record._h))

    def submit(self):
        rc = _ffi.lib().mpm_batch_submit(self._h)
        if rc == MPM_OK:
            self._h = None
        _check(rc)

    def __del__(self):
        try:
            if self._h:
                _ffi.lib().mpm_batch_cancel(self._h)
        except Exception:
            pass


class MpmParticleRenderSource:
    """MpmParticleRenderSource (mpm_render_view.rs:14-16): binding identity
    only; it does not freeze positions, count or physical time."""

    def __init__(self, token: int):
        self._token = int(token)

    def __eq__(self, other):
        return isinstance(other, MpmParticleRenderSource) and other._token == self._token

    def __hash__(self):
        return hash(self._token)

    def __repr__(self):
        return f"MpmParticleRenderSource({self._token})"


class MpmParticleRenderView:
    """MpmParticleRenderView (mpm_render_view.rs:3-36): live read-only
    positions on the simulation's device, float4 per particle (xyz in world
    metres, w = 0, 16-byte stride, original particle order); only the counted
    prefix is live.  Queue reads on the engine's stream after the physics.
    `__cuda_array_interface__` exposes the live prefix, so
    `torch.as_tensor(view, device="cuda")` binds it without a copy.  The
    interface's read-only flag is left clear because torch refuses it; the
    buffer is read-only by contract (the next step overwrites it)."""

    def __init__(self, raw: "_ffi.mpm_render_view", owner):
        self._ptr = int(raw.positions or 0)
        self._count = int(raw.count)
        self._capacity = int(raw.capacity)
        self._source = MpmParticleRenderSource(raw.source)
        self._bytes = int(raw.live_position_bytes)
        self._owner = owner  # keeps the simulation (and so the buffer) alive

    def positions(self) -> int:
        """Device address of the float4 position buffer."""
        return self._ptr

    def particle_count(self) -> int:
        return self._count

    @property
    def capacity(self) -> int:
        return self._capacity

    def live_position_bytes(self) -> int:
        return self._bytes

    def source(self) -> MpmParticleRenderSource:
        return self._source

    def matches_source(self, source: MpmParticleRenderSource) -> bool:
        return self._source == source

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self._count, 4), "typestr": "<f4", "data": (self._ptr if self._count else 0, False),
                "version": 3, "strides": None, "stream": None}


class MpmSimulation:
    """MpmSimulation (crates/molla-solvers/src/mpm.rs:695-2957) on the B200 path."""

    def __init__(self, engine: Engine, cfg: MpmConfig, tile_capacity: int | None = None):
        """tile_capacity: None for the dense grid, else sparse storage of that
        many 4^3-node tiles (MpmSimulation::new_sparse)."""
        self.engine = engine
        self.cfg = cfg
        self.tile_capacity = int(tile_capacity or 0)
        h = C.c_void_p()
        c = cfg.to_c()
        if tile_capacity is not None:
            _check(_ffi.lib().mpm_sim_create_sparse(engine._h, C.byref(c), int(tile_capacity), C.byref(h)))
        else:
            _check(_ffi.lib().mpm_sim_create(engine._h, C.byref(c), C.byref(h)))
        self._h = h
        self.particle_count = 0

    @classmethod
    def new(cls, engine: Engine, cfg: MpmConfig) -> "MpmSimulation":
        return cls(engine, cfg)

    @classmethod
    def new_sparse(cls, engine: Engine, cfg: MpmConfig, tile_capacity: int) -> "MpmSimulation":
        """MpmSimulation::new_sparse (mpm.rs:846-853): grid storage for
        tile_capacity tiles of 4^3 nodes."""
        return cls(engine, cfg, tile_capacity)

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().mpm_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- seeding ------------------------------------------------------------
    def set_particles(self, positions, velocities=None):
        pos = _f32(positions, 3)
        vel = None if velocities is None or len(velocities) == 0 else _f32(velocities, 3)
        if vel is not None and vel.shape[0] != pos.shape[0]:
            raise GpuError(MPM_ERR_GPU, f"velocities len ({vel.shape[0]}) != positions len ({pos.shape[0]})")
        _check(_ffi.lib().mpm_set_particles(self._h, _fp(pos), _fp(vel), pos.shape[0]))
        self.particle_count = pos.shape[0]

    set_particles_with_velocity = set_particles

    def set_particle_mass_volume(self, mass=None, volume=None):
        m = None if mass is None else _f32(mass).reshape(-1)
        v = None if volume is None else _f32(volume).reshape(-1)
        _check(_ffi.lib().mpm_set_particle_mass_volume(self._h, _fp(m), _fp(v), self.particle_count))

    def set_materials(self, materials, particle_material):
        rows = (_ffi.mpm_rheology * max(len(materials), 1))()
        for i, m in enumerate(materials):
            rows[i] = (m if isinstance(m, MpmRheology) else MpmRheology.from_dict(m)).to_c()
        ids = np.ascontiguousarray(np.asarray(particle_material, dtype=np.uint32))
        _check(_ffi.lib().mpm_set_materials(self._h, rows, len(materials), _up(ids), ids.shape[0]))

    def set_rheology(self, rheology: MpmRheology):
        r = rheology.to_c()
        _check(_ffi.lib().mpm_set_rheology(self._h, C.byref(r)))

    def set_material(self, youngs: float, friction_angle: float):
        _check(_ffi.lib().mpm_set_material(self._h, youngs, friction_angle))

    def set_time_step(self, kind: int, jacobi_iters: int = 0):
        _check(_ffi.lib().mpm_set_time_step(self._h, kind, jacobi_iters))

    def set_p2g_mode(self, two_pass: bool):
        _check(_ffi.lib().mpm_set_p2g_mode(self._h, int(bool(two_pass))))

    def prepare_deterministic_p2g(self):
        _check(_ffi.lib().mpm_prepare_deterministic_p2g(self._h))

    def set_deterministic_p2g(self, enabled: bool):
        _check(_ffi.lib().mpm_set_deterministic_p2g(self._h, int(bool(enabled))))

    def release_deterministic_p2g(self):
        _check(_ffi.lib().mpm_release_deterministic_p2g(self._h))

    def _info(self) -> _ffi.mpm_sim_info:
        i = _ffi.mpm_sim_info()
        _check(_ffi.lib().mpm_sim_info_get(self._h, C.byref(i)))
        return i

    def uses_two_pass_p2g(self) -> bool:
        return bool(self._info().uses_two_pass_p2g)

    def deterministic_p2g_enabled(self) -> bool:
        return bool(self._info().deterministic_p2g)

    def particle_tile_ordering_enabled(self) -> bool:
        return bool(self._info().tile_ordering)

    def config(self) -> MpmConfig:
        """The configuration with every later setter applied (mpm.rs:1245-1247)."""
        c = _ffi.mpm_config()
        _check(_ffi.lib().mpm_sim_config(self._h, C.byref(c)))
        return MpmConfig.from_c(c)

    def prepare_particle_tile_ordering(self, capacity: int):
        _check(_ffi.lib().mpm_prepare_particle_tile_ordering(self._h, capacity))

    def set_particle_tile_ordering(self, enabled: bool):
        _check(_ffi.lib().mpm_set_particle_tile_ordering(self._h, int(bool(enabled))))

    def set_sort_interval(self, interval: int):
        _check(_ffi.lib().mpm_set_sort_interval(self._h, interval))

    def autotune(self, dt: float, probe_substeps: int = 64, candidates=(4, 8, 16, 32, 64, 128)):
        """Picks the regrouping interval by timing each candidate on a
        snapshot of the state (the simulation does not advance).  Returns
        (chosen, {candidate: ms per substep})."""
        c = np.ascontiguousarray(np.asarray(candidates, np.uint32))
        ms = np.zeros(len(c), np.float32)
        chosen = C.c_uint32()
        _check(_ffi.lib().mpm_autotune(self._h, dt, probe_substeps, _up(c), len(c), _fp(ms), C.byref(chosen)))
        return int(chosen.value), dict(zip(c.tolist(), ms.tolist()))

    # -- stepping -----------------------------------------------------------
    def autotune_shapes(self, dt: float, probe_substeps: int = 32):
        """MpmGroup.autotune_shapes for this simulation."""
        return _tune_shapes(lambda sh, pr, cap, n: _ffi.lib().mpm_autotune_shapes(
            self._h, dt, probe_substeps, sh, pr, cap, n))

    def step(self, dt: float, engine=None):
        self.step_n(dt, 1)

    def step_n(self, dt: float, substeps: int, engine=None):
        _check(_ffi.lib().mpm_step_n(self._h, dt, substeps))

    def prepare_step(self, dt: float, substeps: int) -> PreparedMpmStep:
        h = C.c_void_p()
        _check(_ffi.lib().mpm_prepare_step(self._h, dt, substeps, C.byref(h)))
        return PreparedMpmStep(h, self)

    def begin_command_batch(self, stream=None) -> MpmCommandBatch:
        return MpmCommandBatch(self, stream)

    # -- readback -----------------------------------------------------------
    def _read3(self, fn, out=None):
        n = C.c_uint32()
        if out is None:
            out = np.empty((max(self.particle_count, 1), 3), np.float32)
        elif (out.dtype != np.float32 or out.ndim != 2 or out.shape[1] != 3 or not out.flags.c_contiguous
              or out.shape[0] < self.particle_count):
            raise SolverError(MPM_ERR_INVALID, "out must be a C-contiguous float32 (>= n, 3) array")
        _check(fn(self._h, _fp(out), self.particle_count, C.byref(n)))
        return out[: n.value]

    def read_positions(self, out=None) -> np.ndarray:
        """Positions in original particle order.  `out` (optional) is a
        float32 (>= n, 3) array to fill, e.g. in pinned memory for a fast
        device-to-host copy; the returned array is its first n rows."""
        return self._read3(_ffi.lib().mpm_read_positions, out)

    def particle_render_view(self, engine=None) -> MpmParticleRenderView:
        """particle_render_view (mpm_render_view.rs:38-56).  The first call
        allocates the buffer and packs it once; later calls neither allocate
        nor launch nor copy."""
        if engine is not None and engine is not self.engine:
            raise GpuError(MPM_ERR_INVALID, "particle render view requested on a foreign engine")
        raw = _ffi.mpm_render_view()
        _check(_ffi.lib().mpm_particle_render_view(self._h, C.byref(raw)))
        return MpmParticleRenderView(raw, self)

    def read_velocities(self, out=None) -> np.ndarray:
        return self._read3(_ffi.lib().mpm_read_velocities, out)

    def read_particle_state(self):
        """(C[n,9], F[n,9], jp[n]), matrices column-major per particle."""
        n = max(self.particle_count, 1)
        Cm = np.empty((n, 9), np.float32)
        Fm = np.empty((n, 9), np.float32)
        jp = np.empty(n, np.float32)
        cnt = C.c_uint32()
        _check(_ffi.lib().mpm_read_particle_state(self._h, _fp(Cm), _fp(Fm), _fp(jp), n, C.byref(cnt)))
        k = cnt.value
        return Cm[:k], Fm[:k], jp[:k]

    def write_particle_state(self, C_=None, F=None, jp=None):
        c = None if C_ is None else _f32(C_, 9)
        f = None if F is None else _f32(F, 9)
        j = None if jp is None else _f32(jp).reshape(-1)
        _check(_ffi.lib().mpm_write_particle_state(self._h, _fp(c), _fp(f), _fp(j), self.particle_count))

    def read_grid_mass_momentum(self):
        n3 = self.cfg.grid_size ** 3
        m = np.empty(n3, np.float32)
        p = np.empty(3 * n3, np.float32)
        _check(_ffi.lib().mpm_read_grid_mass_momentum(self._h, _fp(m), _fp(p), n3))
        return m, p

    def set_rigid_spheres(self, spheres):
        """set_rigid_spheres (mpm.rs:1521-1565): [(center_xyz, radius, velocity_xyz)]."""
        arr = np.zeros((max(len(spheres), 1), 7), np.float32)
        for i, (c, r, v) in enumerate(spheres):
            arr[i, 0:3] = c
            arr[i, 3] = r
            arr[i, 4:7] = v
        _check(_ffi.lib().mpm_set_rigid_spheres(self._h, _fp(arr), len(spheres)))

    def read_rigid_wrenches(self):
        """read_rigid_wrenches (mpm.rs:2809): [(force_xyz, torque_xyz)] of the last substep."""
        cap = 8
        out = np.zeros((cap, 6), np.float32)
        cnt = C.c_uint32()
        _check(_ffi.lib().mpm_read_rigid_wrenches(self._h, _fp(out), cap, C.byref(cnt)))
        return [(out[i, :3].copy(), out[i, 3:].copy()) for i in range(cnt.value)]

    def checkpoint_soil(self) -> bytes:
        """checkpoint_soil_with (mpm_checkpoint.rs:388-434): the particle state
        in molla's versioned soil-checkpoint bytes (BLAKE3 digest)."""
        size = C.c_size_t()
        _check(_ffi.lib().mpm_checkpoint_save(self._h, None, 0, C.byref(size)))
        out = (C.c_ubyte * max(size.value, 1))()
        _check(_ffi.lib().mpm_checkpoint_save(self._h, out, size.value, C.byref(size)))
        return bytes(out)[: size.value]

    def restore_soil(self, data: bytes):
        """from_bytes + restore_soil_with (mpm_checkpoint.rs:218-275, 436-542)."""
        raw = bytes(data)
        _check(_ffi.lib().mpm_checkpoint_load(self._h, raw, len(raw)))
        words = np.frombuffer(raw[44:], dtype="<u4")
        off = (3 if int.from_bytes(raw[8:12], "little") == 2 else 0) + 21
        rows = int(words[off])
        self.particle_count = int(words[off + 1 + 4 * rows])

    def conservation_totals(self) -> np.ndarray:
        out = np.zeros(8, np.float64)
        _check(_ffi.lib().mpm_conservation_totals(self._h, out.ctypes.data_as(_ffi.F64P)))
        return out

    def read_active_grid_status(self) -> MpmActiveGridStats:
        s = _ffi.mpm_status_info()
        _check(_ffi.lib().mpm_read_status(self._h, C.byref(s)))
        return MpmActiveGridStats(bool(s.numerical_fault), int(s.completed_substeps), int(s.fault_bits),
                                  int(s.active_tiles), getattr(self, 'tile_capacity', 0))

    read_active_grid_status_with = read_active_grid_status

    def reset_active_grid(self):
        _check(_ffi.lib().mpm_reset_fault(self._h))

    def read_sort_permutation(self, capacity: int | None = None):
        """Tile keys and identities of the stable (key, index) order over
        ``capacity`` entries (ParticleOrder, mpm_particle_order.rs:118-150)."""
        cap = self.particle_count if capacity is None else capacity
        keys = np.empty(max(cap, 1), np.uint32)
        ids = np.empty(max(cap, 1), np.uint32)
        _check(_ffi.lib().mpm_read_sort_permutation(self._h, _up(keys), _up(ids), cap))
        return keys[:cap], ids[:cap]


def radix_sort_pairs(engine: Engine, keys, values, key_bits: int = 32):
    """Stable sort of (u32 key, u32 value) pairs on the GPU (RadixSortKernel,
    crates/molla-compute-primitives/src/radix_sort.rs:50-110)."""
    k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint32)).copy()
    v = np.ascontiguousarray(np.asarray(values, dtype=np.uint32)).copy()
    if k.shape != v.shape:
        raise SolverError(MPM_ERR_INVALID, "keys and values differ in length")
    _check(_ffi.lib().mpm_radix_sort_pairs(engine._h, _up(k), _up(v), k.shape[0], key_bits))
    return k, v


def _rows_c(rows):
    arr = (_ffi.mpm_rheology * max(len(rows), 1))()
    for i, m in enumerate(rows):
        arr[i] = (m if isinstance(m, MpmRheology) else MpmRheology.from_dict(m)).to_c()
    return arr


def blake3(data: bytes) -> bytes:
    """BLAKE3 (unkeyed, 32 bytes) of data: the soil-checkpoint digest."""
    buf = (C.c_ubyte * 32)()
    raw = bytes(data)
    _check(_ffi.lib().mpm_blake3(raw, len(raw), buf))
    return bytes(buf)


def checkpoint_reencode(data: bytes, max_particles: int):
    """Decodes and validates a soil checkpoint (no GPU) and encodes it again;
    returns (bytes, particle count).  Raises SolverError on invalid data."""
    raw = bytes(data)
    size = C.c_size_t()
    count = C.c_uint32()
    _check(_ffi.lib().mpm_checkpoint_reencode(raw, len(raw), max_particles, None, 0, C.byref(size), C.byref(count)))
    out = (C.c_ubyte * max(size.value, 1))()
    _check(_ffi.lib().mpm_checkpoint_reencode(raw, len(raw), max_particles, out, size.value, C.byref(size),
                                              C.byref(count)))
    return bytes(out)[: size.value], int(count.value)


class MpmSimulation64:
    """All-FP64 run of the reference substep on the GPU (FP64 state, grid and
    Jacobi SVD), for precision studies of the FP32 and FP32 + FP64-SVD modes.
    Positions are set and read in float64."""

    def __init__(self, engine: Engine, cfg: MpmConfig):
        self.engine = engine
        self.cfg = cfg
        h = C.c_void_p()
        c = cfg.to_c()
        _check(_ffi.lib().mpm_sim64_create(engine._h, C.byref(c), C.byref(h)))
        self._h = h
        self.particle_count = 0

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().mpm_sim64_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_particles(self, positions):
        x = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        _check(_ffi.lib().mpm_sim64_set_particles(self._h, x.ctypes.data_as(_ffi.F64P), x.shape[0]))
        self.particle_count = x.shape[0]

    def set_materials(self, materials, particle_material):
        rows = (_ffi.mpm_rheology * max(len(materials), 1))()
        for i, m in enumerate(materials):
            rows[i] = (m if isinstance(m, MpmRheology) else MpmRheology.from_dict(m)).to_c()
        ids = np.ascontiguousarray(np.asarray(particle_material, dtype=np.uint32))
        _check(_ffi.lib().mpm_sim64_set_materials(self._h, rows, len(materials), _up(ids), ids.shape[0]))

    def step_n(self, dt: float, substeps: int):
        _check(_ffi.lib().mpm_sim64_step_n(self._h, float(dt), substeps))

    def read_state(self):
        """(positions (n,3), velocities (n,3), F (n,9) column-major), float64."""
        n = max(self.particle_count, 1)
        pos = np.empty((n, 3), np.float64)
        vel = np.empty((n, 3), np.float64)
        F = np.empty((n, 9), np.float64)
        cnt = C.c_uint32()
        _check(_ffi.lib().mpm_sim64_read_state(self._h, pos.ctypes.data_as(_ffi.F64P), vel.ctypes.data_as(_ffi.F64P),
                                               F.ctypes.data_as(_ffi.F64P), n, C.byref(cnt)))
        k = cnt.value
        return pos[:k], vel[:k], F[:k]

    def read_positions(self):
        return self.read_state()[0]

    def grid_totals(self):
        """(mass, momentum[3]) of the last P2G, FP64."""
        out = np.zeros(4, np.float64)
        _check(_ffi.lib().mpm_sim64_grid_totals(self._h, out.ctypes.data_as(_ffi.F64P)))
        return float(out[0]), out[1:].copy()

    def read_active_grid_status(self) -> MpmActiveGridStats:
        s = _ffi.mpm_status_info()
        _check(_ffi.lib().mpm_sim64_read_status(self._h, C.byref(s)))
        return MpmActiveGridStats(bool(s.numerical_fault), int(s.completed_substeps), int(s.fault_bits),
                                  int(s.active_tiles), getattr(self, 'tile_capacity', 0))


TUNE_KNOBS = ("sort_interval", "item_particles", "fused", "gather_ctas_per_sm", "scatter_ctas_per_sm")


def _shapes_dict(sh) -> dict:
    return {k: int(getattr(sh, k)) for k in TUNE_KNOBS}


def _tune_shapes(call):
    sh = _ffi.mpm_shapes()
    cap = 64
    probes = (_ffi.mpm_tune_probe * cap)()
    n = C.c_uint32()
    _check(call(C.byref(sh), probes, cap, C.byref(n)))
    return _shapes_dict(sh), [(TUNE_KNOBS[p.knob], int(p.value), float(p.ms_per_substep))
                              for p in probes[: min(n.value, cap)]]


class MpmGroup:
    """Many independent scenes stepped by shared launches (no reference
    equivalent; same per-scene numerics as MpmSimulation)."""

    def __init__(self, engine: Engine, max_scenes: int, max_particles: int, max_cells: int):
        self.engine = engine
        h = C.c_void_p()
        _check(_ffi.lib().mpm_group_create(engine._h, max_scenes, max_particles, max_cells, C.byref(h)))
        self._h = h
        self.counts = {}

    def add_scene(self, cfg: MpmConfig, rows, positions, ids=None, dt: float = 1e-4, tile_capacity: int = 0) -> int:
        """tile_capacity > 0: sparse grid storage of that many 4^3-node tiles."""
        c = cfg.to_c()
        r = _rows_c(rows)
        pos = _f32(positions, 3)
        idv = None if ids is None else np.ascontiguousarray(np.asarray(ids, np.uint32))
        sid = C.c_uint32()
        if tile_capacity:
            _check(_ffi.lib().mpm_group_add_scene_sparse(self._h, C.byref(c), r, len(rows), _fp(pos), _up(idv),
                                                         pos.shape[0], dt, int(tile_capacity), C.byref(sid)))
        else:
            _check(_ffi.lib().mpm_group_add_scene(self._h, C.byref(c), r, len(rows), _fp(pos), _up(idv),
                                                  pos.shape[0], dt, C.byref(sid)))
        self.counts[sid.value] = pos.shape[0]
        return sid.value

    def remove_scene(self, sid: int):
        _check(_ffi.lib().mpm_group_remove_scene(self._h, sid))
        self.counts.pop(sid, None)

    def step(self, substeps: int):
        _check(_ffi.lib().mpm_group_step(self._h, substeps))

    def step_graph(self, substeps: int, repeat: int = 1):
        _check(_ffi.lib().mpm_group_step_graph(self._h, substeps, repeat))

    def tune(self, chunk: int = 0, sort_interval: int = 0):
        _check(_ffi.lib().mpm_group_tune(self._h, chunk, sort_interval))

    def set_deterministic(self, enabled: bool):
        _check(_ffi.lib().mpm_group_set_deterministic(self._h, int(bool(enabled))))

    def autotune(self, probe_substeps: int = 64, candidates=(4, 8, 16, 32, 64, 128)):
        """Picks the regrouping interval by timing each candidate on a
        snapshot of the state (the scenes do not advance).  Returns
        (chosen, {candidate: ms per substep})."""
        c = np.ascontiguousarray(np.asarray(candidates, np.uint32))
        ms = np.zeros(len(c), np.float32)
        chosen = C.c_uint32()
        _check(_ffi.lib().mpm_group_autotune(self._h, probe_substeps, _up(c), len(c), _fp(ms), C.byref(chosen)))
        return int(chosen.value), dict(zip(c.tolist(), ms.tolist()))

    def autotune_shapes(self, probe_substeps: int = 32):
        """Tunes the regroup interval, the item size, fused vs separate
        kernels and the CTAs per SM of the gather and scatter on a snapshot
        (the scenes do not advance).  Returns (shapes dict, [(knob, value,
        ms per substep), ...])."""
        return _tune_shapes(lambda sh, pr, cap, n: _ffi.lib().mpm_group_autotune_shapes(
            self._h, probe_substeps, sh, pr, cap, n))

    def shapes(self) -> dict:
        sh = _ffi.mpm_shapes()
        _check(_ffi.lib().mpm_group_get_shapes(self._h, C.byref(sh)))
        return _shapes_dict(sh)

    def set_shapes(self, **kw):
        sh = _ffi.mpm_shapes()
        _check(_ffi.lib().mpm_group_get_shapes(self._h, C.byref(sh)))
        for k, v in kw.items():
            setattr(sh, k, int(v))
        _check(_ffi.lib().mpm_group_set_shapes(self._h, C.byref(sh)))

    def read_positions(self, sid: int) -> np.ndarray:
        n = self.counts[sid]
        out = np.empty((max(n, 1), 3), np.float32)
        cnt = C.c_uint32()
        _check(_ffi.lib().mpm_group_read_positions(self._h, sid, _fp(out), n, C.byref(cnt)))
        return out[: cnt.value]

    def read_status(self, sid: int) -> MpmActiveGridStats:
        s = _ffi.mpm_status_info()
        _check(_ffi.lib().mpm_group_read_status(self._h, sid, C.byref(s)))
        return MpmActiveGridStats(bool(s.numerical_fault), int(s.completed_substeps), int(s.fault_bits),
                                  int(s.active_tiles), getattr(self, 'tile_capacity', 0))

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().mpm_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MpmServer:
    """Continuous-batching request loop: admits scenes by HBM budget, steps
    the resident ones together, retires finished ones."""

    def __init__(self, engine: Engine, hbm_budget_bytes: int, max_scenes: int = 1024):
        self.engine = engine
        h = C.c_void_p()
        _check(_ffi.lib().mpm_server_create(engine._h, hbm_budget_bytes, max_scenes, C.byref(h)))
        self._h = h
        self.counts = {}

    def submit(self, cfg: MpmConfig, rows, positions, ids=None, dt: float = 1e-4, steps: int = 100) -> int:
        c = cfg.to_c()
        r = _rows_c(rows)
        pos = _f32(positions, 3)
        idv = None if ids is None else np.ascontiguousarray(np.asarray(ids, np.uint32))
        t = C.c_uint64()
        _check(_ffi.lib().mpm_server_submit(self._h, C.byref(c), r, len(rows), _fp(pos), _up(idv), pos.shape[0], dt,
                                            steps, C.byref(t)))
        self.counts[t.value] = pos.shape[0]
        return t.value

    def run(self, ticks: int, substeps_per_tick: int = 50):
        _check(_ffi.lib().mpm_server_run(self._h, ticks, substeps_per_tick))

    def poll(self, ticket: int):
        n = self.counts[ticket]
        out = np.empty((max(n, 1), 3), np.float32)
        st = C.c_uint32()
        cnt = C.c_uint32()
        _check(_ffi.lib().mpm_server_poll(self._h, ticket, C.byref(st), _fp(out), n, C.byref(cnt)))
        return int(st.value), (out[: cnt.value] if st.value in (2, 3) else None)

    def ticket_status(self, ticket: int) -> MpmActiveGridStats:
        """Device status of a finished request (state 2 done, 3 faulted) as it
        stood at its retirement."""
        s = _ffi.mpm_status_info()
        _check(_ffi.lib().mpm_server_ticket_status(self._h, ticket, C.byref(s)))
        return MpmActiveGridStats(bool(s.numerical_fault), int(s.completed_substeps), int(s.fault_bits))

    def stats(self) -> dict:
        s = _ffi.mpm_server_stats()
        _check(_ffi.lib().mpm_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _ffi.mpm_server_stats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _ffi.lib().mpm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def config_for_scene(scene, max_particles: int | None = None, svd_precision: int = 0) -> MpmConfig:
    """MpmConfig of a generated scene (molla_b200.scenes.Scene)."""
    return MpmConfig(grid_size=scene.grid_size, cell_size=scene.cell_size, grid_origin=tuple(scene.origin),
                     gravity_y=scene.gravity_y, youngs=scene.youngs, poisson=scene.poisson, friction_angle=0.0,
                     boundary_friction=scene.boundary_friction, particle_mass=scene.particle_mass,
                     particle_volume=scene.particle_volume,
                     max_particles=max_particles if max_particles is not None else scene.n,
                     rheology=MpmRheology.from_dict(scene.rows[0]), boundary_pad=scene.boundary_pad,
                     walls=scene.walls, svd_precision=svd_precision)
