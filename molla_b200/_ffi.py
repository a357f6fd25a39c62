"""ctypes binding of libmolla_mpm.so (the C ABI of include/molla_mpm.h).

The library is the product: there is no CPU or PyTorch fallback.  Loading
fails loudly when the shared object is missing.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmolla_mpm.so"

MPM_OK = 0
MPM_ERR_INVALID = 1
MPM_ERR_GPU = 2
MPM_ERR_FAULT = 3
MPM_ERR_STALE = 4
MPM_ERR_NOMEM = 5
MPM_ERR_UNSUPPORTED = 6
MPM_ERR_BUSY = 7


class mpm_rheology(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("friction_angle", C.c_float),
        ("theta_c", C.c_float),
        ("theta_s", C.c_float),
        ("hardening", C.c_float),
        ("velocity_damping", C.c_float),
        ("affine_damping", C.c_float),
        ("youngs", C.c_float),
        ("poisson", C.c_float),
    ]


class mpm_config(C.Structure):
    _fields_ = [
        ("grid_size", C.c_uint32),
        ("cell_size", C.c_float),
        ("grid_origin", C.c_float * 3),
        ("gravity_y", C.c_float),
        ("youngs", C.c_float),
        ("poisson", C.c_float),
        ("friction_angle", C.c_float),
        ("cohesion", C.c_float),
        ("boundary_friction", C.c_float),
        ("particle_mass", C.c_float),
        ("particle_volume", C.c_float),
        ("max_particles", C.c_uint32),
        ("max_rigid", C.c_uint32),
        ("rheology", mpm_rheology),
        ("time_step", C.c_uint32),
        ("jacobi_iters", C.c_uint32),
        ("boundary_pad", C.c_uint32),
        ("walls", C.c_uint32),
        ("svd_precision", C.c_uint32),
        ("grid_window_cells", C.c_int32 * 3),
        ("reserved", C.c_uint32 * 8),
    ]


class mpm_status_info(C.Structure):
    _fields_ = [
        ("numerical_fault", C.c_uint32),
        ("completed_substeps", C.c_uint32),
        ("fault_bits", C.c_uint32),
        ("active_tiles", C.c_uint32),
    ]


class mpm_server_stats(C.Structure):
    _fields_ = [
        ("admitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("resident_scenes", C.c_uint64),
        ("resident_bytes", C.c_uint64),
        ("particle_steps", C.c_uint64),
        ("tick_ms_p50", C.c_double),
        ("tick_ms_p99", C.c_double),
        ("queue_ms_p50", C.c_double),
        ("queue_ms_p99", C.c_double),
        ("admit_ms", C.c_double),
        ("step_ms", C.c_double),
        ("retire_ms", C.c_double),
        ("ticks", C.c_uint64),
        ("faulted", C.c_uint64),
        ("graph_builds", C.c_uint64),
        ("graph_build_ms", C.c_double),
    ]


class mpm_shapes(C.Structure):
    _fields_ = [
        ("sort_interval", C.c_uint32),
        ("item_particles", C.c_uint32),
        ("fused", C.c_uint32),
        ("gather_ctas_per_sm", C.c_uint32),
        ("scatter_ctas_per_sm", C.c_uint32),
        ("reserved", C.c_uint32 * 3),
    ]


class mpm_tune_probe(C.Structure):
    _fields_ = [("knob", C.c_uint32), ("value", C.c_uint32), ("ms_per_substep", C.c_float)]


class mpm_render_view(C.Structure):
    _fields_ = [
        ("positions", C.c_void_p),
        ("count", C.c_uint32),
        ("capacity", C.c_uint32),
        ("source", C.c_uint64),
        ("live_position_bytes", C.c_uint64),
    ]


class mpm_sim_info(C.Structure):
    _fields_ = [
        ("particle_count", C.c_uint32),
        ("uses_two_pass_p2g", C.c_uint32),
        ("deterministic_p2g", C.c_uint32),
        ("deterministic_prepared", C.c_uint32),
        ("tile_ordering", C.c_uint32),
        ("tile_ordering_capacity", C.c_uint32),
        ("sort_interval", C.c_uint32),
        ("max_particles", C.c_uint32),
    ]


class mpm_profile_stage(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("total_ms", C.c_double)]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
F32P = C.POINTER(C.c_float)
U32P = C.POINTER(C.c_uint32)
U64P = C.POINTER(C.c_uint64)
F64P = C.POINTER(C.c_double)
I = C.c_int
U32 = C.c_uint32
U64 = C.c_uint64

# name -> (restype, argtypes)
SIGNATURES = {
    "mpm_abi_version": (U32, []),
    "mpm_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "mpm_engine_create": (I, [I, PP]),
    "mpm_engine_destroy": (I, [P]),
    "mpm_engine_check": (I, [P]),
    "mpm_engine_synchronize": (I, [P]),
    "mpm_engine_launch_count": (U64, [P]),
    "mpm_selftest_device_wait": (I, [P, U32P, C.POINTER(C.c_double)]),
    "mpm_engine_stream": (P, [P]),
    "mpm_config_preset": (I, [U32, C.POINTER(mpm_config)]),
    "mpm_dp_alpha": (C.c_float, [C.c_float]),
    "mpm_sim_create": (I, [P, C.POINTER(mpm_config), PP]),
    "mpm_sim_create_sparse": (I, [P, C.POINTER(mpm_config), U32, PP]),
    "mpm_sim_destroy": (I, [P]),
    "mpm_set_particles": (I, [P, F32P, F32P, U32]),
    "mpm_set_particle_mass_volume": (I, [P, F32P, F32P, U32]),
    "mpm_set_materials": (I, [P, C.POINTER(mpm_rheology), U32, U32P, U32]),
    "mpm_set_rheology": (I, [P, C.POINTER(mpm_rheology)]),
    "mpm_set_material": (I, [P, C.c_float, C.c_float]),
    "mpm_set_time_step": (I, [P, U32, U32]),
    "mpm_set_p2g_mode": (I, [P, I]),
    "mpm_prepare_deterministic_p2g": (I, [P]),
    "mpm_set_deterministic_p2g": (I, [P, I]),
    "mpm_release_deterministic_p2g": (I, [P]),
    "mpm_sim_info_get": (I, [P, C.POINTER(mpm_sim_info)]),
    "mpm_sim_config": (I, [P, C.POINTER(mpm_config)]),
    "mpm_prepare_particle_tile_ordering": (I, [P, U32]),
    "mpm_set_particle_tile_ordering": (I, [P, I]),
    "mpm_set_sort_interval": (I, [P, U32]),
    "mpm_step_n": (I, [P, C.c_float, U32]),
    "mpm_prepare_step": (I, [P, C.c_float, U32, PP]),
    "mpm_prepared_destroy": (I, [P]),
    "mpm_batch_begin": (I, [P, P, PP]),
    "mpm_batch_encode_step": (I, [P, P]),
    "mpm_batch_submit": (I, [P]),
    "mpm_batch_cancel": (I, [P]),
    "mpm_read_positions": (I, [P, F32P, U32, U32P]),
    "mpm_particle_render_view": (I, [P, C.POINTER(mpm_render_view)]),
    "mpm_read_velocities": (I, [P, F32P, U32, U32P]),
    "mpm_read_particle_state": (I, [P, F32P, F32P, F32P, U32, U32P]),
    "mpm_write_particle_state": (I, [P, F32P, F32P, F32P, U32]),
    "mpm_read_grid_mass_momentum": (I, [P, F32P, F32P, C.c_size_t]),
    "mpm_conservation_totals": (I, [P, F64P]),
    "mpm_read_status": (I, [P, C.POINTER(mpm_status_info)]),
    "mpm_reset_fault": (I, [P]),
    "mpm_read_sort_permutation": (I, [P, U32P, U32P, U32]),
    "mpm_radix_sort_pairs": (I, [P, U32P, U32P, U32, U32]),
    "mpm_radix_sort_pairs_device": (I, [P, P, P, U32, U32, P]),
    "mpm_radix_sort_pairs_noalloc": (I, [P, P, U32, U32, P]),
    "mpm_profile_enable": (I, [P, I]),
    "mpm_profile_read": (I, [P, C.POINTER(mpm_profile_stage), U32]),
    "mpm_profile_reset": (I, [P]),
    "mpm_group_create": (I, [P, U32, U64, U64, PP]),
    "mpm_group_destroy": (I, [P]),
    "mpm_group_add_scene": (I, [P, C.POINTER(mpm_config), C.POINTER(mpm_rheology), U32, F32P, U32P, U32,
                                C.c_float, U32P]),
    "mpm_group_add_scene_sparse": (I, [P, C.POINTER(mpm_config), C.POINTER(mpm_rheology), U32, F32P, U32P, U32,
                                       C.c_float, U32, U32P]),
    "mpm_group_remove_scene": (I, [P, U32]),
    "mpm_group_step": (I, [P, U32]),
    "mpm_group_step_graph": (I, [P, U32, U32]),
    "mpm_group_read_positions": (I, [P, U32, F32P, U32, U32P]),
    "mpm_group_read_status": (I, [P, U32, C.POINTER(mpm_status_info)]),
    "mpm_group_scene_count": (I, [P, U32P]),
    "mpm_group_set_deterministic": (I, [P, I]),
    "mpm_group_autotune": (I, [P, U32, U32P, U32, F32P, U32P]),
    "mpm_autotune": (I, [P, C.c_float, U32, U32P, U32, F32P, U32P]),
    "mpm_group_tune": (I, [P, U32, U32]),
    "mpm_group_autotune_shapes": (I, [P, U32, C.POINTER(mpm_shapes), C.POINTER(mpm_tune_probe), U32, U32P]),
    "mpm_autotune_shapes": (I, [P, C.c_float, U32, C.POINTER(mpm_shapes), C.POINTER(mpm_tune_probe), U32, U32P]),
    "mpm_group_get_shapes": (I, [P, C.POINTER(mpm_shapes)]),
    "mpm_group_set_shapes": (I, [P, C.POINTER(mpm_shapes)]),
    "mpm_set_rigid_spheres": (I, [P, F32P, U32]),
    "mpm_read_rigid_wrenches": (I, [P, F32P, U32, U32P]),
    "mpm_checkpoint_save": (I, [P, P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "mpm_checkpoint_load": (I, [P, P, C.c_size_t]),
    "mpm_checkpoint_reencode": (I, [P, C.c_size_t, U32, P, C.c_size_t, C.POINTER(C.c_size_t), U32P]),
    "mpm_blake3": (I, [P, C.c_size_t, P]),
    "mpm_sim64_create": (I, [P, C.POINTER(mpm_config), PP]),
    "mpm_sim64_destroy": (I, [P]),
    "mpm_sim64_set_particles": (I, [P, F64P, U32]),
    "mpm_sim64_set_materials": (I, [P, C.POINTER(mpm_rheology), U32, U32P, U32]),
    "mpm_sim64_step_n": (I, [P, C.c_double, U32]),
    "mpm_sim64_read_state": (I, [P, F64P, F64P, F64P, U32, U32P]),
    "mpm_sim64_grid_totals": (I, [P, F64P]),
    "mpm_sim64_read_status": (I, [P, C.POINTER(mpm_status_info)]),
    "mpm_server_create": (I, [P, U64, U32, PP]),
    "mpm_server_destroy": (I, [P]),
    "mpm_server_submit": (I, [P, C.POINTER(mpm_config), C.POINTER(mpm_rheology), U32, F32P, U32P, U32, C.c_float,
                              U32, U64P]),
    "mpm_server_run": (I, [P, U32, U32]),
    "mpm_server_poll": (I, [P, U64, U32P, F32P, U32, U32P]),
    "mpm_server_stats_get": (I, [P, C.POINTER(mpm_server_stats)]),
    "mpm_server_ticket_status": (I, [P, C.c_uint64, C.POINTER(mpm_status_info)]),
}

_lib = None


def lib():
    """Load libmolla_mpm.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m molla_b200.build` "
                              "(the MPM path has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().mpm_last_error(buf, 1024)
    return buf.value.decode("utf-8", "replace")
