// mpm_b200_ffi.rs — the `extern "C"` declarations of libmolla_mpm.so
// (include/molla_mpm.h) for crates/molla-solvers/src/mpm_b200_ffi.rs.
// MpmSimulation forwards to the first block; the second block holds the
// calls with no MpmSimulation counterpart (groups, serving, autotuning,
// stage timing, the all-FP64 simulation, the allocation-free sort).
// This file cannot be compiled here (no Rust toolchain); the CPU tests
// check that it declares every entry point of the header with its
// argument count.

#![allow(non_camel_case_types)]
use std::os::raw::{c_char, c_int, c_void};

#[repr(C)] pub struct mpm_engine { _p: [u8; 0] }
#[repr(C)] pub struct mpm_sim { _p: [u8; 0] }
#[repr(C)] pub struct mpm_prepared { _p: [u8; 0] }
#[repr(C)] pub struct mpm_batch { _p: [u8; 0] }
#[repr(C)] pub struct mpm_group { _p: [u8; 0] }
#[repr(C)] pub struct mpm_server { _p: [u8; 0] }

#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_rheology {            // MpmRheology (mpm.rs:320-370)
    pub kind: u32,                   // 0 Sand, 1 Snow, 2 Viscous
    pub friction_angle: f32, pub theta_c: f32, pub theta_s: f32, pub hardening: f32,
    pub velocity_damping: f32, pub affine_damping: f32,
    pub youngs: f32, pub poisson: f32, // per-row modulus (0 = the config's)
}

#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_config {              // MpmConfig (mpm.rs:400-433) + extensions
    pub grid_size: u32, pub cell_size: f32, pub grid_origin: [f32; 3], pub gravity_y: f32,
    pub youngs: f32, pub poisson: f32, pub friction_angle: f32, pub cohesion: f32,
    pub boundary_friction: f32, pub particle_mass: f32, pub particle_volume: f32,
    pub max_particles: u32, pub max_rigid: u32, pub rheology: mpm_rheology,
    pub time_step: u32, pub jacobi_iters: u32,
    pub boundary_pad: u32, pub walls: u32, pub svd_precision: u32,
    pub grid_window_cells: [i32; 3], pub reserved: [u32; 8],
}

#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_status_info { pub numerical_fault: u32, pub completed_substeps: u32,
                             pub fault_bits: u32, pub active_tiles: u32 }

#[repr(C)] #[derive(Clone, Copy)]
pub struct mpm_render_view {         // MpmParticleRenderView (mpm_render_view.rs:9-13)
    pub positions: *const c_void,    // device float4 per particle, w = 0
    pub count: u32, pub capacity: u32,
    pub source: u64,                 // MpmParticleRenderSource identity
    pub live_position_bytes: u64,
}

#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_sim_info {             // particle_count, uses_two_pass_p2g,
    pub particle_count: u32,          // deterministic_p2g_enabled,
    pub uses_two_pass_p2g: u32,       // particle_tile_ordering_enabled
    pub deterministic_p2g: u32,
    pub deterministic_prepared: u32,
    pub tile_ordering: u32,
    pub tile_ordering_capacity: u32,
    pub sort_interval: u32,
    pub max_particles: u32,
}

extern "C" {
    pub fn mpm_engine_create(device: c_int, out: *mut *mut mpm_engine) -> c_int;
    pub fn mpm_engine_destroy(e: *mut mpm_engine) -> c_int;
    pub fn mpm_engine_check(e: *mut mpm_engine) -> c_int;
    pub fn mpm_engine_synchronize(e: *mut mpm_engine) -> c_int;
    pub fn mpm_config_preset(preset: u32, out: *mut mpm_config) -> c_int;
    pub fn mpm_dp_alpha(friction_angle: f32) -> f32;
    pub fn mpm_sim_create(e: *mut mpm_engine, cfg: *const mpm_config, out: *mut *mut mpm_sim) -> c_int;
    pub fn mpm_sim_create_sparse(e: *mut mpm_engine, cfg: *const mpm_config, tile_capacity: u32,
                                 out: *mut *mut mpm_sim) -> c_int;
    pub fn mpm_sim_destroy(s: *mut mpm_sim) -> c_int;
    pub fn mpm_set_particles(s: *mut mpm_sim, xyz: *const f32, vel_or_null: *const f32, n: u32) -> c_int;
    pub fn mpm_set_materials(s: *mut mpm_sim, rows: *const mpm_rheology, n_rows: u32,
                             ids: *const u32, n: u32) -> c_int;
    pub fn mpm_set_rheology(s: *mut mpm_sim, r: *const mpm_rheology) -> c_int;
    pub fn mpm_set_material(s: *mut mpm_sim, youngs: f32, friction_angle: f32) -> c_int;
    pub fn mpm_set_time_step(s: *mut mpm_sim, kind: u32, jacobi_iters: u32) -> c_int;
    pub fn mpm_set_p2g_mode(s: *mut mpm_sim, two_pass: c_int) -> c_int;
    pub fn mpm_prepare_deterministic_p2g(s: *mut mpm_sim) -> c_int;
    pub fn mpm_set_deterministic_p2g(s: *mut mpm_sim, enabled: c_int) -> c_int;
    pub fn mpm_release_deterministic_p2g(s: *mut mpm_sim) -> c_int;
    pub fn mpm_sim_info_get(s: *mut mpm_sim, out: *mut mpm_sim_info) -> c_int;  // the getters
    pub fn mpm_sim_config(s: *mut mpm_sim, out: *mut mpm_config) -> c_int;      // config()
    pub fn mpm_prepare_particle_tile_ordering(s: *mut mpm_sim, capacity: u32) -> c_int;
    pub fn mpm_set_particle_tile_ordering(s: *mut mpm_sim, enabled: c_int) -> c_int;
    pub fn mpm_set_sort_interval(s: *mut mpm_sim, interval: u32) -> c_int;
    pub fn mpm_step_n(s: *mut mpm_sim, dt: f32, substeps: u32) -> c_int;
    pub fn mpm_prepare_step(s: *mut mpm_sim, dt: f32, substeps: u32, out: *mut *mut mpm_prepared) -> c_int;
    pub fn mpm_prepared_destroy(p: *mut mpm_prepared) -> c_int;
    pub fn mpm_batch_begin(s: *mut mpm_sim, stream: *mut c_void, out: *mut *mut mpm_batch) -> c_int;
    pub fn mpm_batch_encode_step(b: *mut mpm_batch, p: *const mpm_prepared) -> c_int;
    pub fn mpm_batch_submit(b: *mut mpm_batch) -> c_int;
    pub fn mpm_batch_cancel(b: *mut mpm_batch) -> c_int;
    pub fn mpm_read_positions(s: *mut mpm_sim, out: *mut f32, cap: u32, count: *mut u32) -> c_int;
    pub fn mpm_read_velocities(s: *mut mpm_sim, out: *mut f32, cap: u32, count: *mut u32) -> c_int;
    pub fn mpm_particle_render_view(s: *mut mpm_sim, out: *mut mpm_render_view) -> c_int;
    pub fn mpm_read_grid_mass_momentum(s: *mut mpm_sim, mass: *mut f32, momentum: *mut f32,
                                       cells: usize) -> c_int;
    pub fn mpm_read_status(s: *mut mpm_sim, out: *mut mpm_status_info) -> c_int;
    pub fn mpm_reset_fault(s: *mut mpm_sim) -> c_int;
    pub fn mpm_read_sort_permutation(s: *mut mpm_sim, keys: *mut u32, ids: *mut u32, cap: u32) -> c_int;
    pub fn mpm_read_particle_state(s: *mut mpm_sim, c: *mut f32, f: *mut f32, jp: *mut f32,
                                   cap: u32, count: *mut u32) -> c_int;
    pub fn mpm_write_particle_state(s: *mut mpm_sim, c: *const f32, f: *const f32, jp: *const f32,
                                    n: u32) -> c_int;
    pub fn mpm_set_particle_mass_volume(s: *mut mpm_sim, mass_or_null: *const f32,
                                        volume_or_null: *const f32, n: u32) -> c_int;
    pub fn mpm_conservation_totals(s: *mut mpm_sim, out8: *mut f64) -> c_int;
    pub fn mpm_engine_stream(e: *mut mpm_engine) -> *mut c_void;    // the engine's cudaStream_t
    pub fn mpm_engine_launch_count(e: *mut mpm_engine) -> u64;
    pub fn mpm_radix_sort_pairs(e: *mut mpm_engine, keys: *mut u32, values: *mut u32, n: u32,
                                key_bits: u32) -> c_int;            // host arrays
    pub fn mpm_radix_sort_pairs_device(e: *mut mpm_engine, d_keys: *mut u32, d_values: *mut u32, n: u32,
                                       key_bits: u32, stream: *mut c_void) -> c_int;
    pub fn mpm_radix_sort_pairs_noalloc(d_keys: *mut u32, d_values: *mut u32, n: u32, key_bits: u32,
                                        stream: *mut c_void) -> c_int;
    pub fn mpm_set_rigid_spheres(s: *mut mpm_sim, spheres: *const f32, n: u32) -> c_int;  // 7 floats each
    pub fn mpm_read_rigid_wrenches(s: *mut mpm_sim, out: *mut f32, cap: u32, count: *mut u32) -> c_int;
    // soil checkpoints in molla's own byte format (mpm_checkpoint.rs)
    pub fn mpm_checkpoint_save(s: *mut mpm_sim, out: *mut u8, cap: usize, size: *mut usize) -> c_int;
    pub fn mpm_checkpoint_load(s: *mut mpm_sim, bytes: *const u8, len: usize) -> c_int;
    pub fn mpm_checkpoint_reencode(bytes: *const u8, len: usize, max_particles: u32, out: *mut u8,
                                   cap: usize, size: *mut usize, count: *mut u32) -> c_int;
    pub fn mpm_blake3(data: *const c_void, len: usize, out32: *mut u8) -> c_int;
    pub fn mpm_last_error(buf: *mut c_char, size: usize) -> usize;
    pub fn mpm_abi_version() -> u32;
}

#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_profile_stage { pub launches: u64, pub total_ms: f64 }
#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_server_stats {
    pub admitted: u64, pub completed: u64, pub resident_scenes: u64, pub resident_bytes: u64,
    pub particle_steps: u64,
    pub tick_ms_p50: f64, pub tick_ms_p99: f64, pub queue_ms_p50: f64, pub queue_ms_p99: f64,
    pub admit_ms: f64, pub step_ms: f64, pub retire_ms: f64, pub ticks: u64, pub faulted: u64,
    pub graph_builds: u64, pub graph_build_ms: f64,
}
#[repr(C)] pub struct mpm_sim64 { _p: [u8; 0] }
#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_shapes {
    pub sort_interval: u32, pub item_particles: u32, pub fused: u32,
    pub gather_ctas_per_sm: u32, pub scatter_ctas_per_sm: u32, pub reserved: [u32; 3],
}
#[repr(C)] #[derive(Clone, Copy, Default)]
pub struct mpm_tune_probe { pub knob: u32, pub value: u32, pub ms_per_substep: f32 }

extern "C" {
    // regroup-interval autotune and per-stage timing
    pub fn mpm_autotune(s: *mut mpm_sim, dt: f32, probe_substeps: u32, candidates: *const u32,
                        n_candidates: u32, ms_per_substep: *mut f32, chosen: *mut u32) -> c_int;
    pub fn mpm_profile_enable(e: *mut mpm_engine, enabled: c_int) -> c_int;
    pub fn mpm_profile_read(e: *mut mpm_engine, out: *mut mpm_profile_stage, cap: u32) -> c_int;
    pub fn mpm_profile_reset(e: *mut mpm_engine) -> c_int;
    // failure detection: the scatter's bounded-wait timeout path, run on purpose
    pub fn mpm_selftest_device_wait(e: *mut mpm_engine, fault_bits: *mut u32, waited_ms: *mut f64) -> c_int;
    // many scenes in the same launches
    pub fn mpm_group_create(e: *mut mpm_engine, max_scenes: u32, max_particles_total: u64,
                            max_cells_total: u64, out: *mut *mut mpm_group) -> c_int;
    pub fn mpm_group_destroy(g: *mut mpm_group) -> c_int;
    pub fn mpm_group_add_scene(g: *mut mpm_group, cfg: *const mpm_config, rows: *const mpm_rheology,
                               n_rows: u32, xyz: *const f32, ids_or_null: *const u32, n: u32, dt: f32,
                               scene_id: *mut u32) -> c_int;
    pub fn mpm_group_add_scene_sparse(g: *mut mpm_group, cfg: *const mpm_config, rows: *const mpm_rheology,
                                      n_rows: u32, xyz: *const f32, ids_or_null: *const u32, n: u32, dt: f32,
                                      tile_capacity: u32, scene_id: *mut u32) -> c_int;
    pub fn mpm_group_remove_scene(g: *mut mpm_group, scene_id: u32) -> c_int;
    pub fn mpm_group_step(g: *mut mpm_group, substeps: u32) -> c_int;
    pub fn mpm_group_step_graph(g: *mut mpm_group, substeps: u32, repeat: u32) -> c_int;
    pub fn mpm_group_read_positions(g: *mut mpm_group, scene_id: u32, out: *mut f32, cap: u32,
                                    count: *mut u32) -> c_int;
    pub fn mpm_group_read_status(g: *mut mpm_group, scene_id: u32, out: *mut mpm_status_info) -> c_int;
    pub fn mpm_group_autotune(g: *mut mpm_group, probe_substeps: u32, candidates: *const u32,
                              n_candidates: u32, ms_per_substep: *mut f32, chosen: *mut u32) -> c_int;
    pub fn mpm_group_set_deterministic(g: *mut mpm_group, enabled: c_int) -> c_int;
    pub fn mpm_group_scene_count(g: *mut mpm_group, count: *mut u32) -> c_int;
    pub fn mpm_group_tune(g: *mut mpm_group, chunk: u32, sort_interval: u32) -> c_int;
    // launch and tile shapes: autotuned on a snapshot, or set directly
    pub fn mpm_group_autotune_shapes(g: *mut mpm_group, probe_substeps: u32, chosen: *mut mpm_shapes,
                                     probes: *mut mpm_tune_probe, cap: u32, n_probes: *mut u32) -> c_int;
    pub fn mpm_autotune_shapes(s: *mut mpm_sim, dt: f32, probe_substeps: u32, chosen: *mut mpm_shapes,
                               probes: *mut mpm_tune_probe, cap: u32, n_probes: *mut u32) -> c_int;
    pub fn mpm_group_get_shapes(g: *mut mpm_group, out: *mut mpm_shapes) -> c_int;
    pub fn mpm_group_set_shapes(g: *mut mpm_group, shapes: *const mpm_shapes) -> c_int;
    // admission-controlled serving over one group
    pub fn mpm_server_create(e: *mut mpm_engine, hbm_budget_bytes: u64, max_scenes: u32,
                             out: *mut *mut mpm_server) -> c_int;
    pub fn mpm_server_destroy(s: *mut mpm_server) -> c_int;
    pub fn mpm_server_submit(s: *mut mpm_server, cfg: *const mpm_config, rows: *const mpm_rheology,
                             n_rows: u32, xyz: *const f32, ids_or_null: *const u32, n: u32, dt: f32,
                             steps: u32, ticket: *mut u64) -> c_int;
    pub fn mpm_server_run(s: *mut mpm_server, ticks: u32, substeps_per_tick: u32) -> c_int;
    pub fn mpm_server_poll(s: *mut mpm_server, ticket: u64, state: *mut u32, positions_out: *mut f32,
                           cap: u32, count: *mut u32) -> c_int;
    pub fn mpm_server_stats_get(s: *mut mpm_server, out: *mut mpm_server_stats) -> c_int;
    pub fn mpm_server_ticket_status(s: *mut mpm_server, ticket: u64, out: *mut mpm_status_info) -> c_int;
    // all-FP64 state and grid (precision studies)
    pub fn mpm_sim64_create(e: *mut mpm_engine, cfg: *const mpm_config, out: *mut *mut mpm_sim64) -> c_int;
    pub fn mpm_sim64_destroy(s: *mut mpm_sim64) -> c_int;
    pub fn mpm_sim64_set_particles(s: *mut mpm_sim64, xyz: *const f64, n: u32) -> c_int;
    pub fn mpm_sim64_set_materials(s: *mut mpm_sim64, rows: *const mpm_rheology, n_rows: u32,
                                   ids: *const u32, n: u32) -> c_int;
    pub fn mpm_sim64_step_n(s: *mut mpm_sim64, dt: f64, substeps: u32) -> c_int;
    pub fn mpm_sim64_read_state(s: *mut mpm_sim64, pos: *mut f64, vel: *mut f64, f: *mut f64, cap: u32,
                                count: *mut u32) -> c_int;
    pub fn mpm_sim64_read_status(s: *mut mpm_sim64, out: *mut mpm_status_info) -> c_int;
    pub fn mpm_sim64_grid_totals(s: *mut mpm_sim64, out4: *mut f64) -> c_int;
}
