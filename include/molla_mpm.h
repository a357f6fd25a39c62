/*
 * molla_mpm.h — C ABI of the B200-native explicit MLS-MPM substep.
 *
 * This is the drop-in boundary for molla's MPM solver interface
 * (crates/molla-solvers/src/lib.rs:180-199 re-exports MpmSimulation,
 * MpmConfig, MpmRheology, MpmTimeStep, PreparedMpmStep, MpmCommandBatch).
 * A Rust `extern "C"` crate binds these symbols one to one; every entry point
 * below names the reference item it replaces (path:line inside the molla
 * repository).  Plain pointers and sizes only: host arrays are borrowed for
 * the duration of the call, device memory is owned by the library.
 *
 * Errors: every function returns an mpm_status code (0 = MPM_OK).  The text
 * of the last error on the calling thread is available from mpm_last_error
 * (the Display string of molla_core::Error, crates/molla-core/src/error.rs:9-40).
 *
 * Threading: one thread at a time per simulation/batch/server object, as the
 * reference's `&mut self` receivers require.  Different objects may be used
 * from different threads.
 */
#ifndef MOLLA_MPM_H
#define MOLLA_MPM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MPM_API __attribute__((visibility("default")))
#else
#define MPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MOLLA_MPM_ABI_VERSION 1u

/* Status codes.  MPM_ERR_INVALID mirrors Error::Solver (invalid input or
 * state), MPM_ERR_GPU mirrors Error::Gpu (device problems), MPM_ERR_FAULT is
 * a latched numerical fault (mpm.rs:1397-1427), MPM_ERR_STALE a prepared step
 * from another simulation or configuration (mpm_command_batch.rs:169-176). */
typedef enum mpm_status {
  MPM_OK = 0,
  MPM_ERR_INVALID = 1,
  MPM_ERR_GPU = 2,
  MPM_ERR_FAULT = 3,
  MPM_ERR_STALE = 4,
  MPM_ERR_NOMEM = 5,
  MPM_ERR_UNSUPPORTED = 6,
  MPM_ERR_BUSY = 7
} mpm_status;

/* Rheology kinds, MpmRheology (crates/molla-solvers/src/mpm.rs:320-370). */
typedef enum mpm_rheology_kind {
  MPM_RHEOLOGY_SAND = 0,
  MPM_RHEOLOGY_SNOW = 1,
  MPM_RHEOLOGY_VISCOUS = 2
} mpm_rheology_kind;

/* One material row.  Sand uses friction_angle (radians); snow uses theta_c,
 * theta_s, hardening; viscous uses velocity_damping, affine_damping (1/s).
 * youngs/poisson > 0 give this row its own elastic moduli — an extension for
 * scenes that mix stiffnesses; 0 keeps the simulation-wide values, which is
 * the reference behaviour (mpm.wgsl:98-99 has global E and nu only). */
typedef struct mpm_rheology {
  uint32_t kind;
  float friction_angle;
  float theta_c;
  float theta_s;
  float hardening;
  float velocity_damping;
  float affine_damping;
  float youngs;
  float poisson;
} mpm_rheology;

/* Time-step selector, MpmTimeStep (mpm.rs:372-398).  IMPLICIT adds
 * `jacobi_iters` semi-implicit Jacobi sweeps on the grid velocity after the
 * grid update (mpm_implicit_apply, mpm.wgsl:1060-1164); rigid-body coupling
 * is not part of this path. */
typedef enum mpm_time_step_kind { MPM_TIME_STEP_EXPLICIT = 0, MPM_TIME_STEP_IMPLICIT = 1 } mpm_time_step_kind;

/* Precision of the per-particle SVD/polar decomposition.  The particle and
 * grid state is FP32 in both cases. */
typedef enum mpm_svd_precision { MPM_SVD_FP32 = 0, MPM_SVD_FP64 = 1 } mpm_svd_precision;

/* Wall models.  MPM_WALLS_REFERENCE: the reference's pad-2 one-sided normal
 * clamp with tangential friction (mpm.wgsl:1044-1056).  MPM_WALLS_STICKY:
 * extension, every velocity component is zeroed inside the pad layer. */
typedef enum mpm_wall_kind { MPM_WALLS_REFERENCE = 0, MPM_WALLS_STICKY = 1 } mpm_wall_kind;

/* MpmConfig (crates/molla-solvers/src/mpm.rs:400-433) plus extensions.
 * Fields after `jacobi_iters` are extensions; zero-initialised they select the
 * reference behaviour (pad 2, reference walls, FP32 SVD, window 0). */
typedef struct mpm_config {
  uint32_t grid_size;
  float cell_size;
  float grid_origin[3];
  float gravity_y;
  float youngs;
  float poisson;
  float friction_angle;
  float cohesion;
  float boundary_friction;
  float particle_mass;
  float particle_volume;
  uint32_t max_particles;
  uint32_t max_rigid;
  mpm_rheology rheology;
  uint32_t time_step;    /* mpm_time_step_kind */
  uint32_t jacobi_iters; /* MpmTimeStep::Implicit */
  /* extensions */
  uint32_t boundary_pad; /* 0 → 2 */
  uint32_t walls;        /* mpm_wall_kind */
  uint32_t svd_precision;/* mpm_svd_precision */
  int32_t grid_window_cells[3];
  uint32_t reserved[8];
} mpm_config;

/* Presets MpmConfig::{sand, sand_calibrated, snow, viscous}
 * (mpm.rs:540-655). */
typedef enum mpm_preset {
  MPM_PRESET_SAND = 0,
  MPM_PRESET_SAND_CALIBRATED = 1,
  MPM_PRESET_SNOW = 2,
  MPM_PRESET_VISCOUS = 3
} mpm_preset;

/* Fault/status word, MpmActiveGridStats (mpm.rs:257-283). */
typedef struct mpm_status_info {
  uint32_t numerical_fault;   /* latched non-finite state (mpm.wgsl:217-231) */
  uint32_t completed_substeps;/* gathers run since the last fault reset (mpm.wgsl:1246) */
  uint32_t fault_bits;        /* raw latch word: 2 numerical fault, 4 a deposit left the fixed
                                 order, 8 a bounded device wait gave up, 16 sparse tile overflow */
  uint32_t active_tiles;      /* sparse grid storage: tiles of the current map (0 when dense) */
} mpm_status_info;

/* Opaque handles. */
typedef struct mpm_engine mpm_engine;
typedef struct mpm_sim mpm_sim;
typedef struct mpm_prepared mpm_prepared;
typedef struct mpm_batch mpm_batch;
typedef struct mpm_group mpm_group;
typedef struct mpm_server mpm_server;

/* ---- engine ---------------------------------------------------------- */

/* Engine::new_gpu (crates/molla-compute/src/engine.rs:140): binds a CUDA
 * device and creates the engine's stream.  `device` is the CUDA ordinal. */
MPM_API int mpm_engine_create(int device, mpm_engine** out);
/* Drops the caller's engine handle.  Simulations, groups and servers created
 * from it keep the device stream alive until they are destroyed, so they may
 * outlive the handle. */
MPM_API int mpm_engine_destroy(mpm_engine* engine);
/* Engine::check_device / DeviceHealth (engine.rs:70-119): MPM_ERR_GPU once a
 * device error was observed on this engine (sticky). */
MPM_API int mpm_engine_check(mpm_engine* engine);
/* Synchronise the engine's stream (the reference's device.poll(wait)). */
MPM_API int mpm_engine_synchronize(mpm_engine* engine);
/* The engine's cudaStream_t (every simulation of the engine launches on it),
 * for callers that order their own work or CUDA events against it. */
MPM_API void* mpm_engine_stream(mpm_engine* engine);

/* ---- configuration ----------------------------------------------------- */

/* MpmConfig::{sand, sand_calibrated, snow, viscous} (mpm.rs:540-655). */
MPM_API int mpm_config_preset(uint32_t preset, mpm_config* out);
/* Host-side Drucker-Prager alpha of a material row, material_row
 * (mpm.rs:662-686): sqrt(2/3)*2 sin(phi)/(3 - sin(phi)). */
MPM_API float mpm_dp_alpha(float friction_angle);

/* ---- simulation -------------------------------------------------------- */

/* MpmSimulation::new (mpm.rs:834-843, validation :855-900). */
MPM_API int mpm_sim_create(mpm_engine* engine, const mpm_config* cfg, mpm_sim** out);
/* MpmSimulation::new_sparse (mpm.rs:846-853): grid storage for
 * `tile_capacity` tiles of 4^3 nodes instead of grid_size^3 nodes
 * (1 <= tile_capacity <= ceil(grid_size / 4)^3).  Every substep the tiles the
 * particles' stencils touch get slots; more than tile_capacity of them latch
 * the tile-overflow bit (16) in the status word, and the scene freezes as on
 * a numerical fault (MpmActiveGridStats::overflow, mpm.rs:257-283).  Results
 * equal the dense storage's.  Explicit time step only; rigid spheres are not
 * coupled to sparse storage (MPM_ERR_UNSUPPORTED). */
MPM_API int mpm_sim_create_sparse(mpm_engine* engine, const mpm_config* cfg, uint32_t tile_capacity,
                                  mpm_sim** out);
MPM_API int mpm_sim_destroy(mpm_sim* sim);

/* set_particles / set_particles_with_velocity (mpm.rs:1451-1519):
 * positions xyz[3n]; velocities vel[3n] or NULL (rest).  F = I, C = 0,
 * jp = 0, mass/volume from the config.  n > max_particles → MPM_ERR_INVALID. */
MPM_API int mpm_set_particles(mpm_sim* sim, const float* xyz, const float* vel_or_null, uint32_t n);

/* Extension of set_particles for scenes with per-particle mass/volume
 * (NULL keeps the config value for every particle). */
MPM_API int mpm_set_particle_mass_volume(mpm_sim* sim, const float* mass_or_null, const float* volume_or_null,
                                 uint32_t n);

/* set_materials (mpm.rs:1589-1621): 1..8 rows, ids[n] < rows, n must equal
 * the particle count. */
MPM_API int mpm_set_materials(mpm_sim* sim, const mpm_rheology* rows, uint32_t n_rows, const uint32_t* ids, uint32_t n);
/* set_rheology (mpm.rs:1623-1629). */
MPM_API int mpm_set_rheology(mpm_sim* sim, const mpm_rheology* rheology);
/* set_material (mpm.rs:1578-1587): live Young's modulus and friction angle. */
MPM_API int mpm_set_material(mpm_sim* sim, float youngs, float friction_angle);
/* set_time_step (mpm.rs:1631-1635). */
MPM_API int mpm_set_time_step(mpm_sim* sim, uint32_t kind, uint32_t jacobi_iters);

/* set_p2g_mode (mpm.rs:1642-1650).  Both reference modes map to the same
 * tile-accumulated scatter here; the flag is kept for API parity.  As in the
 * reference it also turns deterministic P2G off and makes prepared steps
 * stale. */
MPM_API int mpm_set_p2g_mode(mpm_sim* sim, int two_pass);
/* prepare_deterministic_p2g / set_deterministic_p2g
 * (mpm_deterministic_p2g.rs:419-569): fixed-order P2G over particles
 * regrouped by tile after every gather; results are bit-repeatable.
 * Enabling requires a prepare call and enabled particle ordering (as the
 * reference).  A deposit that left the fixed order (positions set outside
 * the grid) sets bit 4 of the status word. */
MPM_API int mpm_prepare_deterministic_p2g(mpm_sim* sim);
MPM_API int mpm_set_deterministic_p2g(mpm_sim* sim, int enabled);
/* release_deterministic_p2g (mpm_deterministic_p2g.rs:606-617): forgets the
 * prepare call (particle ordering stays); refused with MPM_ERR_INVALID while
 * deterministic P2G is enabled.  Prepared steps go stale if it was prepared. */
MPM_API int mpm_release_deterministic_p2g(mpm_sim* sim);

/* The switches and counts the reference's getters return. */
typedef struct mpm_sim_info {
  uint32_t particle_count;          /* particle_count (mpm.rs:1250-1252) */
  uint32_t uses_two_pass_p2g;       /* uses_two_pass_p2g (mpm.rs:1689-1694): the
                                       set_p2g_mode flag (default 1), 0 while
                                       deterministic P2G is enabled */
  uint32_t deterministic_p2g;       /* deterministic_p2g_enabled
                                       (mpm_deterministic_p2g.rs:571-573) */
  uint32_t deterministic_prepared;  /* prepared and not released */
  uint32_t tile_ordering;           /* particle_tile_ordering_enabled
                                       (mpm_particle_order.rs:265-267) */
  uint32_t tile_ordering_capacity;  /* prepared capacity, 0 if never prepared */
  uint32_t sort_interval;           /* regroup interval in effect (substeps) */
  uint32_t max_particles;           /* capacity fixed at creation */
} mpm_sim_info;
MPM_API int mpm_sim_info_get(mpm_sim* sim, mpm_sim_info* out);
/* config (mpm.rs:1245-1247): the configuration with every later setter
 * (rheology, material, time step) applied. */
MPM_API int mpm_sim_config(mpm_sim* sim, mpm_config* out);

/* prepare_particle_tile_ordering (mpm_particle_order.rs:161-230): capacity in
 * 1..=max_particles and >= the live count. */
MPM_API int mpm_prepare_particle_tile_ordering(mpm_sim* sim, uint32_t capacity);
/* set_particle_tile_ordering (mpm_particle_order.rs:232-252). */
MPM_API int mpm_set_particle_tile_ordering(mpm_sim* sim, int enabled);
/* Sort interval of the hot path: particles are physically regrouped by 4^3
 * tile every `interval` substeps (0 → autotuned default).  The cadence runs
 * across step_n calls (it does not restart per call); setting the interval
 * starts a new cadence, whose first regrouping opens the next call. */
MPM_API int mpm_set_sort_interval(mpm_sim* sim, uint32_t interval);

/* step / step_n (mpm.rs:2232-2353): asynchronous; dt finite and > 0. */
MPM_API int mpm_step_n(mpm_sim* sim, float dt, uint32_t substeps);

/* prepare_step (mpm_command_batch.rs:36-140): freezes dt, substeps, material
 * table and sort parameters; the substep sequence is captured once as a CUDA
 * graph.  A later configuration change makes the record stale. */
MPM_API int mpm_prepare_step(mpm_sim* sim, float dt, uint32_t substeps, mpm_prepared** out);
MPM_API int mpm_prepared_destroy(mpm_prepared* prepared);
/* begin_command_batch / encode_step / submit (mpm_command_batch.rs:142-218).
 * `stream` is a caller-owned cudaStream_t (NULL: the engine's stream); encode
 * launches the prepared graph on it, submit records completion. */
MPM_API int mpm_batch_begin(mpm_sim* sim, void* stream, mpm_batch** out);
MPM_API int mpm_batch_encode_step(mpm_batch* batch, const mpm_prepared* prepared);
MPM_API int mpm_batch_submit(mpm_batch* batch);
MPM_API int mpm_batch_cancel(mpm_batch* batch);

/* set_rigid_spheres (mpm.rs:1521-1565): n <= max_rigid (and <= 8) spheres
 * of 7 floats each (center xyz, radius, velocity xyz), replacing the
 * previous set; kept across set_particles.  Each substep, grid nodes inside
 * a sphere take its velocity with the heavy-cell mass 1e6 (rigid_imprint,
 * mpm.wgsl:939-1003) and sand nodes within radius + dx react on it
 * (mpm_rigid_force_integrate, :1175-1228). */
MPM_API int mpm_set_rigid_spheres(mpm_sim* sim, const float* spheres, uint32_t n);
/* read_rigid_wrenches (mpm.rs:2809, 2908-2956): blocking; out[6 * i] =
 * force xyz, torque xyz on sphere i during the last substep. */
MPM_API int mpm_read_rigid_wrenches(mpm_sim* sim, float* out, uint32_t cap, uint32_t* count_out);
/* read_positions / read_velocities (mpm.rs:2718-2798): blocking; writes
 * min(count, cap) rows of 3 floats in the original particle order and
 * stores the particle count in *count_out.  `out` may be pinned host memory
 * (the device-to-host copy is then direct).  Velocities (and C) are those of
 * the last substep of the last step call; after a numerical fault latched in
 * the middle of a call they may be those of the previous call's end. */
MPM_API int mpm_read_positions(mpm_sim* sim, float* out, uint32_t cap, uint32_t* count_out);
/* particle_render_view (crates/molla-solvers/src/mpm_render_view.rs:20-44):
 * live read-only rendering input on the simulation's device.  `positions`
 * is a device buffer of float4 per particle (xyz in world metres, w = 0,
 * 16-byte stride, original particle order); only the first `count` entries
 * are live.  The buffer is the simulation's own and is re-packed on the
 * engine's stream after every step, command batch and set_particles, so a
 * draw queued on that stream after the physics sees that state.  The first
 * call allocates capacity (max_particles) float4 and packs once; later calls
 * allocate, launch and copy nothing.  `source` identifies the buffer
 * (MpmParticleRenderSource): it stays the same across steps and reseeds of
 * this simulation and differs between simulations.  Do not write to the
 * buffer; it is freed with the simulation. */
typedef struct mpm_render_view {
  const void* positions;
  uint32_t count;
  uint32_t capacity;
  uint64_t source;
  uint64_t live_position_bytes;
} mpm_render_view;
MPM_API int mpm_particle_render_view(mpm_sim* sim, mpm_render_view* out);
MPM_API int mpm_read_velocities(mpm_sim* sim, float* out, uint32_t cap, uint32_t* count_out);
/* Full particle state in original order: C[9n], F[9n] column-major, jp[n]
 * (any pointer may be NULL). */
MPM_API int mpm_read_particle_state(mpm_sim* sim, float* C, float* F, float* jp, uint32_t cap, uint32_t* count_out);
/* Overwrite deformation gradients/jp of live particles in original order
 * (checkpoint restore and host-side fault injection; NULL keeps a field). */
MPM_API int mpm_write_particle_state(mpm_sim* sim, const float* C, const float* F, const float* jp, uint32_t n);
/* read_grid_mass_momentum (mpm.rs:2808-2906): grid mass[N^3] and momentum
 * [3 N^3] of the last substep's P2G. */
MPM_API int mpm_read_grid_mass_momentum(mpm_sim* sim, float* mass, float* momentum, size_t cells);
/* Conservation totals accumulated in FP64 on the device:
 * out[0] grid mass, out[1..3] grid momentum, out[4] particle mass,
 * out[5..7] particle momentum. */
MPM_API int mpm_conservation_totals(mpm_sim* sim, double* out8);

/* read_active_grid_status_with (mpm.rs:1418-1427). */
MPM_API int mpm_read_status(mpm_sim* sim, mpm_status_info* out);
/* reset_active_grid (mpm.rs:1387-1390): clears the latch and counters. */
MPM_API int mpm_reset_fault(mpm_sim* sim);

/* ParticleOrder::encode + readback (mpm_particle_order.rs:118-150): computes
 * tile keys for the current positions and sorts (key, identity) stably over
 * `capacity` entries; identities past the live count carry key 0xFFFFFFFF.
 * keys/ids receive capacity entries. */
MPM_API int mpm_read_sort_permutation(mpm_sim* sim, uint32_t* keys, uint32_t* ids, uint32_t capacity);

/* Stable LSD radix sort of (u32 key, u32 value) pairs, RadixSortKernel
 * (crates/molla-compute-primitives/src/radix_sort.rs:50-110).  Host arrays
 * in, sorted in place.  key_bits in 1..32 (passes = ceil(key_bits/8)). */
MPM_API int mpm_radix_sort_pairs(mpm_engine* engine, uint32_t* keys, uint32_t* values, uint32_t n, uint32_t key_bits);

/* Device-pointer form: sorts d_keys/d_values (n entries) on `stream` using
 * library-owned scratch.  Asynchronous. */
MPM_API int mpm_radix_sort_pairs_device(mpm_engine* engine, uint32_t* d_keys, uint32_t* d_values, uint32_t n,
                                uint32_t key_bits, void* stream);

/* Allocation-free variant of mpm_radix_sort_pairs_device; it has no
 * counterpart in the reference.  It is for callers that cannot allocate
 * device memory: code inside a stream-ordered pipeline that must not stall
 * (cudaMalloc/cudaFree can synchronise the device), hosts that reserve the
 * whole device budget up front, and hot paths held to an allocation-free
 * guarantee.  Sorts d_keys/d_values (n pairs, device pointers on the current
 * device) in place on `stream` (NULL: the default stream), stably by the low
 * key_bits bits, using an 8.25 MiB (8,651,776-byte) scratch array that the library keeps in
 * device memory for the whole process (every GPU that loads the library
 * holds one).  n above 1,048,576 is rejected with MPM_ERR_INVALID.  It calls
 * no allocation routine.  The first call on a device looks up the scratch
 * array's address (cudaGetSymbolAddress); make that first call before any
 * stream capture.  All calls share the one scratch array, so calls that
 * overlap on the GPU (different streams, not ordered) race and corrupt each
 * other; order them on one stream or synchronise between them. */
MPM_API int mpm_radix_sort_pairs_noalloc(uint32_t* d_keys, uint32_t* d_values, uint32_t n, uint32_t key_bits,
                                         void* stream);

/* Number of CUDA kernel launches this library issued on the engine since
 * creation (host counter, the equivalent of gpu_metrics::record_dispatch,
 * crates/molla-core/src/gpu_metrics.rs:330-381). */
MPM_API uint64_t mpm_engine_launch_count(mpm_engine* engine);

/* Failure-detection self-test of the scatter's bounded stage wait: one warp
 * waits on a device barrier that nothing completes, gives up after about
 * one second and latches the device-wait bit (8) the way the scatter does.
 * Blocking.  Writes that status word to *fault_bits and the time waited to
 * *waited_ms (may be NULL); the engine stays usable.  The reference's
 * equivalent is its device-health check (molla-core engine.rs:76-119). */
MPM_API int mpm_selftest_device_wait(mpm_engine* engine, uint32_t* fault_bits, double* waited_ms);

/* Per-stage GPU timing, the equivalent of molla's step profiling
 * (prepare_step_profiling / read_step_profile, mpm_profile.rs:542-732):
 * while enabled, each launch of a stage is bracketed by CUDA events on its
 * stream (not inside captured graphs).  Stages: 0 particle ordering (keys,
 * sort, regroup, work list), 1 first-substep stress record (SVD of F),
 * 2 grid update, 3 G2P + F update + return
 * mapping, 4 P2G deposit. */
typedef struct mpm_profile_stage {
  uint64_t launches;
  double total_ms;
} mpm_profile_stage;
MPM_API int mpm_profile_enable(mpm_engine* engine, int enabled);
/* Synchronises, resolves pending events and copies `cap` (<= 5) stages. */
MPM_API int mpm_profile_read(mpm_engine* engine, mpm_profile_stage* out, uint32_t cap);
MPM_API int mpm_profile_reset(mpm_engine* engine);

/* ---- batched scenes ----------------------------------------------------- */

/* A group steps many independent scenes of uneven particle and grid sizes in
 * the same launches (persistent kernels over a (scene, tile) work list).  No
 * reference equivalent; the per-scene numerics are those of mpm_sim. */
MPM_API int mpm_group_create(mpm_engine* engine, uint32_t max_scenes, uint64_t max_particles_total,
                     uint64_t max_cells_total, mpm_group** out);
MPM_API int mpm_group_destroy(mpm_group* group);
/* Adds a scene; returns its id.  Particles xyz[3n] (at rest), one material
 * row per scene plus per-particle material ids (NULL: row 0). */
MPM_API int mpm_group_add_scene(mpm_group* group, const mpm_config* cfg, const mpm_rheology* rows, uint32_t n_rows,
                        const float* xyz, const uint32_t* ids_or_null, uint32_t n, float dt, uint32_t* scene_id);
/* mpm_group_add_scene with sparse grid storage of `tile_capacity` tiles
 * (see mpm_sim_create_sparse); the scene's grid range holds 64 x
 * tile_capacity nodes. */
MPM_API int mpm_group_add_scene_sparse(mpm_group* group, const mpm_config* cfg, const mpm_rheology* rows,
                                       uint32_t n_rows, const float* xyz, const uint32_t* ids_or_null, uint32_t n,
                                       float dt, uint32_t tile_capacity, uint32_t* scene_id);
MPM_API int mpm_group_remove_scene(mpm_group* group, uint32_t scene_id);
/* Advances every scene in the group by `substeps` substeps at its own dt. */
MPM_API int mpm_group_step(mpm_group* group, uint32_t substeps);
/* Captures `substeps` group substeps as a CUDA graph and replays it `repeat`
 * times. */
MPM_API int mpm_group_step_graph(mpm_group* group, uint32_t substeps, uint32_t repeat);
MPM_API int mpm_group_read_positions(mpm_group* group, uint32_t scene_id, float* out, uint32_t cap, uint32_t* count_out);
MPM_API int mpm_group_read_status(mpm_group* group, uint32_t scene_id, mpm_status_info* out);
MPM_API int mpm_group_scene_count(mpm_group* group, uint32_t* count);
/* Fixed-order (deterministic) P2G for every scene of the group: a scene's
 * results are then bit-identical from run to run and alone or in any mix
 * (the group equivalent of mpm_set_deterministic_p2g). */
MPM_API int mpm_group_set_deterministic(mpm_group* group, int enabled);
/* Autotuner: times max(probe_substeps, 2 x candidate) substeps of the group
 * for each candidate regrouping interval (n_candidates values, NULL → {4, 8,
 * 16, 32, 64, 128}) — so every candidate regroups at least twice — on a
 * snapshot of the device state, restores the state (the scenes do not
 * advance) and keeps the fastest interval.  ms_per_substep (may be NULL)
 * receives one timing per candidate; *chosen the interval kept. */
MPM_API int mpm_group_autotune(mpm_group* group, uint32_t probe_substeps, const uint32_t* candidates,
                               uint32_t n_candidates, float* ms_per_substep, uint32_t* chosen);
/* The same for a single simulation (mpm_set_sort_interval is then the
 * tuned value). */
MPM_API int mpm_autotune(mpm_sim* sim, float dt, uint32_t probe_substeps, const uint32_t* candidates,
                         uint32_t n_candidates, float* ms_per_substep, uint32_t* chosen);
/* Group tuning: regroup (sort) interval in substeps (0 → default 32).  The
 * `chunk` argument is reserved (work items are 4^3 tiles of at most 640
 * particles). */
MPM_API int mpm_group_tune(mpm_group* group, uint32_t chunk, uint32_t sort_interval);

/* Launch and tile shapes of the substep (no reference counterpart): the
 * regroup interval, the particles per work item (128..640; a tile with more
 * is cut into several items), whether the non-final substeps run the fused
 * gather + scatter kernel, and the resident gather and scatter CTAs per SM
 * of the persistent kernels (at most their occupancy maxima). */
typedef struct mpm_shapes {
  uint32_t sort_interval;
  uint32_t item_particles;
  uint32_t fused;
  uint32_t gather_ctas_per_sm;
  uint32_t scatter_ctas_per_sm;
  uint32_t reserved[3];
} mpm_shapes;
/* One timing of the shapes autotuner: knob 0 interval, 1 item particles,
 * 2 fused, 3 gather CTAs per SM, 4 scatter CTAs per SM; the value tried and
 * the measured ms per substep. */
typedef struct mpm_tune_probe {
  uint32_t knob;
  uint32_t value;
  float ms_per_substep;
} mpm_tune_probe;
/* Autotuner of the shapes (no reference counterpart): tunes the knobs in the
 * order interval {8,16,32,64}, item particles {640,512,384,256}, fused {0,1},
 * gather CTAs per SM {max, max-1}, scatter CTAs per SM {max, max-1}, each
 * over its candidates with the earlier knobs fixed at their best, timing
 * max(probe_substeps, 2 x interval) substeps per candidate on a snapshot of
 * the device state, which is restored (the scenes do not advance).  Applies
 * and returns the shapes kept; probes (may be NULL) receive up to `cap`
 * timings, *n_probes their count. */
MPM_API int mpm_group_autotune_shapes(mpm_group* group, uint32_t probe_substeps, mpm_shapes* chosen,
                                      mpm_tune_probe* probes, uint32_t cap, uint32_t* n_probes);
/* The same for a single simulation (dt as in mpm_step_n). */
MPM_API int mpm_autotune_shapes(mpm_sim* sim, float dt, uint32_t probe_substeps, mpm_shapes* chosen,
                                mpm_tune_probe* probes, uint32_t cap, uint32_t* n_probes);
/* The shapes in force; setting them marks a regrouping due. */
MPM_API int mpm_group_get_shapes(mpm_group* group, mpm_shapes* out);
MPM_API int mpm_group_set_shapes(mpm_group* group, const mpm_shapes* in);

/* ---- soil checkpoints -------------------------------------------------------
 * The reference's lossless particle checkpoint byte format
 * (crates/molla-solvers/src/mpm_checkpoint.rs:71-92, :187-275): magic
 * "MOLLSOIL", LE u32 version (1, or 2 with a grid window), BLAKE3 digest of
 * the payload, configuration words, material table, then the particle
 * streams (position 4, velocity 4, C 12, F 12, volume, mass, log-Jp,
 * material id, tire compaction 4 words per particle).  Checkpoints written
 * by molla load here and the other way round.  Tire compaction is written
 * as zeros (no tire coupling on this path); per-material Young's modulus
 * and Poisson ratio (an extension) cannot be archived. */
/* checkpoint_soil_with (mpm_checkpoint.rs:388-434): with out == NULL only
 * *size_out is set; otherwise the state is encoded into out[cap].  Blocking.
 * A latched fault is rejected (MPM_ERR_FAULT). */
MPM_API int mpm_checkpoint_save(mpm_sim* sim, uint8_t* out, size_t cap, size_t* size_out);
/* from_bytes + restore_soil_with (mpm_checkpoint.rs:218-275, 436-542):
 * decodes under the simulation's max_particles, rejects corrupt, non-finite,
 * oversized, trailing or incompatible data (the physical configuration must
 * match word for word, capacities aside) and replaces the particle state. */
MPM_API int mpm_checkpoint_load(mpm_sim* sim, const uint8_t* bytes, size_t len);
/* Decodes and validates a checkpoint without a GPU and re-encodes it into
 * out (NULL: only *size_out / *count_out); the encoding is lossless, so the
 * output equals the input for every valid checkpoint. */
MPM_API int mpm_checkpoint_reencode(const uint8_t* bytes, size_t len, uint32_t max_particles, uint8_t* out,
                                    size_t cap, size_t* size_out, uint32_t* count_out);
/* BLAKE3 (unkeyed, 32-byte output) of data[len], the checkpoint digest. */
MPM_API int mpm_blake3(const void* data, size_t len, uint8_t* out32);

/* ---- all-FP64 simulation (precision studies) -------------------------------
 * No reference counterpart as an API: it runs the reference substep
 * (reset, p2g, grid_update, g2p, plasticity; mpm.rs:2476-2551) with FP64
 * particle state, FP64 grid and the FP64 Jacobi SVD (tol 1e-14, 30 sweeps),
 * one GPU thread per particle or node.  It exists to measure the error of
 * the FP32 and FP32 + FP64-SVD modes against an all-FP64 run on the same
 * device; it is not tuned.  Explicit time step only; no groups, graphs or
 * ordering. */
typedef struct mpm_sim64 mpm_sim64;
MPM_API int mpm_sim64_create(mpm_engine* engine, const mpm_config* cfg, mpm_sim64** out);
MPM_API int mpm_sim64_destroy(mpm_sim64* sim);
/* Particles at rest with F = I, C = 0, jp = 0 and the config's mass/volume. */
MPM_API int mpm_sim64_set_particles(mpm_sim64* sim, const double* xyz, uint32_t n);
MPM_API int mpm_sim64_set_materials(mpm_sim64* sim, const mpm_rheology* rows, uint32_t n_rows, const uint32_t* ids,
                                    uint32_t n);
MPM_API int mpm_sim64_step_n(mpm_sim64* sim, double dt, uint32_t substeps);
/* Blocking; any of pos[3n], vel[3n], F[9n] (column-major) may be NULL. */
MPM_API int mpm_sim64_read_state(mpm_sim64* sim, double* pos, double* vel, double* F, uint32_t cap,
                                 uint32_t* count_out);
/* Grid mass and momentum totals of the last P2G: out4 = {m, px, py, pz}. */
MPM_API int mpm_sim64_grid_totals(mpm_sim64* sim, double* out4);
MPM_API int mpm_sim64_read_status(mpm_sim64* sim, mpm_status_info* out);

/* ---- serving ------------------------------------------------------------- */

/* A request loop over a group: scenes are admitted as HBM budget and slots
 * allow, stepped together, and retired when their steps are done. */
MPM_API int mpm_server_create(mpm_engine* engine, uint64_t hbm_budget_bytes, uint32_t max_scenes, mpm_server** out);
MPM_API int mpm_server_destroy(mpm_server* server);
/* Queues a scene for `steps` substeps; returns a ticket. */
MPM_API int mpm_server_submit(mpm_server* server, const mpm_config* cfg, const mpm_rheology* rows, uint32_t n_rows,
                      const float* xyz, const uint32_t* ids_or_null, uint32_t n, float dt, uint32_t steps,
                      uint64_t* ticket);
/* Runs `ticks` scheduling rounds.  A round completes the round before it
 * (waits for its GPU work, retires the scenes that finished in it: their
 * positions are kept for poll, their memory goes back at the next
 * regrouping), admits queued requests in arrival order while the HBM budget
 * allows, and launches one tick of `substeps_per_tick` substeps for every
 * resident scene (each stops on the device after its own step count).  The
 * last round's tick is left running: the call returns while the GPU works,
 * so requests can be submitted meanwhile. */
MPM_API int mpm_server_run(mpm_server* server, uint32_t ticks, uint32_t substeps_per_tick);
/* state: 0 queued, 1 running, 2 done, 3 faulted (the scene's fault latch
 * was set: a non-finite state or a sparse grid out of tiles; it is retired
 * at the first tick that sees it).  When done or faulted, the positions
 * are copied out (for a faulted scene, those frozen at the fault).
 * Completes a tick still running first. */
MPM_API int mpm_server_poll(mpm_server* server, uint64_t ticket, uint32_t* state, float* positions_out, uint32_t cap,
                    uint32_t* count_out);
/* Server statistics: admitted, completed, resident scenes, resident bytes,
 * particle-steps done, and p50/p99 tick latency in milliseconds. */
typedef struct mpm_server_stats {
  uint64_t admitted;
  uint64_t completed;
  uint64_t resident_scenes;
  uint64_t resident_bytes;
  uint64_t particle_steps;
  double tick_ms_p50;
  double tick_ms_p99;
  double queue_ms_p50;
  double queue_ms_p99;
  /* host wall time spent admitting, stepping (launch to completion) and
   * retiring since creation, and the ticks run */
  double admit_ms;
  double step_ms;
  double retire_ms;
  uint64_t ticks;
  /* requests retired as faulted (their particle_steps count only the
   * substeps completed before the fault) */
  uint64_t faulted;
  /* tick graphs captured (a new tick shape, or a layout change since the
   * graph was made) and the host milliseconds spent capturing and
   * instantiating or updating them; the tick latencies above time the
   * graph launches alone */
  uint64_t graph_builds;
  double graph_build_ms;
} mpm_server_stats;
MPM_API int mpm_server_stats_get(mpm_server* server, mpm_server_stats* out);
/* Device status of a finished (done or faulted) request, as it stood when it
 * was retired: fault bits and completed substeps. */
MPM_API int mpm_server_ticket_status(mpm_server* server, uint64_t ticket, mpm_status_info* out);

/* ---- errors ------------------------------------------------------------- */

/* Copies the calling thread's last error message (NUL-terminated, truncated
 * to `size`); returns its full length. */
MPM_API size_t mpm_last_error(char* buf, size_t size);
MPM_API uint32_t mpm_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MOLLA_MPM_H */
