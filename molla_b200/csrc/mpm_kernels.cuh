// mpm_kernels.cuh — host launchers of the substep kernels.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

#include "mpm_device.cuh"

namespace mpm {

constexpr int kParticleThreads = 256;
constexpr int kGatherThreads = 128;
constexpr int kScatterThreads = 192;  // 64 cells x 3 x-slabs of one tile
constexpr int kFusedThreads = 256;    // fused gather + scatter: 2 CTAs per SM (128 registers per thread)
constexpr uint32_t kCellBlock = 256;  // grid pool granularity: one scene per 256-cell block

enum GatherMode : int { kRecord = 0, kG2P = 1, kG2PRecord = 2 };

// publish_all: the gather writes v and C for every particle (a call's last
// substep), not only for scenes whose substep budget ends.
cudaError_t launch_gather(int mode, bool write_keys, bool svd_fp64, const PoolDev& p, double tol, int sweeps,
                          int reuse, int grid, cudaStream_t st, bool publish_all = false);
// The scatter stages its records with TMA through `rec_map`, a 2-D tensor
// map of the record buffer (16 floats x cap, 64-byte swizzle) built by
// make_record_map.
cudaError_t launch_scatter(const PoolDev& p, const CUtensorMap& rec_map, int acc_out, int grid, cudaStream_t st);
// One warp waits (bounded, about one second) on an mbarrier nothing
// completes and reports kFaultDeviceWait: the scatter's timeout path.
cudaError_t launch_selftest_wait(uint32_t* status, unsigned long long* waited_ns, cudaStream_t st);
bool make_record_map(CUtensorMap* out, const float* rec, uint32_t cap, std::string* err);
// Deterministic (fixed-order) scatter: per-tile blocks, then a combine pass.
cudaError_t launch_scatter_det(const PoolDev& p, float4* blocks, int acc_out, int grid, cudaStream_t st);
cudaError_t launch_combine_det(const PoolDev& p, const float4* blocks, const uint32_t* tile_item, uint32_t max_items,
                               int acc_out, cudaStream_t st);
constexpr int kTileNodes = 216;  // 6^3 node footprint of a 4^3-cell tile of base cells
constexpr uint32_t kFaultNondeterministic = 4u;  // a deposit left the fixed-order path
constexpr uint32_t kFaultDeviceWait = 8u;        // a bounded device-side wait gave up (or an item was malformed)
// Particles per scatter item (records staged in shared memory).  640 records
// (41 KB) let k_p2g run 4 CTAs per SM; a full tile at 8 particles per cell is
// 512, so only compressed tiles are cut into two items.
constexpr int kStageMax = 640;
constexpr int kStageBoxRows = 64;                // records per TMA box of the scatter stage
// Persistent grid sizes (SMs x resident CTAs).
int gather_grid_size(bool svd_fp64);
// Fused gather + scatter of a non-final substep (k_g2p2g): gather with the B
// record kept in shared memory, then the record deposit into acc[acc_out].
cudaError_t launch_fused(bool write_keys, bool svd_fp64, const PoolDev& p, double tol, int sweeps, int reuse,
                         int acc_out, int grid, cudaStream_t st);
int fused_grid_size(bool svd_fp64);
int scatter_grid_size();
cudaError_t launch_grid_update(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               int count_substep, cudaStream_t st);
cudaError_t launch_keys(const PoolDev& p, uint32_t n_slots, cudaStream_t st);
cudaError_t launch_init_particles(const PoolDev& p, uint32_t* slot_of, uint32_t slot0, uint32_t id0, uint32_t n,
                                  const float* xyz, const float* vel, const float* mass, const float* vol,
                                  float mass0, float vol0, const uint32_t* mat_ids, uint32_t scene, cudaStream_t st);
cudaError_t launch_set_material_ids(const PoolDev& p, const uint32_t* slot_of, uint32_t id0, uint32_t n,
                                    const uint32_t* ids, cudaStream_t st);
cudaError_t launch_scene_keys(const PoolDev& p, uint32_t sid, const uint32_t* slot_of, uint32_t id0, uint32_t n,
                              uint32_t* keys, cudaStream_t st);
cudaError_t launch_reorder(const float* src, float* dst, uint32_t cap, const uint32_t* meta_src, uint32_t* meta_dst,
                           uint32_t* orig_dst, uint32_t* slot_of, const uint32_t* ids, const uint32_t* keys,
                           uint32_t* slot_key, const float4* rec_src, float4* rec_dst, uint32_t n_live,
                           cudaStream_t st);
// Per item the 64 cells of its tile ranked by particle count at this
// regrouping (descending, ties by cell index): the scatter's lane order.
cudaError_t launch_item_order(const Item* items, const uint32_t* n_items, uint32_t item_top, const uint32_t* slot_key,
                              uint8_t* item_order, cudaStream_t st);
// Semi-implicit Jacobi sweep `sweep` (src -> dst) over the touched blocks.
cudaError_t launch_grid_jacobi(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               const float4* src, float4* dst, uint32_t sweep, cudaStream_t st);
// Rigid-sphere shell reaction over the touched blocks a sphere may reach.
cudaError_t launch_rigid_shell(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               cudaStream_t st);
cudaError_t launch_vel_copy(const uint8_t* touched, const uint32_t* block_scene, uint64_t total_cells,
                            const float4* src, float4* dst, cudaStream_t st);
// Work list of the regrouped particles (see k_items): FP32-SVD items in slots
// [0, n_items[0]), FP64-SVD items in [item_top - n_items[1], item_top).
cudaError_t launch_items(const uint32_t* sorted_keys, int shift, uint32_t n_live, uint32_t K, uint32_t* tile_start,
                         const uint32_t* key_scene, const SceneDev* scenes, uint32_t chunk, uint32_t item_top,
                         Item* items, uint32_t* n_items, uint32_t* tile_item, cudaStream_t st);
// Rebuilds the tile maps of the sparse scenes from the tiles the last gather
// marked (two launches).
cudaError_t launch_tiles_finalize(const PoolDev& p, const uint32_t* key_scene, uint32_t K, uint32_t n_scenes,
                                  cudaStream_t st);
// p[0, n) = v, stream-ordered.
cudaError_t launch_fill_u32(uint32_t* p, uint64_t n, uint32_t v, cudaStream_t st);
cudaError_t launch_pack_positions(const PoolDev& p, const uint32_t* slot_of, uint32_t id_base, uint32_t n,
                                  float4* out, cudaStream_t st);
cudaError_t launch_gather_xyz(const PoolDev& p, int first, const uint32_t* slot_of, uint32_t id_base, uint32_t n,
                              float* out, cudaStream_t st);
cudaError_t launch_gather_rows(const PoolDev& p, int first, int count, const uint32_t* slot_of, uint32_t id_base,
                               uint32_t n, float* out, cudaStream_t st);
cudaError_t launch_scatter_rows(const PoolDev& p, int first, int count, const uint32_t* slot_of, uint32_t id_base,
                                uint32_t n, const float* in, cudaStream_t st);
cudaError_t launch_totals(const PoolDev& p, int acc_idx, uint64_t grid_off, uint64_t cells, const uint32_t* slot_of,
                          uint32_t id_base, uint32_t n, double* out, cudaStream_t st);

}  // namespace mpm
