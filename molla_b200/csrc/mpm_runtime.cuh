// mpm_runtime.cuh — host runtime of the B200 MPM path: engine, scene group
// (pooled particles and grid, regrouping sort, substep sequencing, CUDA-graph
// replay) and the error channel of the C ABI.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/molla_mpm.h"
#include "mpm_device.cuh"
#include "mpm_kernels.cuh"
#include "mpm_sort.cuh"

namespace mpm {

// Error carried to the C ABI: code + message (molla_core::Error's Display).
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what);
#define MPM_CK(expr)                                   \
  do {                                                 \
    cudaError_t _e = (expr);                           \
    if (_e != cudaSuccess) ::mpm::throw_cuda(_e, #expr); \
  } while (0)

// Owned device allocation.
template <class T> struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  DevBuf() = default;
  explicit DevBuf(size_t n) { alloc(n); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void alloc(size_t n) {
    release();
    if (n) {
      cudaError_t e = cudaMalloc((void**)&ptr, n * sizeof(T));
      if (e != cudaSuccess) {
        ptr = nullptr;
        (void)cudaGetLastError();
        throw Error(MPM_ERR_NOMEM, std::string("device allocation of ") + std::to_string(n * sizeof(T)) +
                                       " bytes failed: " + cudaGetErrorString(e));
      }
    }
    count = n;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = 0;
  }
  size_t bytes() const { return count * sizeof(T); }
};

// An owned CUDA event, destroyed on every exit path (errors are thrown).
struct OwnedEvent {
  cudaEvent_t ev = nullptr;
  explicit OwnedEvent(unsigned flags = cudaEventDefault) { MPM_CK(cudaEventCreateWithFlags(&ev, flags)); }
  OwnedEvent(const OwnedEvent&) = delete;
  OwnedEvent& operator=(const OwnedEvent&) = delete;
  ~OwnedEvent() {
    if (ev) cudaEventDestroy(ev);
  }
  operator cudaEvent_t() const { return ev; }
};

// Per-stage GPU timing (the equivalent of molla's MpmProfileStage timestamp
// queries, crates/molla-solvers/src/mpm_profile.rs:8-80): when enabled, each
// launch of a stage is bracketed by CUDA events on the launching stream.
enum Stage : int {
  kStageOrdering = 0,  // keys, sorts, regroup, work list
  kStageRecord = 1,    // first-substep stress record (SVD of F)
  kStageGrid = 2,      // grid update
  kStageGather = 3,    // G2P + F update + return mapping (+ record)
  kStageScatter = 4,   // P2G deposit
  kStages = 5
};

struct ProfRec {
  int stage;
  cudaEvent_t a, b;
};

struct Engine {
  int device = 0;
  bool profiling = false;
  bool capturing = false;
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> event_pool;
  double prof_ms[kStages] = {0, 0, 0, 0, 0};
  uint64_t prof_count[kStages] = {0, 0, 0, 0, 0};
  cudaEvent_t take_event();
  void prof_begin(int stage, cudaStream_t st, ProfRec* r);
  void prof_end(ProfRec* r, cudaStream_t st);
  void prof_resolve();
  cudaStream_t stream = nullptr;
  bool lost = false;
  std::string lost_reason;
  uint64_t launches = 0;
  int sms = 148;
  // scratch of the generic sort entry points
  DevBuf<uint32_t> sk[2], sv[2], shist, skin, svin;
  explicit Engine(int dev);
  ~Engine();
  void check() const;
  void note_error(cudaError_t e);
};

// Host-side description of one scene in a group.
struct SceneHost {
  bool live = false;
  mpm_config cfg{};
  std::vector<mpm_rheology> rows;  // material table (>= 1 row)
  float dt = 0.f;
  uint32_t n = 0;          // particles
  uint32_t id_base = 0;    // identity range
  uint64_t grid_off = 0;   // grid pool range
  uint64_t grid_len = 0;
  uint32_t key_off = 0;
  uint32_t tiles = 0;      // w^3
  uint32_t n_rigid = 0;    // rigid spheres set on this scene
  bool retiring = false;   // retired, its particles not yet compacted out (the slot is not reusable)
  uint32_t tile_cap = 0;   // sparse grid storage: tiles of 4^3 nodes held (0: dense n^3)
};

struct Range {
  uint64_t off, len;
};

// First-fit range allocator over [0, capacity).
struct RangeAlloc {
  uint64_t capacity = 0;
  std::vector<Range> free_list;
  void init(uint64_t cap) {
    capacity = cap;
    free_list.clear();
    if (cap) free_list.push_back({0, cap});
  }
  bool alloc(uint64_t len, uint64_t align, uint64_t* off);
  void release(uint64_t off, uint64_t len);
  uint64_t high_water() const;  // one past the last allocated unit
};

// Build the device record of a scene from its configuration (f32 constants
// computed exactly as the reference host/shader do, see mpm_runtime.cu).
SceneDev make_scene_dev(const mpm_config& cfg, const std::vector<mpm_rheology>& rows, float dt);
float dp_alpha_of(float friction_angle);

// A group of independent scenes stepped by shared launches.
class Group {
 public:
  Group(Engine* e, uint32_t max_scenes, uint64_t particle_cap, uint64_t cell_cap);
  ~Group();

  Engine* eng;
  cudaStream_t stream;

  // capacities
  uint32_t max_scenes;
  uint32_t cap;           // particle slots == identity space
  uint64_t cell_cap;

  // particle pool (double-buffered for the regroup)
  DevBuf<float> planes[2];
  DevBuf<float> rec[2];  // per-slot scatter record, 16 floats (64 B) per slot (rec[1]: deterministic mode)
  CUtensorMap rec_map[2];  // TMA maps of rec[0], rec[1] for the scatter stage
  int rec_cur = 0;
  DevBuf<uint32_t> meta[2], orig[2];
  DevBuf<uint32_t> slot_of, keys_by_id, slot_key, ks[2], vs[2], hist;
  // grid pool
  DevBuf<float4> acc[2], vel;
  DevBuf<float4> vel2;  // semi-implicit Jacobi ping-pong (allocated when a scene needs it)
  // Device side of host uploads and readbacks, grown on demand and kept: a
  // per-call allocation would cost a cudaMalloc and a device-synchronising
  // cudaFree of up to ~36 bytes per particle on every set_particles / read.
  // Every user synchronises the stream before returning, so one buffer
  // serves them all.
  DevBuf<unsigned char> staging;
  unsigned char* staging_bytes(size_t bytes);
  DevBuf<uint8_t> rigid_blocks;  // per 256-cell block: a rigid sphere may reach it
  DevBuf<RigidDev> rigid_d;      // kMaxRigid per scene
  DevBuf<float> wrench_d;        // 8 floats per sphere slot
  DevBuf<uint8_t> touched[2];  // per 256-cell block: acc[i] is nonzero there
  DevBuf<uint32_t> block_scene;
  // scenes
  DevBuf<SceneDev> scenes_d;
  DevBuf<uint32_t> status_d;
  DevBuf<uint32_t> tile_start, n_items;
  // Scene of every tile key (0xffffffff: no live scene).  Each scene holds a
  // stable range of the key space (allocated from `keyr` when it is added),
  // so adding or retiring a scene re-keys no other scene.
  DevBuf<uint32_t> key_scene;
  // Sparse grid storage (scenes added with a tile capacity): slot of every
  // tile key, tile of every slot (by grid pool cell / 64), and the tiles the
  // last gather marked.
  DevBuf<uint32_t> tile_slot, slot_tile;
  DevBuf<uint8_t> tile_mark;
  DevBuf<uint32_t> work_d;  // item counters of the gather and the scatter (PoolDev::work)
  bool any_sparse() const;
  void finalize_tiles(cudaStream_t st);
  DevBuf<Item> items;
  DevBuf<uint8_t> item_order;  // scatter lane order, 64 cells per item
  DevBuf<uint32_t> tile_item;  // deterministic mode: item of each occupied tile
  DevBuf<float4> det_blocks;   // deterministic mode: per-tile 6^3 node blocks
  DevBuf<double> totals_d;
  // pinned staging of scene records
  SceneDev* scenes_h = nullptr;

  std::vector<SceneHost> scenes;
  RangeAlloc ids, cells, keyr;
  uint32_t n_live = 0;
  uint32_t key_space = 0;  // one past the highest allocated tile key
  int cur = 0;       // current particle buffer
  int acc_zero = 0;  // accumulator known to be all zero
  int acc_last = 1;  // accumulator holding the last scatter
  bool need_regroup = true;
  // The scatter records in rec[rec_cur] belong to the current state: the
  // last call ended with a gather that wrote them, and nothing on the host
  // has changed the particles, their materials or their scenes since.  The
  // next call then starts with its scatter instead of a record-only gather
  // (which recomputes every particle's SVD and stress).  Cleared by every
  // host-side change of state and never set in deterministic mode.
  bool records_valid = false;
  bool scenes_dirty = true;
  bool keys_dirty = true;  // scene key offsets changed
  uint32_t sort_interval = 32;
  // Substeps since the last regrouping, carried across calls: the cadence
  // does not depend on how a caller cuts its stepping into step_n calls (a
  // regrouping that falls due on a call's last substep opens the next call).
  uint32_t since = 0;
  uint64_t regroups = 0;  // regroupings issued (device work enqueued or replayed)
  uint32_t chunk = 512;
  // Item slots of the work list: FP32-SVD items fill [0, n32), FP64-SVD items
  // [item_top - n64, item_top) (see k_items).
  uint32_t item_top = 0;
  // Scenes retired by retire_scene and not yet compacted out of the pool:
  // their particles keep their slots (the kernels skip them) until the next
  // regrouping, which sorts them behind every live particle and drops them.
  std::vector<uint32_t> retiring;
  uint32_t n_retiring = 0;    // their particles
  bool compact_issued = false;  // a regrouping that drops them was enqueued
  bool deterministic = false;
  bool reuse_svd = true;
  double svd_tol32 = 1.0e-7;
  // Jacobi tolerance of the mixed-precision SVD, on the off-diagonal of the
  // shifted A' = F^T F - I.  F is FP32 (ulp 6e-8 near 1), so entries of A'
  // below ~3e-8 are the quantisation noise of F itself: rotating them away
  // buys no accuracy (the precision study against the FP64 oracle is
  // unchanged from 1e-9) and cost up to two extra rotations per particle.
  double svd_tol64 = 3.0e-8;
  int svd_sweeps = 16;
  // Fused gather + scatter for the non-final substeps of the atomic P2G
  // (k_g2p2g): -1 picks it for groups of at most kFusedMaxParticles live
  // particles, 1 always, 0 never (MOLLA_MPM_FUSED=1 / 0 in the environment
  // at construction).  Measured on a B200 with the current separate
  // scatter: even at 133k particles, -2% at 1M, -8% at 16M, where the
  // separate kernels' higher occupancy (4 CTAs per SM each against 2) hides
  // the per-item barriers better than the fusion saves.
  int fused_mode = -1;
  static constexpr uint32_t kFusedMaxParticles = 262144;
  bool use_fused() const {
    // the fused kernel deposits an item before the other items are gathered,
    // so a sparse scene's tile map (built from all of them) cannot precede it
    return !deterministic && !any_sparse() &&
           (fused_mode > 0 || (fused_mode < 0 && n_live <= kFusedMaxParticles));
  }
  // Persistent grids: SMs x resident CTAs per SM.  occ_* are the occupancy
  // maxima of each kernel; the tuned counts (0: the maximum) may be lower.
  int occ_gather32 = 1, occ_gather64 = 1, occ_scatter = 1, occ_fused32 = 1, occ_fused64 = 1;
  uint32_t gather_per_sm = 0, scatter_per_sm = 0;
  int gather_grid(bool f64) const;
  int fused_grid(bool f64) const;
  int scatter_grid() const;
  // Particles per work item (a tile with more is cut into several items):
  // at most kStageMax, the scatter's shared-memory record stage.
  uint32_t item_chunk = kStageMax;
  uint64_t substeps_done = 0;
  uint64_t epoch = 1;  // bumps on every change that invalidates captured graphs

  // graph cache: key -> instantiated graph + its kernel count
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    uint64_t epoch = 0;
  };
  struct GraphKey {
    uint32_t substeps, since, interval, flags;
    bool operator<(const GraphKey& o) const {
      if (substeps != o.substeps) return substeps < o.substeps;
      if (since != o.since) return since < o.since;
      if (interval != o.interval) return interval < o.interval;
      return flags < o.flags;
    }
  };
  std::map<GraphKey, Graph> graphs;

  // tile_cap > 0: sparse grid storage of that many 4^3-node tiles
  // (MpmSimulation::new_sparse, mpm.rs:846-853) instead of the dense n^3 grid.
  uint32_t add_scene(const mpm_config& cfg, const std::vector<mpm_rheology>& rows, const float* xyz,
                     const float* vel, const float* mass, const float* vol, const uint32_t* mat_ids, uint32_t n,
                     float dt, uint32_t tile_cap = 0);
  void remove_scene(uint32_t sid);
  // Retires a scene without touching the rest of the pool: its record is
  // marked dead (the kernels skip its items), its identities get the
  // removed-particle key, and its slots, identities and grid range are given
  // back after the next regrouping has sorted its particles out.
  void retire_scene(uint32_t sid);
  // Stops scene sid after `substeps` more substeps (0: no limit).  The
  // particle kernels skip the scene once its completed-substep count has
  // passed the budget, so a scene advances by exactly that many substeps
  // however long the calls that step the group are.
  void set_scene_budget(uint32_t sid, uint32_t substeps, cudaStream_t st, bool fresh = false);
  // Regroups now if retired scenes await compaction, and gives their
  // slots, identities and grid ranges back.
  void compact(cudaStream_t st);
  // SVD forms present among the live scenes.
  bool any_svd32() const;
  bool any_svd64() const;
  void set_scene_dt(uint32_t sid, float dt);
  void set_scene_rows(uint32_t sid, const std::vector<mpm_rheology>& rows);
  void set_scene_cfg(uint32_t sid, const mpm_config& cfg);
  // set_rigid_spheres (mpm.rs:1521-1565): n spheres of 7 floats (center xyz,
  // radius, velocity xyz) for scene sid; replaces the previous set.
  void set_scene_rigid(uint32_t sid, const float* spheres, uint32_t n, cudaStream_t st);
  // read_rigid_wrenches (mpm.rs:2908-2956): force xyz, torque xyz per sphere
  // of the last substep.
  void read_scene_wrench(uint32_t sid, float* out6, uint32_t n, cudaStream_t st);
  bool any_rigid() const;
  void set_material_ids(uint32_t sid, const uint32_t* ids, uint32_t n);

  // Enqueue `substeps` substeps of every live scene on `st`.
  void step(uint32_t substeps, cudaStream_t st);
  // Same through a cached CUDA graph.
  // ev_begin / ev_end (optional) are recorded right before the first graph
  // launch and after the last, so that they time the device work alone
  // (not a capture that precedes it).
  void step_graph(uint32_t substeps, uint32_t repeat, cudaStream_t st, cudaEvent_t ev_begin = nullptr,
                  cudaEvent_t ev_end = nullptr);
  // graphs captured (and host milliseconds spent capturing and instantiating
  // or updating them) since creation
  uint64_t graph_builds = 0;
  double graph_build_ms = 0.0;
  void regroup(bool compute_keys, cudaStream_t st, bool move_records = false);
  // Grid update of accumulator a, then the semi-implicit Jacobi sweeps of
  // the scenes that ask for them.
  void grid_pass(int a, uint32_t max_jacobi, bool rigid, cudaStream_t st);
  void jacobi_pass(int a, uint32_t max_jacobi, cudaStream_t st);
  uint32_t max_jacobi_iters() const;
  // one item per occupied tile, plus one per kMinItemParticles particles of
  // a tile (the smallest item size the tuner may pick)
  static constexpr uint32_t kMinItemParticles = 128;
  size_t max_item_count() const { return (size_t)key_space + cap / kMinItemParticles + 2; }
  void sync_scenes(cudaStream_t st);

  PoolDev pool() const;
  void read_rows(uint32_t sid, int first, int count, float* out, cudaStream_t st);
  // Positions of one scene as float4 (w = 0) in identity order, stream-ordered
  // (no synchronisation).
  void pack_positions(uint32_t sid, float4* out, cudaStream_t st);
  void write_rows(uint32_t sid, int first, int count, const float* in, cudaStream_t st);
  void read_grid(uint32_t sid, float* mass, float* mom, cudaStream_t st);
  void totals(uint32_t sid, double* out8, cudaStream_t st);
  void status(uint32_t sid, mpm_status_info* out, cudaStream_t st);
  // Status words of every scene slot (kStatusWords each) in one copy.
  void status_words(std::vector<uint32_t>& out, cudaStream_t st);
  void reset_status(uint32_t sid, cudaStream_t st);
  // (key, identity) order of one scene's particles (reference permutation).
  void sort_permutation(uint32_t sid, uint32_t* keys, uint32_t* ids, uint32_t capacity, cudaStream_t st);
  uint64_t resident_bytes() const;
  uint32_t live_scenes() const;

 private:
  // Buffers sized by the key space and the item capacity, after a scene was
  // added: grows them (geometrically), marks a regrouping due and drops the
  // captured graphs.
  void layout_changed();
  void invalidate_graphs();
  // Host bookkeeping after a regrouping that dropped the retiring scenes.
  void finish_retirements();
  // Whether a regrouping follows substep s (0-based) of a call of `substeps`
  // substeps; advances `since`.  Sets need_regroup when one falls due on
  // the last substep (it opens the next call instead).
  bool regroup_due(uint32_t s, uint32_t substeps);
  void launch_gather_pass(int mode, bool keys, cudaStream_t st, bool publish_all = false);
  void launch_scatter_pass(int acc_out, cudaStream_t st);
  void launch_fused_pass(int acc_out, bool keys, cudaStream_t st);
 public:
  void set_deterministic(bool on);
  // Picks the regrouping interval: times `probe` substeps for each candidate
  // on a snapshot of the device state, restores the state and keeps the
  // fastest interval.  Returns it and fills ms_per_substep (one per
  // candidate, may be null).
  uint32_t autotune(uint32_t probe, const uint32_t* cands, int n_cands, float* ms_per_substep, cudaStream_t st);
  // The launch and tile shapes an autotuner may pick.
  struct Shapes {
    uint32_t interval;        // substeps between regroupings
    uint32_t item_particles;  // particles per work item (<= kStageMax)
    uint32_t fused;           // 1: fused gather + scatter for the non-final substeps
    uint32_t gather_per_sm;   // resident gather CTAs per SM (<= occupancy maximum)
    uint32_t scatter_per_sm;  // resident scatter CTAs per SM
  };
  enum Knob : uint32_t { kKnobInterval = 0, kKnobItem = 1, kKnobFused = 2, kKnobGatherCtas = 3, kKnobScatterCtas = 4 };
  struct Probe {
    uint32_t knob, value;
    float ms;
  };
  Shapes shapes() const;
  void apply_shapes(const Shapes& sh);
  // Tunes the knobs one after the other, each over its candidates (an empty
  // list takes the defaults), keeping the fastest value before the next
  // knob: every candidate times max(probe, 2 x interval) substeps on a
  // snapshot of the device state, which is restored afterwards (the scenes
  // do not advance).  Returns the shapes kept; `out` receives every probe.
  Shapes autotune_shapes(uint32_t probe, const std::vector<std::pair<uint32_t, std::vector<uint32_t>>>& knobs,
                         std::vector<Probe>* out, cudaStream_t st);
 private:
  void run_substeps(uint32_t substeps, cudaStream_t st);
  GraphKey graph_key(uint32_t substeps) const;
};

}  // namespace mpm
