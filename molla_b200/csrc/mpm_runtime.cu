// mpm_runtime.cu — host runtime of the B200 MPM path.
#include "mpm_runtime.cuh"

#include <chrono>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace mpm {

[[noreturn]] void throw_cuda(cudaError_t e, const char* what) {
  throw Error(MPM_ERR_GPU, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

static bool sticky_error(cudaError_t e) {
  switch (e) {
    case cudaErrorIllegalAddress:
    case cudaErrorLaunchFailure:
    case cudaErrorIllegalInstruction:
    case cudaErrorMisalignedAddress:
    case cudaErrorInvalidAddressSpace:
    case cudaErrorInvalidPc:
    case cudaErrorHardwareStackError:
    case cudaErrorAssert:
    case cudaErrorLaunchTimeout:
    case cudaErrorECCUncorrectable:
    case cudaErrorUnknown:
      return true;
    default:
      return false;
  }
}

Engine::Engine(int dev) : device(dev) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) {
    (void)cudaGetLastError();
    throw Error(MPM_ERR_GPU, "MpmSimulation needs a GPU engine: no CUDA device available");
  }
  if (dev < 0 || dev >= count) throw Error(MPM_ERR_INVALID, "CUDA device ordinal out of range");
  MPM_CK(cudaSetDevice(dev));
  MPM_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  MPM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
}

Engine::~Engine() {
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
  for (ProfRec& r : prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
}

cudaEvent_t Engine::take_event() {
  if (!event_pool.empty()) {
    cudaEvent_t e = event_pool.back();
    event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  MPM_CK(cudaEventCreate(&e));
  return e;
}

void Engine::prof_begin(int stage, cudaStream_t st, ProfRec* r) {
  r->stage = -1;
  if (!profiling || capturing) return;
  r->stage = stage;
  r->a = take_event();
  r->b = take_event();
  MPM_CK(cudaEventRecord(r->a, st));
}

void Engine::prof_end(ProfRec* r, cudaStream_t st) {
  if (r->stage < 0) return;
  MPM_CK(cudaEventRecord(r->b, st));
  prof.push_back(*r);
  if (prof.size() > 4096) prof_resolve();
}

void Engine::prof_resolve() {
  for (ProfRec& r : prof) {
    MPM_CK(cudaEventSynchronize(r.b));
    float ms = 0.f;
    MPM_CK(cudaEventElapsedTime(&ms, r.a, r.b));
    prof_ms[r.stage] += ms;
    prof_count[r.stage] += 1;
    event_pool.push_back(r.a);
    event_pool.push_back(r.b);
  }
  prof.clear();
}

void Engine::check() const {
  if (lost) throw Error(MPM_ERR_GPU, "device lost: " + lost_reason);
}

void Engine::note_error(cudaError_t e) {
  if (e != cudaSuccess && sticky_error(e)) {
    lost = true;
    lost_reason = cudaGetErrorString(e);
  }
}

bool RangeAlloc::alloc(uint64_t len, uint64_t align, uint64_t* off) {
  if (len == 0) {
    *off = 0;
    return true;
  }
  for (size_t i = 0; i < free_list.size(); ++i) {
    Range& r = free_list[i];
    const uint64_t start = (r.off + align - 1) / align * align;
    if (start + len <= r.off + r.len) {
      const uint64_t head = start - r.off;
      const uint64_t tail = r.off + r.len - (start + len);
      const Range old = r;
      free_list.erase(free_list.begin() + (long)i);
      if (tail) free_list.insert(free_list.begin() + (long)i, {start + len, tail});
      if (head) free_list.insert(free_list.begin() + (long)i, {old.off, head});
      *off = start;
      return true;
    }
  }
  return false;
}

void RangeAlloc::release(uint64_t off, uint64_t len) {
  if (!len) return;
  free_list.push_back({off, len});
  std::sort(free_list.begin(), free_list.end(), [](const Range& a, const Range& b) { return a.off < b.off; });
  std::vector<Range> merged;
  for (const Range& r : free_list) {
    if (!merged.empty() && merged.back().off + merged.back().len == r.off)
      merged.back().len += r.len;
    else
      merged.push_back(r);
  }
  free_list.swap(merged);
}

uint64_t RangeAlloc::high_water() const {
  // The free list is sorted and merged; if the last free range reaches the
  // end, everything after its start is unused.
  if (!free_list.empty() && free_list.back().off + free_list.back().len == capacity) return free_list.back().off;
  return capacity;
}

float dp_alpha_of(float friction_angle) {
  // material_row (crates/molla-solvers/src/mpm.rs:662-668), f32.
  const float sin_phi = std::sin(friction_angle);
  const float two_thirds = 2.0f / 3.0f;
  return std::sqrt(two_thirds) * (2.0f * sin_phi) / (3.0f - sin_phi);
}

SceneDev make_scene_dev(const mpm_config& cfg, const std::vector<mpm_rheology>& rows, float dt) {
  SceneDev d;
  std::memset(&d, 0, sizeof(d));
  d.n = cfg.grid_size;
  d.w = (cfg.grid_size + 3u) / 4u;
  d.dx = cfg.cell_size;
  d.inv_dx = 1.0f / cfg.cell_size;  // mpm.rs:2389 inv_cell_size: 1.0 / cell_size in f32
  d.ox = cfg.grid_origin[0];
  d.oy = cfg.grid_origin[1];
  d.oz = cfg.grid_origin[2];
  d.winx = cfg.grid_window_cells[0];
  d.winy = cfg.grid_window_cells[1];
  d.winz = cfg.grid_window_cells[2];
  d.dt = dt;
  d.gy = cfg.gravity_y;
  d.friction = cfg.boundary_friction;
  d.pad = cfg.boundary_pad ? (int32_t)cfg.boundary_pad : 2;
  d.sticky = cfg.walls == MPM_WALLS_STICKY ? 1 : 0;
  const int32_t win[3] = {d.winx, d.winy, d.winz};
  const float o[3] = {d.ox, d.oy, d.oz};
  for (int a = 0; a < 3; ++a) {
    // mpm.wgsl:1323-1326: lo = o + f32(window + pad) * dx, hi = o + f32(window + n - pad - 1) * dx
    const float flo = (float)(win[a] + d.pad);
    const float fhi = (float)(win[a] + (int32_t)cfg.grid_size - d.pad - 1);
    volatile float tlo = flo * d.dx;
    volatile float thi = fhi * d.dx;
    d.lo[a] = o[a] + tlo;
    d.hi[a] = o[a] + thi;
  }
  d.n_mat = (uint32_t)rows.size();
  d.live = 1;
  d.svd64 = cfg.svd_precision == MPM_SVD_FP64 ? 1u : 0u;
  d.jacobi_iters = cfg.time_step == MPM_TIME_STEP_IMPLICIT ? cfg.jacobi_iters : 0u;
  d.youngs = cfg.youngs;
  for (size_t i = 0; i < rows.size() && i < (size_t)kMaxMaterials; ++i) {
    const mpm_rheology& r = rows[i];
    MatDev& m = d.mat[i];
    const float e = r.youngs > 0.f ? r.youngs : cfg.youngs;
    const float nu = r.youngs > 0.f ? r.poisson : cfg.poisson;
    // mpm.wgsl:550-551 (f32)
    volatile float one_nu = 1.0f + nu;
    m.mu = e / (2.0f * one_nu);
    volatile float lam_den = (1.0f + nu) * (1.0f - 2.0f * nu);
    m.lam = e * nu / lam_den;
    // mpm.wgsl:1441 kappa = (d * lam + 2 mu) / (2 mu), d = 3
    volatile float k_num = 3.0f * m.lam + 2.0f * m.mu;
    m.kappa = k_num / (2.0f * m.mu);
    m.rheo = (int32_t)r.kind;
    m.dp_alpha = r.kind == MPM_RHEOLOGY_SAND ? dp_alpha_of(r.friction_angle) : 0.f;
    m.theta_c = r.kind == MPM_RHEOLOGY_SNOW ? r.theta_c : 0.f;
    m.theta_s = r.kind == MPM_RHEOLOGY_SNOW ? r.theta_s : 0.f;
    m.hardening = r.kind == MPM_RHEOLOGY_SNOW ? r.hardening : 0.f;
    // mpm.wgsl:1306-1307: exp(-max(damping, 0) * dt)
    const float vd = r.kind == MPM_RHEOLOGY_VISCOUS ? r.velocity_damping : 0.f;
    const float ad = r.kind == MPM_RHEOLOGY_VISCOUS ? r.affine_damping : 0.f;
    m.vfac = std::exp(-std::max(vd, 0.0f) * dt);
    m.afac = std::exp(-std::max(ad, 0.0f) * dt);
  }
  return d;
}

// ---------------------------------------------------------------------------

static uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

Group::Group(Engine* e, uint32_t max_scenes_, uint64_t particle_cap, uint64_t cell_cap_)
    : eng(e), stream(e->stream), max_scenes(std::max<uint32_t>(max_scenes_, 1)) {
  if (particle_cap > 0x7fffffffull) throw Error(MPM_ERR_INVALID, "particle capacity exceeds 2^31");
  cap = (uint32_t)std::max<uint64_t>(particle_cap, 1);
  cell_cap = round_up(std::max<uint64_t>(cell_cap_, 1), kCellBlock);
  MPM_CK(cudaSetDevice(eng->device));
  planes[0].alloc((size_t)kPlanes * cap);
  planes[1].alloc((size_t)kPlanes * cap);
  rec[0].alloc((size_t)16 * cap);
  {
    std::string err;
    if (!make_record_map(&rec_map[0], rec[0].ptr, cap, &err)) throw Error(MPM_ERR_GPU, "MPM scatter stage: " + err);
  }
  for (int i = 0; i < 2; ++i) {
    meta[i].alloc(cap);
    orig[i].alloc(cap);
    ks[i].alloc(cap);
    vs[i].alloc(cap);
    acc[i].alloc(cell_cap);
  }
  slot_of.alloc(cap);
  slot_tile.alloc(cell_cap / 64);
  keys_by_id.alloc(cap);
  slot_key.alloc(cap);
  hist.alloc(sort_hist_words(cap));
  vel.alloc(cell_cap);
  block_scene.alloc(cell_cap / kCellBlock);
  rigid_blocks.alloc(cell_cap / kCellBlock);
  rigid_d.alloc((size_t)max_scenes * kMaxRigid);
  wrench_d.alloc((size_t)max_scenes * kMaxRigid * 8);
  touched[0].alloc(cell_cap / kCellBlock);
  touched[1].alloc(cell_cap / kCellBlock);
  scenes_d.alloc(max_scenes);
  status_d.alloc((size_t)kStatusWords * max_scenes);
  work_d.alloc(2);
  n_items.alloc(2);
  totals_d.alloc(8);
  MPM_CK(cudaMallocHost((void**)&scenes_h, sizeof(SceneDev) * max_scenes));
  std::memset(scenes_h, 0, sizeof(SceneDev) * max_scenes);
  MPM_CK(cudaMemsetAsync(acc[0].ptr, 0, acc[0].bytes(), stream));
  MPM_CK(cudaMemsetAsync(acc[1].ptr, 0, acc[1].bytes(), stream));
  MPM_CK(cudaMemsetAsync(vel.ptr, 0, vel.bytes(), stream));
  MPM_CK(cudaMemsetAsync(rigid_blocks.ptr, 0, rigid_blocks.bytes(), stream));
  MPM_CK(cudaMemsetAsync(wrench_d.ptr, 0, wrench_d.bytes(), stream));
  MPM_CK(cudaMemsetAsync(touched[0].ptr, 0, touched[0].bytes(), stream));
  MPM_CK(cudaMemsetAsync(touched[1].ptr, 0, touched[1].bytes(), stream));
  MPM_CK(cudaMemsetAsync(keys_by_id.ptr, 0xff, keys_by_id.bytes(), stream));
  MPM_CK(cudaMemsetAsync(block_scene.ptr, 0xff, block_scene.bytes(), stream));
  MPM_CK(cudaMemsetAsync(status_d.ptr, 0, status_d.bytes(), stream));
  MPM_CK(cudaMemsetAsync(n_items.ptr, 0, n_items.bytes(), stream));
  MPM_CK(cudaMemsetAsync(scenes_d.ptr, 0, scenes_d.bytes(), stream));
  ids.init(cap);
  cells.init(cell_cap);
  // tile keys carry 6 cell bits below them in 32-bit sort keys, and the
  // all-ones key marks removed particles
  keyr.init((1ull << (32 - kCellBits)) - 2);
  const int nsm = std::max(eng->sms, 1);
  occ_gather32 = std::max(1, gather_grid_size(false) / nsm);
  occ_gather64 = std::max(1, gather_grid_size(true) / nsm);
  occ_scatter = std::max(1, scatter_grid_size() / nsm);
  occ_fused32 = std::max(1, fused_grid_size(false) / nsm);
  occ_fused64 = std::max(1, fused_grid_size(true) / nsm);
  if (const char* env = std::getenv("MOLLA_MPM_FUSED")) fused_mode = std::strcmp(env, "0") != 0 ? 1 : 0;
  MPM_CK(cudaStreamSynchronize(stream));
}

Group::~Group() {
  if (stream) cudaStreamSynchronize(stream);
  invalidate_graphs();
  if (scenes_h) cudaFreeHost(scenes_h);
}

void Group::invalidate_graphs() {
  for (auto& kv : graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  graphs.clear();
  ++epoch;
}

PoolDev Group::pool() const {
  PoolDev p;
  p.planes = planes[cur].ptr;
  p.cap = cap;
  p.meta = meta[cur].ptr;
  p.orig = orig[cur].ptr;
  p.keys_by_id = keys_by_id.ptr;
  p.acc[0] = acc[0].ptr;
  p.acc[1] = acc[1].ptr;
  p.touched[0] = touched[0].ptr;
  p.touched[1] = touched[1].ptr;
  p.rigid_blocks = rigid_blocks.ptr;
  p.rigid = rigid_d.ptr;
  p.wrench = wrench_d.ptr;
  p.vel = vel.ptr;
  p.rec = rec[rec_cur].ptr;
  p.slot_key = slot_key.ptr;
  p.scenes = scenes_d.ptr;
  p.status = status_d.ptr;
  p.items = items.ptr;
  p.n_items = n_items.ptr;
  p.item_top = item_top;
  p.tile_slot = tile_slot.ptr;
  p.slot_tile = slot_tile.ptr;
  p.tile_mark = tile_mark.ptr;
  p.work = work_d.ptr;
  p.item_order = item_order.ptr;
  return p;
}

uint32_t Group::live_scenes() const {
  uint32_t c = 0;
  for (const SceneHost& s : scenes) c += s.live ? 1u : 0u;
  return c;
}

uint64_t Group::resident_bytes() const {
  uint64_t b = 0;
  for (const SceneHost& s : scenes)
    if (s.live) b += (uint64_t)s.n * (2ull * kPlanes * 4ull + 64ull + 44ull) + s.grid_len * 48ull;
  return b;
}

// Geometric growth; the contents are not kept.
template <class T> static void grow(DevBuf<T>& b, size_t need) {
  if (b.count < need) b.alloc(std::max(need, b.count + b.count / 2));
}

// Geometric growth keeping the contents (stream-ordered copy, then the old
// allocation is freed).
template <class T> static void grow_keep(DevBuf<T>& b, size_t need, cudaStream_t st) {
  if (b.count >= need) return;
  DevBuf<T> nb(std::max(need, b.count + b.count / 2));
  if (b.count) MPM_CK(cudaMemcpyAsync(nb.ptr, b.ptr, b.bytes(), cudaMemcpyDeviceToDevice, st));
  MPM_CK(cudaStreamSynchronize(st));
  std::swap(b.ptr, nb.ptr);
  std::swap(b.count, nb.count);
}

void Group::layout_changed() {
  key_space = (uint32_t)keyr.high_water();
  grow(tile_start, (size_t)key_space + 2);
  const size_t max_items = max_item_count();
  if (items.count < max_items) {
    grow(items, max_items);
    grow(item_order, 64 * items.count);
  }
  // The work list's FP64-SVD items count down from item_top: it may change
  // only here, where a regrouping (which rebuilds the list) falls due.
  item_top = (uint32_t)items.count;
  if (deterministic) {
    grow(tile_item, (size_t)key_space + 2);
    grow(det_blocks, (size_t)item_top * kTileNodes);
  }
  scenes_dirty = true;
  need_regroup = true;
  invalidate_graphs();
  if (max_jacobi_iters() && vel2.count < cell_cap) vel2.alloc(cell_cap);
}

void Group::sync_scenes(cudaStream_t st) {
  if (!scenes_dirty) return;
  if (!scenes.empty())
    MPM_CK(cudaMemcpyAsync(scenes_d.ptr, scenes_h, sizeof(SceneDev) * scenes.size(), cudaMemcpyHostToDevice, st));
  // The pinned staging may be rewritten by the host after this call; make
  // the copy complete before returning.
  MPM_CK(cudaStreamSynchronize(st));
  scenes_dirty = false;
}

uint32_t Group::add_scene(const mpm_config& cfg, const std::vector<mpm_rheology>& rows, const float* xyz,
                          const float* velp, const float* mass, const float* vol, const uint32_t* mat_ids, uint32_t n,
                          float dt, uint32_t tile_cap) {
  records_valid = false;  // the state (or what its records depend on) changes
  eng->check();
  if (rows.empty() || rows.size() > (size_t)kMaxMaterials)
    throw Error(MPM_ERR_INVALID, "MPM scene needs 1..=8 material rows");
  {
    const uint64_t wt = (cfg.grid_size + 3u) / 4u;
    if (tile_cap > wt * wt * wt) throw Error(MPM_ERR_INVALID, "MPM tile pool capacity is invalid");
    if (tile_cap && cfg.time_step == MPM_TIME_STEP_IMPLICIT)
      throw Error(MPM_ERR_UNSUPPORTED, "sparse MPM grid storage runs the explicit time step only");
  }
  // dense: the n^3 block; sparse: tile_cap tiles of 64 nodes
  const uint64_t n3 = tile_cap ? 64ull * tile_cap
                               : (uint64_t)cfg.grid_size * cfg.grid_size * cfg.grid_size;
  uint32_t sid = (uint32_t)scenes.size();
  for (uint32_t i = 0; i < scenes.size(); ++i)
    if (!scenes[i].live && !scenes[i].retiring) {
      sid = i;
      break;
    }
  if (sid >= max_scenes) throw Error(MPM_ERR_BUSY, "MPM group has no free scene slot");
  if ((uint64_t)n_live + n > cap) throw Error(MPM_ERR_BUSY, "MPM group particle pool is full");
  uint64_t id0 = 0, g0 = 0;
  if (!ids.alloc(n, 1, &id0)) throw Error(MPM_ERR_BUSY, "MPM group identity space is full");
  const uint64_t glen = round_up(n3, kCellBlock);
  if (!cells.alloc(glen, kCellBlock, &g0)) {
    ids.release(id0, n);
    throw Error(MPM_ERR_BUSY, "MPM group grid pool is full");
  }
  const uint32_t w = (cfg.grid_size + 3u) / 4u;
  const uint64_t tiles = (uint64_t)w * w * w;
  uint64_t k0 = 0;
  if (!keyr.alloc(tiles, 1, &k0)) {
    ids.release(id0, n);
    cells.release(g0, glen);
    throw Error(MPM_ERR_BUSY, "MPM group key space is full");
  }
  if (sid == scenes.size()) scenes.emplace_back();
  SceneHost& s = scenes[sid];
  s.live = true;
  s.cfg = cfg;
  s.rows = rows;
  s.dt = dt;
  s.n = n;
  s.id_base = (uint32_t)id0;
  s.grid_off = g0;
  s.grid_len = glen;
  s.tiles = (uint32_t)tiles;
  s.key_off = (uint32_t)k0;
  s.tile_cap = tile_cap;

  // upload particles
  if (n) {
    // carve the uploads out of the staging buffer (256-byte aligned pieces)
    const size_t b3 = round_up((size_t)n * 12, 256), b1 = round_up((size_t)n * 4, 256);
    unsigned char* st = staging_bytes(b3 + (velp ? b3 : 0) + (mass ? b1 : 0) + (vol ? b1 : 0) + (mat_ids ? b1 : 0));
    auto take = [&](const void* src, size_t bytes, size_t span) -> void* {
      if (!src) return nullptr;
      void* dst = st;
      MPM_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
      st += span;
      return dst;
    };
    const float* dx = static_cast<const float*>(take(xyz, (size_t)n * 12, b3));
    const float* dv = static_cast<const float*>(take(velp, (size_t)n * 12, b3));
    const float* dm = static_cast<const float*>(take(mass, (size_t)n * 4, b1));
    const float* dvol = static_cast<const float*>(take(vol, (size_t)n * 4, b1));
    const uint32_t* dmat = static_cast<const uint32_t*>(take(mat_ids, (size_t)n * 4, b1));
    MPM_CK(launch_init_particles(pool(), slot_of.ptr, n_live, (uint32_t)id0, n, dx, dv, dm, dvol,
                                 cfg.particle_mass, cfg.particle_volume, dmat, sid, stream));
    eng->launches += 1;
    MPM_CK(cudaStreamSynchronize(stream));
  }
  // fresh grid range and status
  MPM_CK(cudaMemsetAsync(acc[0].ptr + g0, 0, glen * sizeof(float4), stream));
  MPM_CK(cudaMemsetAsync(acc[1].ptr + g0, 0, glen * sizeof(float4), stream));
  MPM_CK(cudaMemsetAsync(vel.ptr + g0, 0, glen * sizeof(float4), stream));
  MPM_CK(cudaMemsetAsync(rigid_blocks.ptr + g0 / kCellBlock, 0, glen / kCellBlock, stream));
  MPM_CK(cudaMemsetAsync(touched[0].ptr + g0 / kCellBlock, 0, glen / kCellBlock, stream));
  MPM_CK(cudaMemsetAsync(touched[1].ptr + g0 / kCellBlock, 0, glen / kCellBlock, stream));
  MPM_CK(launch_fill_u32(block_scene.ptr + g0 / kCellBlock, glen / kCellBlock, sid, stream));
  grow_keep(key_scene, (size_t)keyr.high_water(), stream);
  MPM_CK(launch_fill_u32(key_scene.ptr + k0, tiles, sid, stream));
  eng->launches += 2;
  if (tile_cap) {
    grow_keep(tile_slot, (size_t)keyr.high_water(), stream);
    if (tile_mark.count < (size_t)keyr.high_water()) {
      const size_t old = tile_mark.count;
      grow_keep(tile_mark, (size_t)keyr.high_water(), stream);
      MPM_CK(cudaMemsetAsync(tile_mark.ptr + old, 0, tile_mark.count - old, stream));
    }
    MPM_CK(launch_fill_u32(tile_slot.ptr + k0, tiles, kNoSlot, stream));
    MPM_CK(cudaMemsetAsync(tile_mark.ptr + k0, 0, tiles, stream));
    eng->launches += 1;
  }
  MPM_CK(cudaMemsetAsync(status_d.ptr + (size_t)sid * kStatusWords, 0, kStatusWords * 4, stream));
  n_live += n;
  SceneDev d = make_scene_dev(cfg, rows, dt);
  d.n_rigid = 0;
  d.key_off = s.key_off;
  d.status = sid;
  d.grid_off = g0;
  d.id_base = s.id_base;
  d.n_particles = n;
  d.tile_cap = tile_cap;
  scenes_h[sid] = d;
  s.n_rigid = 0;
  layout_changed();
  return sid;
}

void Group::remove_scene(uint32_t sid) {
  // A retirement compacted out at once: one regrouping of the pool.
  retire_scene(sid);
  compact(stream);
}

void Group::retire_scene(uint32_t sid) {
  if (sid >= scenes.size() || !scenes[sid].live) throw Error(MPM_ERR_INVALID, "unknown MPM scene");
  SceneHost& s = scenes[sid];
  s.live = false;
  s.retiring = true;
  s.n_rigid = 0;
  scenes_h[sid].live = 0;
  scenes_h[sid].n_rigid = 0;
  scenes_dirty = true;
  // Removed-particle keys, so that the next regrouping (the gather does not
  // write keys for a dead scene) sorts these identities behind every live one.
  if (s.n) MPM_CK(cudaMemsetAsync(keys_by_id.ptr + s.id_base, 0xff, (size_t)s.n * 4, stream));
  retiring.push_back(sid);
  n_retiring += s.n;
  // The regrouping baked into a captured graph moves a fixed particle count.
  invalidate_graphs();
}

void Group::finish_retirements() {
  if (!compact_issued) return;
  compact_issued = false;
  for (uint32_t sid : retiring) {
    SceneHost& s = scenes[sid];
    MPM_CK(launch_fill_u32(block_scene.ptr + s.grid_off / kCellBlock, s.grid_len / kCellBlock, 0xffffffffu, stream));
    MPM_CK(launch_fill_u32(key_scene.ptr + s.key_off, s.tiles, 0xffffffffu, stream));
    eng->launches += 2;
    ids.release(s.id_base, s.n);
    cells.release(s.grid_off, s.grid_len);
    keyr.release(s.key_off, s.tiles);
    n_live -= s.n;
    s.n = 0;
    s.retiring = false;
  }
  retiring.clear();
  n_retiring = 0;
  // Later regroupings sort fewer keys over a smaller key space; graphs
  // captured with the old counts are stale.
  key_space = (uint32_t)keyr.high_water();
  invalidate_graphs();
}

void Group::set_scene_budget(uint32_t sid, uint32_t substeps, cudaStream_t st, bool fresh) {
  records_valid = false;  // the state (or what its records depend on) changes
  if (sid >= scenes.size() || !scenes[sid].live) throw Error(MPM_ERR_INVALID, "unknown MPM scene");
  uint32_t done = 0;  // a scene just added has completed none
  if (!fresh) {
    MPM_CK(cudaMemcpyAsync(&done, status_d.ptr + (size_t)sid * kStatusWords + 1, 4, cudaMemcpyDeviceToHost, st));
    MPM_CK(cudaStreamSynchronize(st));
  }
  const uint32_t budget = substeps ? done + substeps : 0u;
  MPM_CK(launch_fill_u32(status_d.ptr + (size_t)sid * kStatusWords + 2, 1, budget, st));
  eng->launches += 1;
}

bool Group::any_sparse() const {
  for (size_t i = 0; i < scenes.size(); ++i)
    if (scenes[i].live && scenes[i].tile_cap) return true;
  return false;
}

void Group::finalize_tiles(cudaStream_t st) {
  if (!any_sparse()) return;
  MPM_CK(launch_tiles_finalize(pool(), key_scene.ptr, key_space, (uint32_t)scenes.size(), st));
  eng->launches += 2;
}

bool Group::any_svd32() const {
  for (size_t i = 0; i < scenes.size(); ++i)
    if (scenes[i].live && scenes[i].cfg.svd_precision != MPM_SVD_FP64) return true;
  return false;
}

bool Group::any_svd64() const {
  for (size_t i = 0; i < scenes.size(); ++i)
    if (scenes[i].live && scenes[i].cfg.svd_precision == MPM_SVD_FP64) return true;
  return false;
}

void Group::set_scene_dt(uint32_t sid, float dt) {
  SceneHost& s = scenes.at(sid);
  if (s.dt == dt) return;
  records_valid = false;  // the records hold dt (the stress term)
  s.dt = dt;
  SceneDev d = make_scene_dev(s.cfg, s.rows, dt);
  d.n_rigid = s.n_rigid;
  d.key_off = s.key_off;
  d.status = sid;
  d.grid_off = s.grid_off;
  d.id_base = s.id_base;
  d.n_particles = s.n;
  d.tile_cap = s.tile_cap;
  scenes_h[sid] = d;
  scenes_dirty = true;
  if (d.jacobi_iters && vel2.count < cell_cap) vel2.alloc(cell_cap);
}

bool Group::any_rigid() const {
  for (const SceneHost& s : scenes)
    if (s.live && s.n_rigid) return true;
  return false;
}

void Group::set_scene_rigid(uint32_t sid, const float* sp, uint32_t n, cudaStream_t st) {
  SceneHost& s = scenes.at(sid);
  if (!s.live) throw Error(MPM_ERR_INVALID, "scene is not live");
  if (n > (uint32_t)kMaxRigid) throw Error(MPM_ERR_INVALID, "at most 8 rigid spheres per scene");
  if (n && s.tile_cap)
    throw Error(MPM_ERR_UNSUPPORTED, "rigid spheres are not coupled to sparse MPM grid storage");
  std::vector<RigidDev> rd(n);
  for (uint32_t r = 0; r < n; ++r) {
    const float* q = sp + 7 * (size_t)r;
    for (int k = 0; k < 7; ++k)
      if (!std::isfinite(q[k])) throw Error(MPM_ERR_INVALID, "rigid sphere values must be finite");
    rd[r] = RigidDev{q[0], q[1], q[2], q[3], q[4], q[5], q[6], 0.f};
  }
  if (n)
    MPM_CK(cudaMemcpyAsync(rigid_d.ptr + (size_t)sid * kMaxRigid, rd.data(), n * sizeof(RigidDev),
                           cudaMemcpyHostToDevice, st));
  // Blocks a sphere may reach: every node within radius + dx of a center
  // (the imprint needs radius, the shell reaction radius + dx), with a cell
  // of margin for rounding.
  const uint32_t nn = s.cfg.grid_size;
  const uint64_t blocks = s.grid_len / kCellBlock;
  std::vector<uint8_t> mark(blocks, 0);
  const double dx = s.cfg.cell_size;
  for (uint32_t r = 0; r < n; ++r) {
    const RigidDev& R = rd[r];
    const double c[3] = {R.cx, R.cy, R.cz};
    int lo[3], hi[3];
    bool empty = !(R.radius > 0.f);
    for (int a = 0; a < 3; ++a) {
      const double rel0 = (c[a] - R.radius - 2.0 * dx - s.cfg.grid_origin[a]) / dx - s.cfg.grid_window_cells[a];
      const double rel1 = (c[a] + R.radius + 2.0 * dx - s.cfg.grid_origin[a]) / dx - s.cfg.grid_window_cells[a];
      lo[a] = (int)std::max(0.0, std::floor(rel0));
      hi[a] = (int)std::min((double)nn - 1, std::ceil(rel1));
      empty = empty || hi[a] < lo[a];
    }
    if (empty) continue;
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int y = lo[1]; y <= hi[1]; ++y) {
        const uint64_t row = (uint64_t)nn * ((uint64_t)y + (uint64_t)nn * z);
        const uint64_t b0 = (row + lo[0]) / kCellBlock, b1 = (row + hi[0]) / kCellBlock;
        for (uint64_t b = b0; b <= b1 && b < blocks; ++b) mark[b] = 1;
      }
  }
  if (blocks)
    MPM_CK(cudaMemcpyAsync(rigid_blocks.ptr + s.grid_off / kCellBlock, mark.data(), blocks, cudaMemcpyHostToDevice,
                           st));
  MPM_CK(cudaMemsetAsync(wrench_d.ptr + (size_t)sid * kMaxRigid * 8, 0, kMaxRigid * 8 * sizeof(float), st));
  MPM_CK(cudaStreamSynchronize(st));
  s.n_rigid = n;
  const float dt = s.dt;
  s.dt = -1.f;
  set_scene_dt(sid, dt);
  invalidate_graphs();
}

void Group::read_scene_wrench(uint32_t sid, float* out6, uint32_t n, cudaStream_t st) {
  const SceneHost& s = scenes.at(sid);
  n = std::min(n, s.n_rigid);
  if (!n) return;
  std::vector<float> w((size_t)n * 8);
  MPM_CK(cudaMemcpyAsync(w.data(), wrench_d.ptr + (size_t)sid * kMaxRigid * 8, w.size() * sizeof(float),
                         cudaMemcpyDeviceToHost, st));
  MPM_CK(cudaStreamSynchronize(st));
  for (uint32_t r = 0; r < n; ++r)
    for (int k = 0; k < 3; ++k) {
      out6[6 * r + k] = w[8 * r + k];
      out6[6 * r + 3 + k] = w[8 * r + 4 + k];
    }
}

void Group::set_scene_rows(uint32_t sid, const std::vector<mpm_rheology>& rows) {
  records_valid = false;  // the state (or what its records depend on) changes
  SceneHost& s = scenes.at(sid);
  s.rows = rows;
  const float dt = s.dt;
  s.dt = -1.f;
  set_scene_dt(sid, dt);
}

void Group::set_scene_cfg(uint32_t sid, const mpm_config& cfg) {
  records_valid = false;  // the state (or what its records depend on) changes
  SceneHost& s = scenes.at(sid);
  if (s.tile_cap && cfg.time_step == MPM_TIME_STEP_IMPLICIT)
    throw Error(MPM_ERR_UNSUPPORTED, "sparse MPM grid storage runs the explicit time step only");
  s.cfg = cfg;
  invalidate_graphs();
  const float dt = s.dt;
  s.dt = -1.f;
  set_scene_dt(sid, dt);
}

unsigned char* Group::staging_bytes(size_t bytes) {
  if (staging.count < bytes) {
    MPM_CK(cudaStreamSynchronize(stream));
    staging.alloc(bytes + bytes / 4);
  }
  return staging.ptr;
}

void Group::set_material_ids(uint32_t sid, const uint32_t* host_ids, uint32_t n) {
  records_valid = false;  // the state (or what its records depend on) changes
  SceneHost& s = scenes.at(sid);
  if (n != s.n) throw Error(MPM_ERR_INVALID, "material id count does not match the particle count");
  if (!n) return;
  uint32_t* d = reinterpret_cast<uint32_t*>(staging_bytes((size_t)n * 4));
  MPM_CK(cudaMemcpyAsync(d, host_ids, (size_t)n * 4, cudaMemcpyHostToDevice, stream));
  MPM_CK(launch_set_material_ids(pool(), slot_of.ptr, s.id_base, n, d, stream));
  eng->launches += 1;
  MPM_CK(cudaStreamSynchronize(stream));
}

static int bits_for(uint64_t values) {
  // smallest b with values < 2^b - 1 (so that the all-ones pattern of b bits
  // is free for removed particles)
  int b = 1;
  while (b < 32 && ((1ull << b) - 1ull) <= values) ++b;
  return b;
}

// Regrouping: sort (base-cell key, identity) stably — key = (scene tile
// offset + 4^3 tile of the base cell, cell inside the tile) — and move the
// particle state to that order, so that each tile's particles are
// contiguous and, inside the tile, grouped by base cell.  The sorted key of
// every slot is kept for the scatter, and the work list is rebuilt from the
// tile boundaries.
void Group::regroup(bool compute_keys, cudaStream_t st, bool move_records) {
  if (!move_records) records_valid = false;  // the records stay in the old order
  ProfRec pr;
  eng->prof_begin(kStageOrdering, st, &pr);
  if (compute_keys) {
    MPM_CK(launch_keys(pool(), n_live, st));
    eng->launches += 1;
  }
  const uint32_t n_sort = (uint32_t)ids.high_water();
  uint32_t* skeys = nullptr;
  uint32_t* sids = nullptr;
  MPM_CK(radix_sort_pairs(st, keys_by_id.ptr, nullptr, ks[0].ptr, ks[1].ptr, vs[0].ptr, vs[1].ptr, hist.ptr, n_sort,
                          bits_for((uint64_t)key_space << kCellBits), &skeys, &sids, &eng->launches));
  // both record buffers exist only in deterministic mode (set_deterministic)
  if (move_records && (rec[0].count < (size_t)16 * cap || rec[1].count < (size_t)16 * cap))
    throw Error(MPM_ERR_INVALID, "MPM regroup: records can move only between two allocated record buffers");
  const float4* rsrc = move_records ? reinterpret_cast<const float4*>(rec[rec_cur].ptr) : nullptr;
  float4* rdst = move_records ? reinterpret_cast<float4*>(rec[rec_cur ^ 1].ptr) : nullptr;
  // Particles of retired scenes sorted behind the live ones: only the live
  // prefix moves, which drops them.
  const uint32_t n_keep = n_live - n_retiring;
  MPM_CK(launch_reorder(planes[cur].ptr, planes[cur ^ 1].ptr, cap, meta[cur].ptr, meta[cur ^ 1].ptr,
                        orig[cur ^ 1].ptr, slot_of.ptr, sids, skeys, slot_key.ptr, rsrc, rdst, n_keep, st));
  eng->launches += 1;
  cur ^= 1;
  if (move_records) rec_cur ^= 1;
  if (!retiring.empty()) compact_issued = true;
  // Items: whole tiles for the fixed-order scatter (one item per tile);
  // otherwise tiles cut into pieces of at most kStageMax particles, whose
  // scatter records fit the shared-memory stage.
  MPM_CK(launch_items(skeys, kCellBits, n_keep, key_space, tile_start.ptr, key_scene.ptr, scenes_d.ptr,
                      deterministic ? 0u : item_chunk, item_top, items.ptr,
                      n_items.ptr, deterministic ? tile_item.ptr : nullptr, st));
  eng->launches += key_space ? 2 : 1;
  if (!deterministic && key_space) {
    MPM_CK(launch_item_order(items.ptr, n_items.ptr, item_top, slot_key.ptr, item_order.ptr, st));
    eng->launches += 1;
  }
  need_regroup = false;
  since = 0;
  ++regroups;
  eng->prof_end(&pr, st);
}

int Group::gather_grid(bool f64) const {
  const int mx = f64 ? occ_gather64 : occ_gather32;
  return std::max(eng->sms, 1) * (gather_per_sm ? std::min<int>((int)gather_per_sm, mx) : mx);
}

int Group::fused_grid(bool f64) const {
  // the fused kernel follows the gather's count, scaled to its own maximum
  const int mx = f64 ? occ_fused64 : occ_fused32;
  const int g = f64 ? occ_gather64 : occ_gather32;
  const int k = gather_per_sm ? std::max(1, (int)(gather_per_sm * mx + g - 1) / g) : mx;
  return std::max(eng->sms, 1) * std::min(k, mx);
}

int Group::scatter_grid() const {
  return std::max(eng->sms, 1) * (scatter_per_sm ? std::min<int>((int)scatter_per_sm, occ_scatter) : occ_scatter);
}

// The gather runs once per SVD form present: over the FP32-SVD items, then
// over the FP64-SVD items of the work list.
void Group::launch_gather_pass(int mode, bool keys, cudaStream_t st, bool publish_all) {
  ProfRec pr;
  eng->prof_begin(mode == kRecord ? kStageRecord : kStageGather, st, &pr);
  for (int f64 = 0; f64 < 2; ++f64) {
    if (!(f64 ? any_svd64() : any_svd32())) continue;
    MPM_CK(launch_gather(mode, keys, f64 != 0, pool(), f64 ? svd_tol64 : svd_tol32, svd_sweeps, reuse_svd ? 1 : 0,
                         gather_grid(f64 != 0), st, publish_all));
    eng->launches += 1;
  }
  eng->prof_end(&pr, st);
}

void Group::launch_scatter_pass(int acc_out, cudaStream_t st) {
  ProfRec pr;
  eng->prof_begin(kStageScatter, st, &pr);
  if (deterministic) {
    MPM_CK(launch_scatter_det(pool(), det_blocks.ptr, acc_out, scatter_grid(), st));
    MPM_CK(launch_combine_det(pool(), det_blocks.ptr, tile_item.ptr, key_space, acc_out, st));
    eng->launches += 1;
  } else {
    MPM_CK(launch_scatter(pool(), rec_map[rec_cur], acc_out, scatter_grid(), st));
  }
  eng->prof_end(&pr, st);
  eng->launches += 1;
}

void Group::launch_fused_pass(int acc_out, bool keys, cudaStream_t st) {
  ProfRec pr;
  eng->prof_begin(kStageGather, st, &pr);
  for (int f64 = 0; f64 < 2; ++f64) {
    if (!(f64 ? any_svd64() : any_svd32())) continue;
    MPM_CK(launch_fused(keys, f64 != 0, pool(), f64 ? svd_tol64 : svd_tol32, svd_sweeps, reuse_svd ? 1 : 0, acc_out,
                        fused_grid(f64 != 0), st));
    eng->launches += 1;
  }
  eng->prof_end(&pr, st);
}

Group::Shapes Group::shapes() const {
  Shapes sh;
  sh.interval = sort_interval;
  sh.item_particles = item_chunk;
  sh.fused = use_fused() ? 1u : 0u;
  sh.gather_per_sm = gather_per_sm ? gather_per_sm : (uint32_t)occ_gather32;
  sh.scatter_per_sm = scatter_per_sm ? scatter_per_sm : (uint32_t)occ_scatter;
  return sh;
}

void Group::apply_shapes(const Shapes& sh) {
  if (sh.item_particles < kMinItemParticles || sh.item_particles > (uint32_t)kStageMax)
    throw Error(MPM_ERR_INVALID, "MPM item size must be in 128..=" + std::to_string(kStageMax) + " particles");
  if (sh.gather_per_sm < 1 || sh.scatter_per_sm < 1)
    throw Error(MPM_ERR_INVALID, "MPM CTAs per SM must be at least 1");
  if (sh.interval != sort_interval) {
    sort_interval = sh.interval;
    need_regroup = true;
  }
  if (sh.item_particles != item_chunk) {
    item_chunk = sh.item_particles;
    need_regroup = true;  // the work list is cut anew
  }
  fused_mode = sh.fused ? 1 : 0;
  gather_per_sm = std::min<uint32_t>(sh.gather_per_sm, (uint32_t)std::max(occ_gather32, occ_gather64));
  scatter_per_sm = std::min<uint32_t>(sh.scatter_per_sm, (uint32_t)occ_scatter);
  invalidate_graphs();
}

uint32_t Group::autotune(uint32_t probe, const uint32_t* cands, int n_cands, float* ms_out, cudaStream_t st) {
  if (!n_live || !probe || n_cands <= 0) return sort_interval;
  std::vector<Probe> probes;
  const Shapes sh = autotune_shapes(probe, {{kKnobInterval, std::vector<uint32_t>(cands, cands + n_cands)}}, &probes, st);
  for (size_t i = 0; i < probes.size() && ms_out; ++i) ms_out[i] = probes[i].ms;
  return sh.interval;
}

Group::Shapes Group::autotune_shapes(uint32_t probe, const std::vector<std::pair<uint32_t, std::vector<uint32_t>>>& knobs,
                                     std::vector<Probe>* out, cudaStream_t st) {
  eng->check();
  Shapes best_sh = shapes();
  if (!n_live || !probe) return best_sh;
  // The probes regroup; retired scenes must not leave the pool behind the
  // host's back.
  if (n_retiring) throw Error(MPM_ERR_BUSY, "MPM autotune with retired scenes awaiting compaction");
  sync_scenes(st);
  // Snapshot of everything a substep reads or writes.
  const size_t pbytes = (size_t)kPlanes * cap * sizeof(float);
  const uint64_t cells_hw = cells.high_water();
  DevBuf<float> bplanes((size_t)kPlanes * cap);
  DevBuf<uint32_t> bmeta(cap), borig(cap), bslot(cap), bkey(cap), bstatus(status_d.count);
  DevBuf<float4> bacc0(cells_hw), bacc1(cells_hw), bvel(cells_hw);
  DevBuf<uint8_t> btouch0(cells_hw / kCellBlock + 1), btouch1(cells_hw / kCellBlock + 1);
  DevBuf<uint32_t> bslots(tile_slot.count), bslot_tile(cells_hw / 64 + 1);
  auto save = [&](bool to_backup) {
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (bytes) MPM_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st));
    };
    if (to_backup) {
      cp(bplanes.ptr, planes[cur].ptr, pbytes);
      cp(bmeta.ptr, meta[cur].ptr, cap * 4);
      cp(borig.ptr, orig[cur].ptr, cap * 4);
      cp(bslot.ptr, slot_of.ptr, cap * 4);
      cp(bkey.ptr, slot_key.ptr, cap * 4);
      cp(bstatus.ptr, status_d.ptr, status_d.bytes());
      cp(bacc0.ptr, acc[0].ptr, cells_hw * sizeof(float4));
      cp(bacc1.ptr, acc[1].ptr, cells_hw * sizeof(float4));
      cp(bvel.ptr, vel.ptr, cells_hw * sizeof(float4));
      cp(btouch0.ptr, touched[0].ptr, cells_hw / kCellBlock);
      cp(btouch1.ptr, touched[1].ptr, cells_hw / kCellBlock);
      cp(bslots.ptr, tile_slot.ptr, tile_slot.bytes());
      cp(bslot_tile.ptr, slot_tile.ptr, (cells_hw / 64) * 4);
    } else {
      cp(planes[cur].ptr, bplanes.ptr, pbytes);
      cp(meta[cur].ptr, bmeta.ptr, cap * 4);
      cp(orig[cur].ptr, borig.ptr, cap * 4);
      cp(slot_of.ptr, bslot.ptr, cap * 4);
      cp(slot_key.ptr, bkey.ptr, cap * 4);
      cp(status_d.ptr, bstatus.ptr, status_d.bytes());
      cp(acc[0].ptr, bacc0.ptr, cells_hw * sizeof(float4));
      cp(acc[1].ptr, bacc1.ptr, cells_hw * sizeof(float4));
      cp(vel.ptr, bvel.ptr, cells_hw * sizeof(float4));
      cp(touched[0].ptr, btouch0.ptr, cells_hw / kCellBlock);
      cp(touched[1].ptr, btouch1.ptr, cells_hw / kCellBlock);
      cp(tile_slot.ptr, bslots.ptr, tile_slot.bytes());
      cp(slot_tile.ptr, bslot_tile.ptr, (cells_hw / 64) * 4);
    }
  };
  const int cur0 = cur, az0 = acc_zero, al0 = acc_last;
  const uint64_t done0 = substeps_done, regroups0 = regroups;
  save(true);
  OwnedEvent e0, e1;
  auto rewind = [&]() {
    cur = cur0;
    acc_zero = az0;
    acc_last = al0;
    need_regroup = true;  // every run starts from a fresh regrouping
    records_valid = false;  // the records are not part of the snapshot
    save(false);
  };
  auto time_current = [&]() {
    // at least two regroupings inside the timed window
    const uint32_t n = std::max<uint32_t>(probe, 2u * std::max<uint32_t>(sort_interval, 1u));
    rewind();
    run_substeps(n, st);  // warm
    rewind();
    MPM_CK(cudaEventRecord(e0, st));
    run_substeps(n, st);
    MPM_CK(cudaEventRecord(e1, st));
    MPM_CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    MPM_CK(cudaEventElapsedTime(&ms, e0, e1));
    return ms / (float)n;
  };
  try {
    for (const auto& kv : knobs) {
      const uint32_t knob = kv.first;
      std::vector<uint32_t> cands = kv.second;
      if (cands.empty()) {
        switch (knob) {
          case kKnobInterval: cands = {8, 16, 32, 64}; break;
          case kKnobItem: cands = {(uint32_t)kStageMax, 512, 384, 256}; break;
          case kKnobFused: cands = {0, 1}; break;
          case kKnobGatherCtas: cands = {best_sh.gather_per_sm, best_sh.gather_per_sm - 1}; break;
          case kKnobScatterCtas: cands = {best_sh.scatter_per_sm, best_sh.scatter_per_sm - 1}; break;
          default: throw Error(MPM_ERR_INVALID, "unknown MPM tuning knob");
        }
      }
      if (deterministic && (knob == kKnobItem || knob == kKnobFused)) continue;  // whole tiles, never fused
      float best = 1e30f;
      Shapes keep = best_sh;
      for (uint32_t v : cands) {
        if (knob == kKnobFused ? v > 1 : v == 0) continue;
        Shapes sh = best_sh;
        switch (knob) {
          case kKnobInterval: sh.interval = v; break;
          case kKnobItem: sh.item_particles = std::min<uint32_t>(std::max<uint32_t>(v, kMinItemParticles), kStageMax); break;
          case kKnobFused: sh.fused = v; break;
          case kKnobGatherCtas: sh.gather_per_sm = v; break;
          case kKnobScatterCtas: sh.scatter_per_sm = v; break;
          default: break;
        }
        apply_shapes(sh);
        const float ms = time_current();
        if (out) out->push_back({knob, v, ms});
        if (ms < best) {
          best = ms;
          keep = shapes();
        }
      }
      best_sh = keep;
    }
  } catch (...) {
    rewind();
    cudaStreamSynchronize(st);
    substeps_done = done0;
    regroups = regroups0;
    since = 0;
    throw;
  }
  apply_shapes(best_sh);
  rewind();
  MPM_CK(cudaStreamSynchronize(st));
  need_regroup = true;  // the work list belongs to the probes; rebuild it
  substeps_done = done0;
  regroups = regroups0;
  since = 0;
  invalidate_graphs();
  return best_sh;
}

// Fixed-order P2G: a regrouping after every gather (so every particle sits in
// its base cell when it is deposited) and the two-pass deterministic scatter.
void Group::set_deterministic(bool on) {
  records_valid = false;  // the state (or what its records depend on) changes
  if (on == deterministic) return;
  deterministic = on;
  if (on) {
    if (rec[1].count < (size_t)16 * cap) {
      rec[1].alloc((size_t)16 * cap);
      std::string err;
      if (!make_record_map(&rec_map[1], rec[1].ptr, cap, &err)) throw Error(MPM_ERR_GPU, "MPM scatter stage: " + err);
    }
    const size_t tiles = (size_t)key_space + 2;
    if (tile_item.count < tiles) tile_item.alloc(tiles);
    // blocks are indexed by item slot (one item per tile in this mode)
    const size_t slots = std::max<size_t>(item_top, tiles);
    if (det_blocks.count < slots * kTileNodes) det_blocks.alloc(slots * kTileNodes);
  }
  need_regroup = true;
  invalidate_graphs();
}

// One call: record + scatter of the first substep, then per substep the grid
// update, the gather (which also records B for the next substep unless it is
// the last) and the next scatter.  Regrouping happens after a scatter, every
// `sort_interval` substeps.
uint32_t Group::max_jacobi_iters() const {
  uint32_t mj = 0;
  for (size_t i = 0; i < scenes.size(); ++i)
    if (scenes[i].live) mj = std::max(mj, scenes_h[i].jacobi_iters);
  return mj;
}

void Group::grid_pass(int a, uint32_t max_jacobi, bool rigid, cudaStream_t st) {
  const uint64_t total_cells = cells.high_water();
  if (rigid) MPM_CK(cudaMemsetAsync(wrench_d.ptr, 0, wrench_d.bytes(), st));  // wrench of this substep only
  MPM_CK(launch_grid_update(pool(), block_scene.ptr, total_cells, a, 1, st));
  eng->launches += 1;
  if (max_jacobi) jacobi_pass(a, max_jacobi, st);
  if (rigid) {
    MPM_CK(launch_rigid_shell(pool(), block_scene.ptr, total_cells, a, st));
    eng->launches += 1;
  }
}

void Group::jacobi_pass(int a, uint32_t max_jacobi, cudaStream_t st) {
  const uint64_t total_cells = cells.high_water();
  float4* bufs[2] = {vel.ptr, vel2.ptr};
  int cur = 0;
  for (uint32_t k = 0; k < max_jacobi; ++k) {
    MPM_CK(launch_grid_jacobi(pool(), block_scene.ptr, total_cells, a, bufs[cur], bufs[cur ^ 1], k, st));
    eng->launches += 1;
    cur ^= 1;
  }
  if (cur) {
    MPM_CK(launch_vel_copy(touched[a].ptr, block_scene.ptr, total_cells, bufs[1], bufs[0], st));
    eng->launches += 1;
  }
}

bool Group::regroup_due(uint32_t s, uint32_t substeps) {
  const bool last = s + 1 == substeps;
  if (deterministic) return !last;
  if (sort_interval == 0) return false;
  if (++since < sort_interval) return false;
  if (last) {
    // the last substep of a call writes no record and no keys: the
    // regrouping opens the next call instead (keys computed there)
    need_regroup = true;
    return false;
  }
  return true;
}

void Group::run_substeps(uint32_t substeps, cudaStream_t st) {
  // With the records of the last call still valid and no regrouping to open
  // this call, the record-only gather is skipped.  (A regrouping moves the
  // particles but not the records, whose second buffer exists only in
  // deterministic mode, so after one the records are recomputed.)
  const bool reuse_records = records_valid && !deterministic && !need_regroup;
  if (need_regroup || deterministic) regroup(true, st);
  const uint32_t max_jacobi = max_jacobi_iters();
  const bool rigid = any_rigid();
  if (!reuse_records) launch_gather_pass(kRecord, false, st);
  finalize_tiles(st);  // sparse scenes: the tile map of the first deposit
  launch_scatter_pass(acc_zero, st);
  int a = acc_zero;
  const bool fused = use_fused();
  for (uint32_t s = 0; s < substeps; ++s) {
    ProfRec pr;
    eng->prof_begin(kStageGrid, st, &pr);
    grid_pass(a, max_jacobi, rigid, st);
    eng->prof_end(&pr, st);
    const bool last = s + 1 == substeps;
    const bool due = regroup_due(s, substeps);
    if (!last && fused) {
      // gather + scatter in one launch; the regrouping follows the deposit
      launch_fused_pass(a ^ 1, due, st);
      if (due) regroup(false, st);
      a ^= 1;
      continue;
    }
    // The last gather of a call publishes v and C; outside deterministic
    // mode it also writes the records, for the next call's first scatter.
    launch_gather_pass(last && deterministic ? kG2P : kG2PRecord, due, st, last);
    if (!last) {
      finalize_tiles(st);  // sparse scenes: the tile map of the next deposit
      if (deterministic) {
        // Fixed order: particles (and their records) regrouped into the
        // cells of their new positions before they are deposited.
        regroup(false, st, true);
        launch_scatter_pass(a ^ 1, st);
      } else {
        launch_scatter_pass(a ^ 1, st);
        if (due) regroup(false, st);
      }
      a ^= 1;
    }
  }
  acc_last = a;
  acc_zero = a ^ 1;
  substeps_done += substeps;
  records_valid = !deterministic;
}

void Group::compact(cudaStream_t st) {
  eng->check();
  if (retiring.empty()) return;
  if (n_retiring && n_live > n_retiring) {
    sync_scenes(st);
    regroup(true, st);
  } else {
    // nothing live to sort out from among them: every slot is dropped
    compact_issued = true;
    need_regroup = true;
  }
  finish_retirements();
}

void Group::step(uint32_t substeps, cudaStream_t st) {
  eng->check();
  if (substeps && n_live == n_retiring) compact(st);
  if (!substeps || n_live == 0 || n_live == n_retiring) return;
  sync_scenes(st);
  run_substeps(substeps, st);
  finish_retirements();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    eng->note_error(e);
    throw_cuda(e, "MPM step launch");
  }
}

Group::GraphKey Group::graph_key(uint32_t substeps) const {
  GraphKey k;
  k.substeps = substeps;
  k.since = deterministic ? 0u : since;
  k.interval = sort_interval;
  k.flags = ((uint32_t)(records_valid && !deterministic && !need_regroup) << 6) | ((uint32_t)rec_cur << 5) |
            ((uint32_t)cur << 4) |
            ((uint32_t)acc_zero << 3) |
            ((uint32_t)any_svd64() << 2) | ((uint32_t)any_svd32() << 1) | (need_regroup ? 1u : 0u);
  return k;
}

void Group::step_graph(uint32_t substeps, uint32_t repeat, cudaStream_t st, cudaEvent_t ev_begin,
                       cudaEvent_t ev_end) {
  eng->check();
  if (substeps && repeat && n_live == n_retiring) compact(st);
  if (!substeps || n_live == 0 || n_live == n_retiring || !repeat) return;
  sync_scenes(st);
  for (uint32_t r = 0; r < repeat; ++r) {
    const GraphKey key = graph_key(substeps);
    const int cur0 = cur, az0 = acc_zero, rc0 = rec_cur;
    const bool nr0 = need_regroup;
    const bool rv0 = records_valid;
    const uint32_t since0 = since;
    const uint64_t regroups0 = regroups;
    auto it = graphs.find(key);
    Graph g;
    if (it == graphs.end() || it->second.epoch != epoch) {
      const auto t_build0 = std::chrono::steady_clock::now();
      const uint64_t saved = eng->launches;
      cudaGraph_t graph = nullptr;
      MPM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      eng->capturing = true;
      try {
        run_substeps(substeps, st);
      } catch (...) {
        eng->capturing = false;
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      eng->capturing = false;
      MPM_CK(cudaStreamEndCapture(st, &graph));
      g.kernels = eng->launches - saved;
      eng->launches = saved;
      // A layout change (a scene added or retired, a regrouping moved)
      // mostly changes launch parameters, not the sequence: update the
      // existing executable graph in place when the topology allows, which
      // costs far less host time than instantiating a new one.
      bool updated = false;
      if (it != graphs.end() && it->second.exec) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(it->second.exec, graph, &info) == cudaSuccess) {
          g.exec = it->second.exec;
          updated = true;
        } else {
          (void)cudaGetLastError();  // the failed update is not a sticky error
          cudaGraphExecDestroy(it->second.exec);
          it->second.exec = nullptr;
        }
      }
      if (!updated) {
        const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
        if (ie != cudaSuccess) {
          cudaGraphDestroy(graph);
          MPM_CK(ie);
        }
      }
      cudaGraphDestroy(graph);
      g.epoch = epoch;
      // run_substeps advanced the host bookkeeping; rewind it, the launch
      // below applies the same transition.
      cur = cur0;
      acc_zero = az0;
      rec_cur = rc0;
      need_regroup = nr0;
      records_valid = rv0;
      since = since0;
      regroups = regroups0;
      compact_issued = false;
      substeps_done -= substeps;
      graphs[key] = g;
      ++graph_builds;
      graph_build_ms +=
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_build0).count();
    } else {
      g = it->second;
    }
    if (ev_begin && r == 0) MPM_CK(cudaEventRecord(ev_begin, st));
    MPM_CK(cudaGraphLaunch(g.exec, st));
    if (ev_end && r + 1 == repeat) MPM_CK(cudaEventRecord(ev_end, st));
    eng->launches += g.kernels;
    // Replay the host-side state transition of the captured sequence (the
    // same decisions run_substeps made while it was captured).
    auto regrouped = [&](bool records) {
      cur ^= 1;
      if (records) rec_cur ^= 1;
      need_regroup = false;
      since = 0;
      ++regroups;
      if (!retiring.empty()) compact_issued = true;
    };
    if (need_regroup || deterministic) regrouped(false);
    int a = acc_zero;
    for (uint32_t s = 0; s < substeps; ++s) {
      const bool last = s + 1 == substeps;
      const bool due = regroup_due(s, substeps);
      if (deterministic && !last) regrouped(true);
      else if (due) regrouped(false);
      if (!last) a ^= 1;
    }
    acc_last = a;
    acc_zero = a ^ 1;
    substeps_done += substeps;
    records_valid = !deterministic;
    finish_retirements();
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    eng->note_error(e);
    throw_cuda(e, "MPM graph launch");
  }
}

void Group::read_rows(uint32_t sid, int first, int count, float* out, cudaStream_t st) {
  const SceneHost& s = scenes.at(sid);
  if (!s.n) return;
  const size_t bytes = (size_t)count * s.n * sizeof(float);
  float* d = reinterpret_cast<float*>(staging_bytes(bytes));
  if (count == 3)
    MPM_CK(launch_gather_xyz(pool(), first, slot_of.ptr, s.id_base, s.n, d, st));
  else
    MPM_CK(launch_gather_rows(pool(), first, count, slot_of.ptr, s.id_base, s.n, d, st));
  eng->launches += 1;
  MPM_CK(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, st));
  MPM_CK(cudaStreamSynchronize(st));
}

void Group::pack_positions(uint32_t sid, float4* out, cudaStream_t st) {
  const SceneHost& s = scenes.at(sid);
  if (!s.n) return;
  MPM_CK(launch_pack_positions(pool(), slot_of.ptr, s.id_base, s.n, out, st));
  eng->launches += 1;
}

void Group::write_rows(uint32_t sid, int first, int count, const float* in, cudaStream_t st) {
  records_valid = false;  // the state (or what its records depend on) changes
  const SceneHost& s = scenes.at(sid);
  if (!s.n) return;
  const size_t bytes = (size_t)count * s.n * sizeof(float);
  float* d = reinterpret_cast<float*>(staging_bytes(bytes));
  MPM_CK(cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, st));
  MPM_CK(launch_scatter_rows(pool(), first, count, slot_of.ptr, s.id_base, s.n, d, st));
  eng->launches += 1;
  MPM_CK(cudaStreamSynchronize(st));
}

void Group::read_grid(uint32_t sid, float* mass, float* mom, cudaStream_t st) {
  const SceneHost& s = scenes.at(sid);
  const uint32_t n = s.cfg.grid_size;
  const uint64_t n3 = (uint64_t)n * n * n;
  auto put = [&](uint64_t i, const float4& v) {
    if (mass) mass[i] = v.x;
    if (mom) {
      mom[3 * i] = v.y;
      mom[3 * i + 1] = v.z;
      mom[3 * i + 2] = v.w;
    }
  };
  if (!s.tile_cap) {
    std::vector<float4> h(n3);
    MPM_CK(cudaMemcpyAsync(h.data(), acc[acc_last].ptr + s.grid_off, n3 * sizeof(float4), cudaMemcpyDeviceToHost,
                           st));
    MPM_CK(cudaStreamSynchronize(st));
    for (uint64_t i = 0; i < n3; ++i) put(i, h[i]);
    return;
  }
  // sparse: the slots and the tile map, scattered into the dense layout
  std::vector<float4> h((size_t)s.tile_cap * 64);
  std::vector<uint32_t> map(s.tiles);
  MPM_CK(cudaMemcpyAsync(h.data(), acc[acc_last].ptr + s.grid_off, h.size() * sizeof(float4), cudaMemcpyDeviceToHost,
                         st));
  MPM_CK(cudaMemcpyAsync(map.data(), tile_slot.ptr + s.key_off, map.size() * 4, cudaMemcpyDeviceToHost, st));
  MPM_CK(cudaStreamSynchronize(st));
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint64_t i = 0; i < n3; ++i) put(i, zero);
  const uint32_t w = (n + 3u) / 4u;
  for (uint32_t t = 0; t < s.tiles; ++t) {
    if (map[t] == kNoSlot || map[t] >= s.tile_cap) continue;
    const uint32_t tx = t % w, ty = (t / w) % w, tz = t / (w * w);
    for (uint32_t l = 0; l < 64; ++l) {
      const uint32_t ix = 4 * tx + (l & 3u), iy = 4 * ty + ((l >> 2) & 3u), iz = 4 * tz + (l >> 4);
      if (ix >= n || iy >= n || iz >= n) continue;
      put((uint64_t)ix + (uint64_t)n * ((uint64_t)iy + (uint64_t)n * iz), h[(size_t)map[t] * 64 + l]);
    }
  }
}

void Group::totals(uint32_t sid, double* out8, cudaStream_t st) {
  const SceneHost& s = scenes.at(sid);
  // the grid range: the n^3 block, or every slot of a sparse scene (slots
  // outside the current map hold zero)
  const uint64_t cells = s.tile_cap ? 64ull * s.tile_cap
                                    : (uint64_t)s.cfg.grid_size * s.cfg.grid_size * s.cfg.grid_size;
  MPM_CK(launch_totals(pool(), acc_last, s.grid_off, cells, slot_of.ptr, s.id_base, s.n, totals_d.ptr, st));
  eng->launches += 1;
  MPM_CK(cudaMemcpyAsync(out8, totals_d.ptr, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  MPM_CK(cudaStreamSynchronize(st));
}

void Group::status(uint32_t sid, mpm_status_info* out, cudaStream_t st) {
  uint32_t w[kStatusWords];
  MPM_CK(cudaMemcpyAsync(w, status_d.ptr + (size_t)sid * kStatusWords, sizeof(w), cudaMemcpyDeviceToHost, st));
  MPM_CK(cudaStreamSynchronize(st));
  out->fault_bits = w[0];
  out->numerical_fault = (w[0] & kFaultNumerical) ? 1u : 0u;
  // a scene stopped by its substep budget counts one past it (see k_grid_update)
  out->completed_substeps = (w[2] != 0u && w[1] > w[2]) ? w[2] : w[1];
  const SceneHost& s = scenes.at(sid);
  out->active_tiles = s.tile_cap ? std::min(w[3], s.tile_cap) : 0u;
}

void Group::status_words(std::vector<uint32_t>& out, cudaStream_t st) {
  out.resize((size_t)max_scenes * kStatusWords);
  MPM_CK(cudaMemcpyAsync(out.data(), status_d.ptr, out.size() * 4, cudaMemcpyDeviceToHost, st));
  MPM_CK(cudaStreamSynchronize(st));
}

void Group::reset_status(uint32_t sid, cudaStream_t st) {
  records_valid = false;  // the state (or what its records depend on) changes
  MPM_CK(cudaMemsetAsync(status_d.ptr + (size_t)sid * kStatusWords, 0, kStatusWords * 4, st));
  MPM_CK(cudaStreamSynchronize(st));
}

void Group::sort_permutation(uint32_t sid, uint32_t* keys_out, uint32_t* ids_out, uint32_t capacity,
                             cudaStream_t st) {
  const SceneHost& s = scenes.at(sid);
  sync_scenes(st);
  const uint32_t n = s.n;
  if (n) {
    DevBuf<uint32_t> kin(n);
    MPM_CK(launch_scene_keys(pool(), sid, slot_of.ptr, s.id_base, n, kin.ptr, st));
    eng->launches += 1;
    uint32_t* sk = nullptr;
    uint32_t* sv = nullptr;
    MPM_CK(radix_sort_pairs(st, kin.ptr, nullptr, ks[0].ptr, ks[1].ptr, vs[0].ptr, vs[1].ptr, hist.ptr, n,
                            bits_for(s.tiles), &sk, &sv, &eng->launches));
    MPM_CK(cudaMemcpyAsync(keys_out, sk, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    MPM_CK(cudaMemcpyAsync(ids_out, sv, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    MPM_CK(cudaStreamSynchronize(st));
  }
  for (uint32_t i = n; i < capacity; ++i) {
    keys_out[i] = 0xffffffffu;
    ids_out[i] = i;
  }
}

}  // namespace mpm
