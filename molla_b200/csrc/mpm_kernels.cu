// mpm_kernels.cu — grid update, regrouping, work-list and data-movement
// kernels of the B200 MLS-MPM path (the particle kernel is in
// mpm_particles.cu).
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_device.cuh"
#include "mpm_kernels.cuh"

namespace mpm {

namespace {

constexpr int kCellThreads = 256;

__device__ __forceinline__ uint32_t tile_key_of(const SceneDev& sc, float x, float y, float z) {
  // mpm_particle_order.wgsl:17-24: cell = i32(floor((x - o) * inv_dx)) - window,
  // clamped to [0, n-1] per axis; tile = cell / 4; key = tx + w (ty + w tz).
  const float p[3] = {x, y, z};
  const float o[3] = {sc.ox, sc.oy, sc.oz};
  const int win[3] = {sc.winx, sc.winy, sc.winz};
  uint32_t t[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float f = floorf(__fmul_rn(__fsub_rn(p[a], o[a]), sc.inv_dx));
    int c;
    if (!(f == f)) c = 0;
    else if (f >= 2147483520.0f) c = 2147483647;
    else if (f <= -2147483648.0f) c = (int)0x80000000;
    else c = (int)f;
    c -= win[a];
    c = c < 0 ? 0 : c;
    c = c > (int)sc.n - 1 ? (int)sc.n - 1 : c;
    t[a] = (uint32_t)c >> 2;
  }
  return t[0] + sc.w * (t[1] + sc.w * t[2]);
}

}  // namespace

// grid_update (mpm.wgsl:1013-1058) over the grid pool, kGridBlocksPerCta
// 256-cell pool blocks per thread block, one node of each per thread
// (grid_node is the per-node body).  Only blocks the last scatter touched
// (or a rigid sphere may reach) are converted; the blocks touched by the scatter before it are
// cleared in the other accumulator (ready for the next scatter) and
// unmarked.  Counts completed substeps.  The rigid-sphere imprint
// (rigid_imprint, mpm.wgsl:939-1003) is fused in front of the conversion: a
// node inside a sphere takes the sphere's velocity with the heavy-cell mass
// 1e6, its sand mass and momentum give the reaction wrench, and the node is
// marked rigid (negative w in the velocity buffer) so that gravity, walls
// and the implicit sweeps leave it alone.
constexpr int kGridBlocksPerCta = 4;

__device__ __forceinline__ void grid_node(const PoolDev& p, uint32_t sid, const SceneDev& sc, uint64_t blk,
                                          uint64_t g, float4 a, bool in_a, bool rb, int acc_in) {
  const uint32_t n = sc.n;
  const uint32_t local = (uint32_t)(g - sc.grid_off);  // grids hold fewer than 2^32 cells
  int ix, iy, iz;
  if (sc.tile_cap) {
    // sparse storage: node (local & 63) of the tile in slot local / 64
    const uint32_t tile = p.slot_tile[g >> 6];
    const uint32_t tx = tile % sc.w, ty = (tile / sc.w) % sc.w, tz = tile / (sc.w * sc.w);
    ix = 4 * (int)tx + (int)(local & 3u);
    iy = 4 * (int)ty + (int)((local >> 2) & 3u);
    iz = 4 * (int)tz + (int)((local >> 4) & 3u);
  } else {
    const uint32_t q = local / n;
    ix = (int)(local - q * n);
    iy = (int)(q % n);
    iz = (int)(q / n);
  }
  bool rigid = false;
  if (rb && sc.n_rigid) {
    const float node[3] = {sc.ox + (float)(ix + sc.winx) * sc.dx, sc.oy + (float)(iy + sc.winy) * sc.dx,
                           sc.oz + (float)(iz + sc.winz) * sc.dx};
    for (uint32_t r = 0; r < sc.n_rigid; ++r) {
      const RigidDev R = p.rigid[(size_t)sid * kMaxRigid + r];
      const float arm[3] = {node[0] - R.cx, node[1] - R.cy, node[2] - R.cz};
      if (!(sqrtf(arm[0] * arm[0] + arm[1] * arm[1] + arm[2] * arm[2]) < R.radius)) continue;
      const float m_old = a.x;
      const float mom_old[3] = {a.y, a.z, a.w};
      const float stamp = 1.0e6f;
      a = make_float4(stamp, stamp * R.vx, stamp * R.vy, stamp * R.vz);
      p.acc[acc_in][g] = a;
      if (!in_a) p.touched[acc_in][blk] = 1;
      rigid = true;
      if (m_old > 1.0e-9f) {
        const float inv_dt = 1.0f / fmaxf(sc.dt, 1.0e-6f);
        const float f[3] = {-(m_old * R.vx - mom_old[0]) * inv_dt, -(m_old * R.vy - mom_old[1]) * inv_dt,
                            -(m_old * R.vz - mom_old[2]) * inv_dt};
        const float t[3] = {arm[1] * f[2] - arm[2] * f[1], arm[2] * f[0] - arm[0] * f[2], arm[0] * f[1] - arm[1] * f[0]};
        float* w = p.wrench + ((size_t)sid * kMaxRigid + r) * 8;
        atomicAdd(w + 0, f[0]);
        atomicAdd(w + 1, f[1]);
        atomicAdd(w + 2, f[2]);
        atomicAdd(w + 4, t[0]);
        atomicAdd(w + 5, t[1]);
        atomicAdd(w + 6, t[2]);
      }
      break;
    }
  }
  const float m = a.x;
  if (m <= 1.0e-9f || !(m == m)) {
    p.vel[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  float v[3] = {a.y / m, a.z / m, a.w / m};
  if (rigid) {
    p.vel[g] = make_float4(v[0], v[1], v[2], -m);  // skip integration on rigid-imprinted nodes
    return;
  }
  v[1] = v[1] + sc.dt * sc.gy;
  const int pad = sc.pad, nn = (int)n;
  const float f = sc.friction;
  if (sc.sticky) {
    if (ix < pad || ix >= nn - pad || iy < pad || iy >= nn - pad || iz < pad || iz >= nn - pad)
      v[0] = v[1] = v[2] = 0.f;
  } else {
    if (ix < pad) { v[0] = fmaxf(v[0], 0.f); v[1] *= f; v[2] *= f; }
    if (ix >= nn - pad) { v[0] = fminf(v[0], 0.f); v[1] *= f; v[2] *= f; }
    if (iy < pad) { v[1] = fmaxf(v[1], 0.f); v[0] *= f; v[2] *= f; }
    if (iy >= nn - pad) { v[1] = fminf(v[1], 0.f); v[0] *= f; v[2] *= f; }
    if (iz < pad) { v[2] = fmaxf(v[2], 0.f); v[0] *= f; v[1] *= f; }
    if (iz >= nn - pad) { v[2] = fminf(v[2], 0.f); v[0] *= f; v[1] *= f; }
  }
  p.vel[g] = make_float4(v[0], v[1], v[2], m);
}

__global__ void __launch_bounds__(kCellThreads, 5) k_grid_update(PoolDev p, const uint32_t* __restrict__ block_scene,
                                                              uint64_t total_cells, int acc_in, int count_substep) {
  static_assert(kCellThreads == kCellBlock, "one thread per cell of a grid-pool block");
  constexpr int K = kGridBlocksPerCta;
  // Every load of the marks and of the accumulators is issued before any is
  // used, so that a thread keeps K requests in flight.
  uint32_t sid[K];
  bool in_a[K], in_b[K], rb[K], conv[K];
  float4 acc_v[K];
#pragma unroll
  for (int b = 0; b < K; ++b) {
    const uint64_t blk = (uint64_t)blockIdx.x * K + b;
    const bool exists = blk * kCellThreads < total_cells;
    sid[b] = exists ? block_scene[blk] : 0xffffffffu;
    in_a[b] = exists && p.touched[acc_in][blk] != 0;
    in_b[b] = exists && p.touched[acc_in ^ 1][blk] != 0;
    rb[b] = exists && p.rigid_blocks[blk] != 0;
  }
#pragma unroll
  for (int b = 0; b < K; ++b) {
    conv[b] = false;
    if (sid[b] == 0xffffffffu) continue;
    const uint64_t g = ((uint64_t)blockIdx.x * K + b) * kCellThreads + threadIdx.x;
    if (in_b[b]) p.acc[acc_in ^ 1][g] = make_float4(0.f, 0.f, 0.f, 0.f);
    const SceneDev& sc = p.scenes[sid[b]];
    const uint64_t local64 = g - sc.grid_off;
    if (count_substep && local64 == 0) {
      // completed substeps; a scene with a budget counts one past it and
      // stops there (its particle kernels then stand still)
      volatile uint32_t* status = p.status + (size_t)sc.status * kStatusWords;
      if (status[0] == 0u && (status[2] == 0u || status[1] <= status[2]))
        atomicAdd(const_cast<uint32_t*>(status) + 1, 1u);
    }
    // dense: the n^3 block; sparse: the slots of the current tile map
    const uint64_t extent =
        sc.tile_cap ? 64ull * min(*((volatile uint32_t*)p.status + (size_t)sc.status * kStatusWords + 3), sc.tile_cap)
                    : (uint64_t)sc.n * sc.n * sc.n;
    conv[b] = (in_a[b] || rb[b]) && local64 < extent;
    if (conv[b]) acc_v[b] = p.acc[acc_in][g];
  }
  __syncthreads();  // every thread has read the marks
  if (threadIdx.x == 0) {
#pragma unroll
    for (int b = 0; b < K; ++b)
      if (sid[b] != 0xffffffffu && in_b[b]) p.touched[acc_in ^ 1][(uint64_t)blockIdx.x * K + b] = 0;
  }
#pragma unroll
  for (int b = 0; b < K; ++b) {
    if (!conv[b]) continue;
    const uint64_t blk = (uint64_t)blockIdx.x * K + b;
    grid_node(p, sid[b], p.scenes[sid[b]], blk, blk * kCellThreads + threadIdx.x, acc_v[b], in_a[b], rb[b], acc_in);
  }
}

// mpm_rigid_force_integrate (mpm.wgsl:1175-1228): every non-rigid node with
// sand mass within radius + dx of a sphere adds the reaction
// -(m w / dt) (v_sphere - v_node) (w tapered linearly over the outer cell)
// and its torque to the sphere's wrench.
__global__ void __launch_bounds__(kCellThreads) k_rigid_shell(PoolDev p, const uint32_t* __restrict__ block_scene,
                                                              uint64_t total_cells, int acc_in) {
  const uint64_t blk = blockIdx.x;
  if (blk * kCellThreads >= total_cells) return;
  const uint32_t sid = block_scene[blk];
  if (sid == 0xffffffffu || !p.rigid_blocks[blk] || !p.touched[acc_in][blk]) return;
  const SceneDev& sc = p.scenes[sid];
  if (!sc.n_rigid) return;
  const uint64_t g = blk * kCellThreads + threadIdx.x;
  const uint64_t local64 = g - sc.grid_off;
  const uint32_t n = sc.n;
  if (local64 >= (uint64_t)n * n * n) return;
  const float m = p.acc[acc_in][g].x;
  if (m <= 1.0e-9f || !(m == m)) return;
  const float4 vg = p.vel[g];
  if (vg.w < 0.f) return;  // rigid-stamped node
  const uint32_t local = (uint32_t)local64;
  const uint32_t q = local / n;
  const int ix = (int)(local - q * n), iy = (int)(q % n), iz = (int)(q / n);
  const float node[3] = {sc.ox + (float)(ix + sc.winx) * sc.dx, sc.oy + (float)(iy + sc.winy) * sc.dx,
                         sc.oz + (float)(iz + sc.winz) * sc.dx};
  for (uint32_t r = 0; r < sc.n_rigid; ++r) {
    const RigidDev R = p.rigid[(size_t)sid * kMaxRigid + r];
    const float arm[3] = {node[0] - R.cx, node[1] - R.cy, node[2] - R.cz};
    const float d = sqrtf(arm[0] * arm[0] + arm[1] * arm[1] + arm[2] * arm[2]);
    if (d > R.radius + sc.dx) continue;
    float w = 1.0f;
    if (d > R.radius) w = fmaxf(0.0f, 1.0f - (d - R.radius) / sc.dx);
    const float k = -(m * w / fmaxf(sc.dt, 1.0e-6f));
    const float f[3] = {k * (R.vx - vg.x), k * (R.vy - vg.y), k * (R.vz - vg.z)};
    const float t[3] = {arm[1] * f[2] - arm[2] * f[1], arm[2] * f[0] - arm[0] * f[2], arm[0] * f[1] - arm[1] * f[0]};
    float* wr = p.wrench + ((size_t)sid * kMaxRigid + r) * 8;
    atomicAdd(wr + 0, f[0]);
    atomicAdd(wr + 1, f[1]);
    atomicAdd(wr + 2, f[2]);
    atomicAdd(wr + 4, t[0]);
    atomicAdd(wr + 5, t[1]);
    atomicAdd(wr + 6, t[2]);
  }
}

// One semi-implicit Jacobi sweep on the grid velocity (mpm_implicit_apply,
// mpm.wgsl:1060-1164), src -> dst, over the blocks the last scatter touched:
// a node with mass m blends its velocity with the mean velocity of its
// face neighbours that carry mass, v = (m v + a v_avg) / (m + a), with
// a = dt^2 m c^2 / dx^2 and c^2 = E / 1500 (the reference's wave-speed
// stiffness estimate); massless nodes and scenes whose sweeps are done copy.
__global__ void __launch_bounds__(kCellThreads) k_grid_jacobi(PoolDev p, const uint32_t* __restrict__ block_scene,
                                                              uint64_t total_cells, int acc_in,
                                                              const float4* __restrict__ src, float4* __restrict__ dst,
                                                              uint32_t sweep) {
  const uint64_t blk = blockIdx.x;
  if (blk * kCellThreads >= total_cells) return;
  const uint32_t sid = block_scene[blk];
  if (sid == 0xffffffffu || !p.touched[acc_in][blk]) return;
  const uint64_t g = blk * kCellThreads + threadIdx.x;
  const SceneDev& sc = p.scenes[sid];
  const uint64_t local64 = g - sc.grid_off;
  const uint32_t n = sc.n;
  if (local64 >= (uint64_t)n * n * n) return;
  const float4 cur = src[g];
  const float m = p.acc[acc_in][g].x;
  // massless, rigid-stamped (negative w) or done: copy through
  if (sweep >= sc.jacobi_iters || m <= 1.0e-9f || !(m == m) || cur.w < 0.f) {
    dst[g] = cur;
    return;
  }
  const uint32_t local = (uint32_t)local64;
  const uint32_t q = local / n;
  const int ix = (int)(local - q * n), iy = (int)(q % n), iz = (int)(q / n);
  const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  float ax = 0.f, ay = 0.f, az = 0.f, count = 0.f;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int nx = ix + off[k][0], ny = iy + off[k][1], nz = iz + off[k][2];
    if ((unsigned)nx >= n || (unsigned)ny >= n || (unsigned)nz >= n) continue;
    const uint64_t ng = sc.grid_off + (uint64_t)nx + (uint64_t)n * ((uint64_t)ny + (uint64_t)n * (uint64_t)nz);
    const float nm = p.acc[acc_in][ng].x;
    if (nm <= 1.0e-9f || !(nm == nm)) continue;
    const float4 nv = src[ng];
    ax = ax + nv.x;
    ay = ay + nv.y;
    az = az + nv.z;
    count = count + 1.0f;
  }
  if (count > 0.f) {
    ax = ax / count;
    ay = ay / count;
    az = az / count;
  } else {
    ax = cur.x;
    ay = cur.y;
    az = cur.z;
  }
  const float c2 = sc.youngs / 1500.0f;
  const float alpha = sc.dt * sc.dt * m * c2 * sc.inv_dx * sc.inv_dx;
  const float denom = m + alpha;
  const float vx = (m * cur.x + alpha * ax) / denom, vy = (m * cur.y + alpha * ay) / denom,
              vz = (m * cur.z + alpha * az) / denom;
  const bool nan = !(vx == vx) || !(vy == vy) || !(vz == vz);
  dst[g] = nan ? make_float4(cur.x, cur.y, cur.z, m) : make_float4(vx, vy, vz, m);
}

// dst <- src over the touched blocks (the last Jacobi sweep's result back into
// the velocity buffer the gather reads).
__global__ void __launch_bounds__(kCellThreads) k_vel_copy(const uint8_t* __restrict__ touched,
                                                           const uint32_t* __restrict__ block_scene,
                                                           uint64_t total_cells, const float4* __restrict__ src,
                                                           float4* __restrict__ dst) {
  const uint64_t blk = blockIdx.x;
  if (blk * kCellThreads >= total_cells) return;
  if (block_scene[blk] == 0xffffffffu || !touched[blk]) return;
  const uint64_t g = blk * kCellThreads + threadIdx.x;
  dst[g] = src[g];
}

// Sort keys of the live slots (tile_keys, mpm_particle_order.wgsl:11-25)
// written at the particle's identity.
__global__ void k_keys(PoolDev p, uint32_t n_slots) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const SceneDev& sc = p.scenes[p.meta[s] >> 8];
  if (!sc.live) {
    // Particles of a removed scene sort behind every live key.
    p.keys_by_id[p.orig[s]] = 0xffffffffu;
    return;
  }
  const float pos[3] = {plane(p, PX)[s], plane(p, PY)[s], plane(p, PZ)[s]};
  const float o[3] = {sc.ox, sc.oy, sc.oz};
  const int win[3] = {sc.winx, sc.winy, sc.winz};
  uint32_t t[3], c[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float xp = (pos[a] - o[a]) * sc.inv_dx;
    const float bf = floorf(xp - 0.5f);
    int b = (xp == xp) ? (int)bf - win[a] : 0;
    b = b < 0 ? 0 : b;
    b = b > (int)sc.n - 1 ? (int)sc.n - 1 : b;
    t[a] = (uint32_t)b >> 2;
    c[a] = (uint32_t)b & 3u;
  }
  const uint32_t tile = t[0] + sc.w * (t[1] + sc.w * t[2]);
  p.keys_by_id[p.orig[s]] = ((sc.key_off + tile) << kCellBits) | c[0] | (c[1] << 2) | (c[2] << 4);
}

// set_particles_with_velocity (mpm.rs:1458-1519) into pool slots
// [slot0, slot0 + n): F = I, C = 0, jp = 0, v = vel or 0, mass/volume per
// particle or uniform, identities id0 + i.
__global__ void k_init_particles(PoolDev p, uint32_t* __restrict__ slot_of, uint32_t slot0, uint32_t id0, uint32_t n,
                                 const float* __restrict__ xyz, const float* __restrict__ vel,
                                 const float* __restrict__ mass, const float* __restrict__ vol, float mass0,
                                 float vol0, const uint32_t* __restrict__ mat_ids, uint32_t scene) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = slot0 + i;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    plane(p, PX + a)[s] = xyz[3 * (size_t)i + a];
    plane(p, VX + a)[s] = vel ? vel[3 * (size_t)i + a] : 0.f;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    plane(p, C0 + k)[s] = 0.f;
    plane(p, F0 + k)[s] = (k % 4 == 0) ? 1.f : 0.f;
  }
  plane(p, MASS)[s] = mass ? mass[i] : mass0;
  plane(p, VOL)[s] = vol ? vol[i] : vol0;
  plane(p, JP)[s] = 0.f;
  p.meta[s] = (scene << 8) | (mat_ids ? (mat_ids[i] & 7u) : 0u);
  p.orig[s] = id0 + i;
  slot_of[id0 + i] = s;
}

// set_materials (mpm.rs:1589-1621): material row ids in identity order.
__global__ void k_set_material_ids(PoolDev p, const uint32_t* __restrict__ slot_of, uint32_t id0, uint32_t n,
                                   const uint32_t* __restrict__ ids) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = slot_of[id0 + i];
  p.meta[s] = (p.meta[s] & ~0xffu) | (ids ? (ids[i] & 7u) : 0u);
}

// Tile keys of one scene's particles in identity order (no scene offset).
__global__ void k_scene_keys(PoolDev p, uint32_t sid, const uint32_t* __restrict__ slot_of, uint32_t id0, uint32_t n,
                             uint32_t* __restrict__ keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SceneDev& sc = p.scenes[sid];
  const uint32_t s = slot_of[id0 + i];
  keys[i] = tile_key_of(sc, plane(p, PX)[s], plane(p, PY)[s], plane(p, PZ)[s]);
}

// Physically regroup particles into sorted order: slot s of the new pool
// receives identity ids[s].
__global__ void k_reorder(const float* __restrict__ src, float* __restrict__ dst, uint32_t cap,
                          const uint32_t* __restrict__ meta_src, uint32_t* __restrict__ meta_dst,
                          uint32_t* __restrict__ orig_dst, uint32_t* __restrict__ slot_of,
                          const uint32_t* __restrict__ ids, const uint32_t* __restrict__ keys,
                          uint32_t* __restrict__ slot_key, const float4* __restrict__ rec_src,
                          float4* __restrict__ rec_dst, uint32_t n_live) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_live) return;
  const uint32_t id = ids[s];
  slot_key[s] = keys[s];
  const uint32_t old = slot_of[id];
  if (rec_src) {
#pragma unroll
    for (int k = 0; k < 4; ++k) rec_dst[4 * (size_t)s + k] = rec_src[4 * (size_t)old + k];
  }
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) dst[(size_t)k * cap + s] = src[(size_t)k * cap + old];
  meta_dst[s] = meta_src[old];
  orig_dst[s] = id;
  slot_of[id] = s;
}

// tile_start[t] = first sorted position whose key is >= t, for t in [0, K].
__global__ void k_tile_start(const uint32_t* __restrict__ sorted_keys, uint32_t n_live, uint32_t K, int shift,
                             uint32_t* __restrict__ tile_start) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > K) return;
  uint32_t lo = 0, hi = n_live;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if ((sorted_keys[mid] >> shift) < t) lo = mid + 1;
    else hi = mid;
  }
  tile_start[t] = lo;
}

// Work items: every occupied tile, cut into chunks of at most `chunk` slots.
// key_scene gives the scene of every tile key (each scene holds a stable
// range of the key space).  Items of FP32-SVD scenes take slots from 0 up
// (count n_items[0]), items of FP64-SVD scenes slots from item_top - 1 down
// (count n_items[1]), so that the gather of each SVD form is one launch over
// a contiguous range.
__global__ void k_items(const uint32_t* __restrict__ tile_start, uint32_t K, const uint32_t* __restrict__ key_scene,
                        const SceneDev* __restrict__ scenes, uint32_t chunk, uint32_t item_top,
                        Item* __restrict__ items, uint32_t* __restrict__ n_items, uint32_t* __restrict__ tile_item) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= K) return;
  const uint32_t a = tile_start[t], b = tile_start[t + 1];
  if (b <= a) return;
  const uint32_t scene = key_scene[t];
  if (scene == 0xffffffffu) return;  // no live scene holds this key (cannot carry particles)
  const uint32_t cnt = b - a;
  chunk = chunk ? chunk : cnt;
  const uint32_t pieces = (cnt + chunk - 1) / chunk;
  const bool up = scenes[scene].svd64 == 0u;
  const uint32_t base = atomicAdd(&n_items[up ? 0 : 1], pieces);
  for (uint32_t i = 0; i < pieces; ++i) {
    Item it;
    it.start = a + i * chunk;
    it.count = min(chunk, cnt - i * chunk);
    it.scene = scene;
    it.tile = t - scenes[scene].key_off;
    const uint32_t slot = up ? base + i : item_top - 1u - (base + i);
    items[slot] = it;
    if (tile_item && i == 0) tile_item[t] = slot;
  }
}

// One 64-thread block per item: the table that gives the scatter's deposit
// its cell for each of 64 slots.  Slots 10w..10w+9 are warp w's cells (three
// adjacent lanes each, one per x-slab), slots 60..63 the spare lanes'.
// A cell's flush atomics use the shared-memory banks b, b+1, b+2 (b the bank
// of its node row, region_index(x+1, y+1, z+1) mod 32), and every b is the
// bank of exactly two of the tile's 64 cells.  Cells with b in 0..29 fall
// into three classes by b mod 3; within a class the runs of the ten b values
// tile 30 banks without overlap, so the class's two warps take one cell of
// each b (the one with more particles to the first warp), and a warp's 30
// flush atomics of one node and channel fall on 30 different banks.  Inside
// a warp the cells are in the order of their particle counts (thread c
// counts cell c in the item's slot keys, sorted by cell within a tile, by
// binary search).  The four cells with b of 30 or 31 go to the spare lanes.
__device__ __forceinline__ void item_order_one(const Item* __restrict__ items, uint32_t it,
                                               const uint32_t* __restrict__ slot_key, uint8_t* __restrict__ item_order,
                                               uint32_t (&s_cnt)[64], uint8_t (&s_pair)[32][2],
                                               uint32_t (&s_fill)[32]) {
  const Item item = items[it];
  const uint32_t c = threadIdx.x;
  const uint32_t* keys = slot_key + item.start;
  auto lower = [&](uint32_t cell) {
    uint32_t lo = 0, hi = item.count;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if ((keys[mid] & 63u) < cell) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  if (c < 32) s_fill[c] = 0;
  s_cnt[c] = (c == 63 ? item.count : lower(c + 1)) - lower(c);
  __syncthreads();
  static_assert(kRsy == 8 && kRsz % 32 == 4, "with these strides every bank is the row bank of two core cells");
  const uint32_t bank = (((c & 3u) + 1u) + kRsy * (((c >> 2) & 3u) + 1u) + kRsz * ((c >> 4) + 1u)) & 31u;
  const uint32_t slot = atomicAdd(&s_fill[bank], 1u);
  if (slot < 2u) s_pair[bank][slot] = (uint8_t)c;
  __syncthreads();
  if (c < 4) {
    uint8_t* out = item_order + (size_t)it * 64;
    uint8_t a[10], b[10];
    uint32_t n = 0;
    auto more = [&](uint8_t x, uint8_t y) {  // x before y: more particles, then lower index
      return s_cnt[x] > s_cnt[y] || (s_cnt[x] == s_cnt[y] && x < y);
    };
    auto sort = [&](uint8_t* v, uint32_t len) {
      for (uint32_t i = 1; i < len; ++i)
        for (uint32_t j = i; j > 0 && more(v[j], v[j - 1]); --j) {
          const uint8_t t = v[j];
          v[j] = v[j - 1];
          v[j - 1] = t;
        }
    };
    if (c < 3) {
      for (uint32_t bb = c; bb < 30; bb += 3, ++n) {
        const uint8_t x = s_pair[bb][0], y = s_pair[bb][1];
        a[n] = more(x, y) ? x : y;
        b[n] = more(x, y) ? y : x;
      }
      sort(a, 10);
      sort(b, 10);
      for (uint32_t i = 0; i < 10; ++i) {
        out[20 * c + i] = a[i];
        out[20 * c + 10 + i] = b[i];
      }
    } else {
      a[0] = s_pair[30][0];
      a[1] = s_pair[30][1];
      a[2] = s_pair[31][0];
      a[3] = s_pair[31][1];
      sort(a, 4);
      for (uint32_t i = 0; i < 4; ++i) out[60 + i] = a[i];
    }
  }
}

// Grid-stride over the work list's items (the FP32-SVD items, then the
// FP64-SVD ones at the top of the slot range), so that only the items that
// exist are visited.
__global__ void __launch_bounds__(64) k_item_order(const Item* __restrict__ items,
                                                   const uint32_t* __restrict__ n_items, uint32_t item_top,
                                                   const uint32_t* __restrict__ slot_key,
                                                   uint8_t* __restrict__ item_order) {
  __shared__ uint32_t s_cnt[64];
  __shared__ uint8_t s_pair[32][2];
  __shared__ uint32_t s_fill[32];
  const uint32_t n32 = n_items[0], total = n32 + n_items[1];
  for (uint32_t li = blockIdx.x; li < total; li += gridDim.x) {
    const uint32_t it = li < n32 ? li : item_top - 1u - (li - n32);
    item_order_one(items, it, slot_key, item_order, s_cnt, s_pair, s_fill);
    __syncthreads();  // the shared tables are reused by the next item
  }
}

// Copy one scene's positions / velocities (3 planes from `first`) into a
// packed xyz buffer in identity order.
__global__ void k_gather_xyz(PoolDev p, int first, const uint32_t* __restrict__ slot_of, uint32_t id_base,
                             uint32_t n, float* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = slot_of[id_base + i];
  out[3 * (size_t)i] = plane(p, first)[s];
  out[3 * (size_t)i + 1] = plane(p, first + 1)[s];
  out[3 * (size_t)i + 2] = plane(p, first + 2)[s];
}

// Render view (mpm_render_view.rs:20-44, position write mpm.wgsl:1349):
// one scene's positions as float4 (xyz, w = 0) in identity order.  Coalesced
// 16-byte stores; the plane reads follow slot_of.
__global__ void k_pack_positions(PoolDev p, const uint32_t* __restrict__ slot_of, uint32_t id_base, uint32_t n,
                                 float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = slot_of[id_base + i];
  out[i] = make_float4(plane(p, PX)[s], plane(p, PX + 1)[s], plane(p, PX + 2)[s], 0.0f);
}

// Copy `count` planes starting at `first` into [n x count] rows in identity order.
__global__ void k_gather_rows(PoolDev p, int first, int count, const uint32_t* __restrict__ slot_of,
                              uint32_t id_base, uint32_t n, float* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = slot_of[id_base + i];
  for (int k = 0; k < count; ++k) out[(size_t)count * i + k] = plane(p, first + k)[s];
}

// Inverse of k_gather_rows (host-provided state in identity order).
__global__ void k_scatter_rows(PoolDev p, int first, int count, const uint32_t* __restrict__ slot_of,
                               uint32_t id_base, uint32_t n, const float* __restrict__ in) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = slot_of[id_base + i];
  for (int k = 0; k < count; ++k) plane(p, first + k)[s] = in[(size_t)count * i + k];
}

// FP64 conservation totals of one scene: grid mass + momentum of the last
// scatter, particle mass + momentum.  out[8] must be zeroed.
__global__ void k_totals(PoolDev p, int acc_idx, uint64_t grid_off, uint64_t cells,
                         const uint32_t* __restrict__ slot_of, uint32_t id_base, uint32_t n,
                         double* __restrict__ out) {
  double g[4] = {0, 0, 0, 0}, q[4] = {0, 0, 0, 0};
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += stride) {
    const float4 a = p.acc[acc_idx][grid_off + i];
    g[0] += a.x;
    g[1] += a.y;
    g[2] += a.z;
    g[3] += a.w;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t s = slot_of[id_base + (uint32_t)i];
    const double m = plane(p, MASS)[s];
    q[0] += m;
    q[1] += m * plane(p, VX)[s];
    q[2] += m * plane(p, VY)[s];
    q[3] += m * plane(p, VZ)[s];
  }
  double vals[8] = {g[0], g[1], g[2], g[3], q[0], q[1], q[2], q[3]};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double x = vals[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[k], x);
  }
}

// ---------------------------------------------------------------------------
// Host launchers.

cudaError_t launch_grid_update(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               int count_substep, cudaStream_t st) {
  const uint64_t pool_blocks = (total_cells + kCellThreads - 1) / kCellThreads;
  const uint64_t blocks = (pool_blocks + kGridBlocksPerCta - 1) / kGridBlocksPerCta;
  if (blocks == 0) return cudaSuccess;
  k_grid_update<<<(unsigned)blocks, kCellThreads, 0, st>>>(p, block_scene, total_cells, acc_in, count_substep);
  return cudaGetLastError();
}

cudaError_t launch_grid_jacobi(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               const float4* src, float4* dst, uint32_t sweep, cudaStream_t st) {
  const uint64_t blocks = (total_cells + kCellThreads - 1) / kCellThreads;
  if (blocks == 0) return cudaSuccess;
  k_grid_jacobi<<<(unsigned)blocks, kCellThreads, 0, st>>>(p, block_scene, total_cells, acc_in, src, dst, sweep);
  return cudaGetLastError();
}

cudaError_t launch_rigid_shell(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               cudaStream_t st) {
  const uint64_t blocks = (total_cells + kCellThreads - 1) / kCellThreads;
  if (blocks == 0) return cudaSuccess;
  k_rigid_shell<<<(unsigned)blocks, kCellThreads, 0, st>>>(p, block_scene, total_cells, acc_in);
  return cudaGetLastError();
}

cudaError_t launch_vel_copy(const uint8_t* touched, const uint32_t* block_scene, uint64_t total_cells,
                            const float4* src, float4* dst, cudaStream_t st) {
  const uint64_t blocks = (total_cells + kCellThreads - 1) / kCellThreads;
  if (blocks == 0) return cudaSuccess;
  k_vel_copy<<<(unsigned)blocks, kCellThreads, 0, st>>>(touched, block_scene, total_cells, src, dst);
  return cudaGetLastError();
}

cudaError_t launch_keys(const PoolDev& p, uint32_t n_slots, cudaStream_t st) {
  if (!n_slots) return cudaSuccess;
  k_keys<<<(n_slots + 255) / 256, 256, 0, st>>>(p, n_slots);
  return cudaGetLastError();
}

cudaError_t launch_init_particles(const PoolDev& p, uint32_t* slot_of, uint32_t slot0, uint32_t id0, uint32_t n,
                                  const float* xyz, const float* vel, const float* mass, const float* vol,
                                  float mass0, float vol0, const uint32_t* mat_ids, uint32_t scene, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_init_particles<<<(n + 255) / 256, 256, 0, st>>>(p, slot_of, slot0, id0, n, xyz, vel, mass, vol, mass0, vol0,
                                                    mat_ids, scene);
  return cudaGetLastError();
}

cudaError_t launch_set_material_ids(const PoolDev& p, const uint32_t* slot_of, uint32_t id0, uint32_t n,
                                    const uint32_t* ids, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_set_material_ids<<<(n + 255) / 256, 256, 0, st>>>(p, slot_of, id0, n, ids);
  return cudaGetLastError();
}

cudaError_t launch_scene_keys(const PoolDev& p, uint32_t sid, const uint32_t* slot_of, uint32_t id0, uint32_t n,
                              uint32_t* keys, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_scene_keys<<<(n + 255) / 256, 256, 0, st>>>(p, sid, slot_of, id0, n, keys);
  return cudaGetLastError();
}

cudaError_t launch_reorder(const float* src, float* dst, uint32_t cap, const uint32_t* meta_src, uint32_t* meta_dst,
                           uint32_t* orig_dst, uint32_t* slot_of, const uint32_t* ids, const uint32_t* keys,
                           uint32_t* slot_key, const float4* rec_src, float4* rec_dst, uint32_t n_live,
                           cudaStream_t st) {
  if (!n_live) return cudaSuccess;
  k_reorder<<<(n_live + 255) / 256, 256, 0, st>>>(src, dst, cap, meta_src, meta_dst, orig_dst, slot_of, ids, keys,
                                                  slot_key, rec_src, rec_dst, n_live);
  return cudaGetLastError();
}

cudaError_t launch_items(const uint32_t* sorted_keys, int shift, uint32_t n_live, uint32_t K, uint32_t* tile_start,
                         const uint32_t* key_scene, const SceneDev* scenes, uint32_t chunk, uint32_t item_top,
                         Item* items, uint32_t* n_items, uint32_t* tile_item, cudaStream_t st) {
  cudaMemsetAsync(n_items, 0, 2 * sizeof(uint32_t), st);
  if (tile_item) cudaMemsetAsync(tile_item, 0xff, (size_t)(K + 1) * sizeof(uint32_t), st);
  k_tile_start<<<(K + 1 + 255) / 256, 256, 0, st>>>(sorted_keys, n_live, K, shift, tile_start);
  if (K > 0)
    k_items<<<(K + 255) / 256, 256, 0, st>>>(tile_start, K, key_scene, scenes, chunk, item_top, items, n_items,
                                             tile_item);
  return cudaGetLastError();
}

// Sparse tile maps (the reference marks the active tiles and builds its
// hashed map every step, crates/molla-solvers/src/mpm_active_tiles.rs:242-302):
// the active-tile counters of the sparse scenes start at zero ...
__global__ void k_tiles_reset(PoolDev p, uint32_t n_scenes) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_scenes; s += gridDim.x * blockDim.x) {
    const SceneDev& sc = p.scenes[s];
    if (sc.live && sc.tile_cap) p.status[(size_t)sc.status * kStatusWords + 3] = 0u;
  }
}

// ... then every tile the gather marked gets a slot (slot order is
// immaterial: each tile owns its 64 nodes), every other tile none, and the
// marks are cleared.  More active tiles than the capacity latch
// kFaultTileOverflow; the excess tiles get no slot (their deposits are
// dropped and the scene freezes from the next substep).
__global__ void k_tiles_finalize(PoolDev p, const uint32_t* __restrict__ key_scene, uint32_t K) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= K) return;
  const uint32_t sid = key_scene[t];
  if (sid == 0xffffffffu) return;
  const SceneDev& sc = p.scenes[sid];
  if (!sc.tile_cap || !sc.live) return;
  uint32_t slot = kNoSlot;
  if (p.tile_mark[t]) {
    p.tile_mark[t] = 0;
    uint32_t* status = p.status + (size_t)sc.status * kStatusWords;
    const uint32_t s = atomicAdd(status + 3, 1u);
    if (s < sc.tile_cap) {
      slot = s;
      p.slot_tile[(sc.grid_off >> 6) + s] = t - sc.key_off;
    } else {
      atomicOr(status, kFaultTileOverflow);
    }
  }
  p.tile_slot[t] = slot;
}

cudaError_t launch_tiles_finalize(const PoolDev& p, const uint32_t* key_scene, uint32_t K, uint32_t n_scenes,
                                  cudaStream_t st) {
  k_tiles_reset<<<(n_scenes + 255) / 256, 256, 0, st>>>(p, n_scenes);
  if (K) k_tiles_finalize<<<(K + 255) / 256, 256, 0, st>>>(p, key_scene, K);
  return cudaGetLastError();
}

__global__ void k_fill_u32(uint32_t* __restrict__ p, uint64_t n, uint32_t v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

cudaError_t launch_fill_u32(uint32_t* p, uint64_t n, uint32_t v, cudaStream_t st) {
  if (!n) return cudaSuccess;
  const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 4096);
  k_fill_u32<<<(unsigned)blocks, 256, 0, st>>>(p, n, v);
  return cudaGetLastError();
}

cudaError_t launch_item_order(const Item* items, const uint32_t* n_items, uint32_t item_top, const uint32_t* slot_key,
                              uint8_t* item_order, cudaStream_t st) {
  if (!item_top) return cudaSuccess;
  k_item_order<<<std::min<uint32_t>(item_top, 148u * 32u), 64, 0, st>>>(items, n_items, item_top, slot_key,
                                                                        item_order);
  return cudaGetLastError();
}

cudaError_t launch_gather_xyz(const PoolDev& p, int first, const uint32_t* slot_of, uint32_t id_base, uint32_t n,
                              float* out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_gather_xyz<<<(n + 255) / 256, 256, 0, st>>>(p, first, slot_of, id_base, n, out);
  return cudaGetLastError();
}

cudaError_t launch_pack_positions(const PoolDev& p, const uint32_t* slot_of, uint32_t id_base, uint32_t n,
                                  float4* out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_pack_positions<<<(n + 255) / 256, 256, 0, st>>>(p, slot_of, id_base, n, out);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const PoolDev& p, int first, int count, const uint32_t* slot_of, uint32_t id_base,
                               uint32_t n, float* out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_gather_rows<<<(n + 255) / 256, 256, 0, st>>>(p, first, count, slot_of, id_base, n, out);
  return cudaGetLastError();
}

cudaError_t launch_scatter_rows(const PoolDev& p, int first, int count, const uint32_t* slot_of, uint32_t id_base,
                                uint32_t n, const float* in, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_scatter_rows<<<(n + 255) / 256, 256, 0, st>>>(p, first, count, slot_of, id_base, n, in);
  return cudaGetLastError();
}

cudaError_t launch_totals(const PoolDev& p, int acc_idx, uint64_t grid_off, uint64_t cells, const uint32_t* slot_of,
                          uint32_t id_base, uint32_t n, double* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, 8 * sizeof(double), st);
  k_totals<<<296, 256, 0, st>>>(p, acc_idx, grid_off, cells, slot_of, id_base, n, out);
  return cudaGetLastError();
}

}  // namespace mpm
