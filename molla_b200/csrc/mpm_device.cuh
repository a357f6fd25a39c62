// mpm_device.cuh — device-side data layout and per-particle physics of the
// B200 MLS-MPM substep.
//
// Layout (HBM):
//   * particles: a pool of structure-of-arrays planes, one float plane per
//     scalar (x, y, z, vx, vy, vz, C[9], F[9], mass, volume, jp), each plane
//     `cap` floats long, so that every per-particle access of a warp is one
//     coalesced 128-byte transaction.  Matrices are column-major per
//     particle (plane C0 + 3*col + row), the WGSL mat3x3 order of
//     crates/molla-solvers/shaders/mpm.wgsl:116-118.  Particles are kept
//     physically grouped by 4^3 grid tile; `orig` maps a slot to the
//     particle's identity and `slot_of` maps back.
//   * grid: per cell one float4 accumulator (mass, momentum xyz), double
//     buffered, and one float4 velocity (vx, vy, vz, mass) written by the grid
//     update.  Cells of all scenes of a group live in one pool.
//   * scenes: one SceneDev record per scene (constants of the substep).
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace mpm {

constexpr int kPlanes = 27;
enum Plane : int {
  PX = 0, PY = 1, PZ = 2,
  VX = 3, VY = 4, VZ = 5,
  C0 = 6,   // C[col*3+row] in planes 6..14
  F0 = 15,  // F[col*3+row] in planes 15..23
  MASS = 24, VOL = 25, JP = 26
};

constexpr uint32_t kFaultNumerical = 2u;  // mpm.wgsl:229 numerical_fault()
// Status words per scene: [fault bits, completed substeps, substep budget
// (0 = unlimited), spare].  A scene with a budget stops after that many
// substeps: the grid update counts one past the budget and stops counting,
// and the particle kernels skip a scene whose count is past its budget.
constexpr uint32_t kStatusWords = 4u;
// Status word 3 of a sparse scene counts its active tiles (the slots of the
// current map).
constexpr uint32_t kFaultTileOverflow = 16u;  // more active tiles than the sparse scene's capacity
constexpr uint32_t kNoSlot = 0xffffffffu;
constexpr int kMaxMaterials = 8;          // MAX_MPM_MATERIALS, mpm.rs:660

// Work items cover the particles regrouped under one 4^3 tile of base cells
// (base = floor(x/dx - 0.5), the lowest node of the quadratic stencil).  A
// particle whose base lies in tile t touches nodes [4t, 4t+5]; the item
// accumulates in a shared-memory block of 8^3 nodes starting at 4t - 1, which
// leaves one cell of drift on each side for particles that moved since the
// last regrouping.  Anything further out is deposited with global atomics.
// Node (lx, ly, lz) of the block lives at lx + 8 ly + 68 lz: the 68-float z
// stride maps a 4x4x2 block of distinct nodes onto 32 distinct banks.
constexpr int kRegion = 8;
constexpr int kRegionNodes = kRegion * kRegion * kRegion;
constexpr int kRsy = 8;
constexpr int kRsz = 68;
constexpr int kRegionFloats = kRsz * kRegion;  // 544
// Bits of the cell-in-tile part of the regroup key (tile, cell).
constexpr int kCellBits = 6;

struct MatDev {
  int32_t rheo;      // 0 sand, 1 snow, 2 viscous (mpm.wgsl:556-557)
  float mu, lam;     // mpm.wgsl:550-551 (per row when the row overrides E/nu)
  float kappa;       // (3 lam + 2 mu) / (2 mu), mpm.wgsl:1441
  float dp_alpha;    // material_row, mpm.rs:665-668
  float theta_c, theta_s, hardening;
  float vfac, afac;  // exp(-max(damping,0) dt), mpm.wgsl:1306-1307
  float pad0, pad1;
};

struct SceneDev {
  uint32_t n;        // grid cells per axis
  uint32_t w;        // tiles per axis, ceil(n/4)
  uint32_t key_off;  // first key of this scene in the group key space
  uint32_t status;   // index of this scene's status words
  uint64_t grid_off; // first cell of this scene in the grid pool
  float dx, inv_dx;
  float ox, oy, oz;
  int32_t winx, winy, winz;
  float dt, gy, friction;
  int32_t pad, sticky;
  float lo[3], hi[3];  // g2p position clamp bounds (mpm.wgsl:1323-1326)
  uint32_t n_mat;
  uint32_t id_base;    // first identity of this scene
  uint32_t n_particles;
  uint32_t live;       // 0 once the scene was removed (its particles leave at the next regroup)
  uint32_t jacobi_iters;  // semi-implicit sweeps per substep (MpmTimeStep::Implicit), 0 explicit
  float youngs;           // the configuration's Young's modulus (implicit stiffness estimate)
  uint32_t n_rigid;       // rigid spheres of this scene (slots scene * kMaxRigid ...)
  uint32_t svd64;         // 1: the mixed-precision (FP64) SVD and principal-frame stress, 0: the FP32 reference form
  // Sparse grid storage (MpmSimulation::new_sparse, mpm.rs:846-853): 0 keeps
  // the dense n^3 grid; otherwise the scene's grid range holds tile_cap
  // 4^3-node tiles, and the tile map (tile_slot, by tile key) gives each
  // active tile its slot.  The map is rebuilt every substep from the tiles
  // the particles' stencils touch; more active tiles than tile_cap latch
  // kFaultTileOverflow.
  uint32_t tile_cap;
  uint32_t pad_sparse;
  MatDev mat[kMaxMaterials];
};

// A rigid sphere coupled to a scene (set_rigid_spheres, mpm.rs:1521-1565):
// center, radius and linear velocity.
constexpr int kMaxRigid = 8;
struct RigidDev {
  float cx, cy, cz, radius;
  float vx, vy, vz, pad;
};

// A work item: `count` consecutive particle slots starting at `start`, all
// belonging to `scene` and regrouped under local tile `tile`.
struct Item {
  uint32_t start, count, scene, tile;
};

// Everything a particle/grid kernel needs, passed by value.
struct PoolDev {
  float* planes;        // kPlanes * cap floats
  uint32_t cap;
  uint32_t* meta;       // scene << 8 | material id, per slot
  uint32_t* orig;       // identity per slot
  uint32_t* keys_by_id; // sort key per identity (written when a regroup is due)
  float4* acc[2];       // grid accumulators (mass, momentum)
  uint8_t* touched[2];  // per 256-cell block of the grid pool: acc[i] holds deposits there
  const uint8_t* rigid_blocks;  // per 256-cell block: a rigid sphere may reach it
  const RigidDev* rigid;        // kMaxRigid per scene
  float* wrench;                // 8 floats per sphere slot: force xyz, 0, torque xyz, 0
  float4* vel;          // grid velocity (vx, vy, vz, mass)
  float* rec;           // per slot 16 floats: (x, y, z, m), (m v, B0), (B1..B4), (B5..B8)
  const uint32_t* slot_key;  // regroup key of each slot: (tile << 6) | cell in tile
  const SceneDev* scenes;
  uint32_t* status;     // kStatusWords per scene
  // Work list: items of FP32-SVD scenes fill it from slot 0 up (count
  // n_items[0]), items of FP64-SVD scenes from slot item_top - 1 down (count
  // n_items[1]), so that each SVD form is one contiguous range of logical
  // item indices (item_slot).
  const Item* items;
  const uint32_t* n_items;
  uint32_t item_top;
  const uint8_t* item_order;  // per item: its tile's 64 cells by descending count at the regrouping
  // Sparse grid storage: slot of every tile key (kNoSlot: none), the tile
  // (scene-local index) of every slot of the grid pool (indexed by grid pool
  // cell / 64), and the tiles marked by this substep's gather.
  uint32_t* tile_slot;
  uint32_t* slot_tile;
  uint8_t* tile_mark;
  // Item counters of the persistent particle kernels (0: gather, 1:
  // scatter), zeroed before each launch: a CTA takes its first item by its
  // index and every later one from the counter, so the items spread over
  // the CTAs by finishing order rather than by a fixed stride.
  uint32_t* work;
};

__device__ __forceinline__ float* plane(const PoolDev& p, int k) { return p.planes + (size_t)k * p.cap; }

// Slot of logical item i (0 <= i < n_items[0] + n_items[1]): the FP32-SVD
// items first, then the FP64-SVD items.
__device__ __forceinline__ uint32_t item_slot(const PoolDev& p, uint32_t n32, uint32_t i) {
  return i < n32 ? i : p.item_top - 1u - (i - n32);
}

// Grid pool index of node (ix, iy, iz) of a scene (scene-local lattice
// coordinates), or -1 when the node lies outside the grid or, in a sparse
// scene, in a tile without a slot.  Dense: row-major x-fastest n^3 block;
// sparse: 64 nodes per tile slot, x-fastest inside the 4^3 tile.
__device__ __forceinline__ int64_t node_index(const SceneDev& sc, const uint32_t* __restrict__ tile_slot, int ix,
                                              int iy, int iz) {
  const int n = (int)sc.n;
  if ((unsigned)ix >= (unsigned)n || (unsigned)iy >= (unsigned)n || (unsigned)iz >= (unsigned)n) return -1;
  if (!sc.tile_cap)
    return (int64_t)(sc.grid_off + (uint64_t)ix + (uint64_t)n * ((uint64_t)iy + (uint64_t)n * (uint64_t)iz));
  const uint32_t t = (uint32_t)(ix >> 2) + sc.w * ((uint32_t)(iy >> 2) + sc.w * (uint32_t)(iz >> 2));
  const uint32_t slot = tile_slot[sc.key_off + t];
  if (slot == kNoSlot) return -1;
  return (int64_t)(sc.grid_off + 64ull * slot + (uint64_t)((ix & 3) + 4 * (iy & 3) + 16 * (iz & 3)));
}

// Marks the tiles of the 3^3 stencil of a particle with base node (bx, by,
// bz) in a sparse scene (1 or 2 tiles per axis).
__device__ __forceinline__ void mark_stencil_tiles(const SceneDev& sc, uint8_t* __restrict__ tile_mark, int bx, int by,
                                                   int bz) {
  const int n = (int)sc.n;
  int lo[3], hi[3];
  const int b[3] = {bx, by, bz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int l = max(b[a], 0), h = min(b[a] + 2, n - 1);
    if (l > h) return;  // the stencil misses the grid on this axis
    lo[a] = l >> 2;
    hi[a] = h >> 2;
  }
  for (int tz = lo[2]; tz <= hi[2]; ++tz)
    for (int ty = lo[1]; ty <= hi[1]; ++ty)
      for (int tx = lo[0]; tx <= hi[0]; ++tx) {
        uint8_t* m = tile_mark + sc.key_off + (uint32_t)tx + sc.w * ((uint32_t)ty + sc.w * (uint32_t)tz);
        if (*m == 0) *m = 1;
      }
}

// Whether a scene's particles stand still this substep: a latched fault, or
// a substep budget (status word 2) that the completed-substep count (word 1)
// has passed.
__device__ __forceinline__ bool scene_frozen(const uint32_t* status) {
  const volatile uint32_t* s = status;
  const uint32_t fault = s[0], done = s[1], budget = s[2];
  return fault != 0u || (budget != 0u && done > budget);
}
// Whether this substep is the last one of the scene's budget (its gather then
// publishes v and C, as the last substep of a call does).
__device__ __forceinline__ bool budget_ends(const uint32_t* status) {
  const volatile uint32_t* s = status;
  const uint32_t done = s[1], budget = s[2];
  return budget != 0u && done == budget;
}

// Marks the 256-cell block of grid-pool cell g as holding deposits (the grid
// update then converts and later clears only marked blocks).
__device__ __forceinline__ void touch(uint8_t* touched, uint64_t g) { touched[g >> 8] = 1; }

__device__ __forceinline__ bool finitef(float x) {
  return (__float_as_uint(x) & 0x7f800000u) != 0x7f800000u;  // mpm.wgsl:217-219
}
// Finiteness of many values at once: 0 * v is NaN exactly when v is infinite
// or NaN, so an accumulator started at 0 stays 0 (or -0) while every value
// folded in is finite -- one fused multiply-add per value in a chain beside
// the arithmetic it checks, and one compare at the end (nf_ok), instead of a
// classify-and-branch per value.  Relies on IEEE arithmetic (no fast-math).
__device__ __forceinline__ float nf_acc(float acc, float v) { return fmaf(0.0f, v, acc); }
__device__ __forceinline__ double nf_acc(double acc, double v) { return fma(0.0, v, acc); }
__device__ __forceinline__ bool nf_ok(float acc) { return acc == 0.0f; }
__device__ __forceinline__ bool nf_ok(double acc) { return acc == 0.0; }
// The same test over N values folded into four independent accumulators, so
// that the chain the final compare waits on is N/4 fused multiply-adds long
// rather than N (the sum of the four is NaN exactly when one of them is).
template <int N>
__device__ __forceinline__ bool all_finite(const float (&v)[N]) {
  float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int i = 0; i < N; ++i) a[i & 3] = nf_acc(a[i & 3], v[i]);
  return nf_ok((a[0] + a[1]) + (a[2] + a[3]));
}

// ---------------------------------------------------------------------------
// 3x3 helpers on register arrays, column-major a[3*col+row].
template <class T>
__device__ __forceinline__ void matmul(const T* a, const T* b, T* o) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) o[3 * c + r] = a[r] * b[3 * c] + a[3 + r] * b[3 * c + 1] + a[6 + r] * b[3 * c + 2];
}
// u * diag(d) * v^T
template <class T>
__device__ __forceinline__ void sandwich(const T* u, const T* d, const T* v, T* o) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      o[3 * c + r] = (u[r] * d[0]) * v[c] + (u[3 + r] * d[1]) * v[3 + c] + (u[6 + r] * d[2]) * v[6 + c];
}
template <class T>
__device__ __forceinline__ T det3(const T* a) {
  // first-column expansion; a[3*col+row]
  return a[0] * (a[4] * a[8] - a[7] * a[5]) - a[3] * (a[1] * a[8] - a[7] * a[2]) + a[6] * (a[1] * a[5] - a[4] * a[2]);
}

// ---------------------------------------------------------------------------
// Symmetric Jacobi SVD of a 3x3 F (F = U diag(s) V^T), the algorithm of
// mpm.wgsl:365-468: cyclic Jacobi on A = F^T F over (0,1), (0,2), (1,2), at
// most `sweeps` sweeps, stop when the largest off-diagonal is below `tol`;
// sigma_i = |F v_i|, u_i = F v_i / sigma_i; sign fixes so det U = det V = +1.
//
// Both forms run the iteration on the shifted matrix A' = F^T F - I (the same
// eigenvectors and the same off-diagonal entries, so the same rotations and
// stopping test in exact arithmetic), held in FP32 and formed there as
// E + E^T + E^T E from the exact E = F - I, so that its entries keep full
// relative precision however small the strain.  (F^T F itself carries
// rounding noise of half an ulp of 1 on its diagonal, which a tolerance of
// 1e-7 on the off-diagonal then chases through extra sweeps.)  Each rotation
// angle t = sgn(d) e / (|d| + sqrt(d^2+e^2)) (d = a'_qq - a'_pp,
// e = 2 a'_pq; algebraically 1/(theta + sgn(theta) sqrt(1 + theta^2)), the
// reference's formula) is computed in FP32 with the hardware reciprocal
// square root and division.
//
// The FP32 form accumulates V in FP32; sigma_i = |F v_i| and u_i = F v_i /
// sigma_i in FP32.
//
// The FP64 form (svd3<double>) is mixed precision: V accumulates the same
// rotations in FP64 with c = (1 + t^2)^(-1/2) Newton-refined to FP64 and
// s = t c, so V stays orthogonal to FP64 rounding.  sigma_i = |F v_i| and
// u_i = F v_i / sigma_i are FP64.  Double division and square roots are replaced by
// Newton-Raphson refinement of single-precision seeds (two steps each,
// quadratic convergence from 2^-22 to below 2^-52).
// U is held in FP32 in both forms: its consumers (the stress record and
// the rebuilt F) are FP32, while sigma and V carry the form's precision.
template <class T> struct SvdOut {
  float u[9], v[9];
  T s[3];
};

// Newton-Raphson reciprocal square root of x > 0: y <- y (3 - x y^2) / 2
// from the FP32 rsqrtf seed.  Outside the FP32 range of the seed, x is first
// rescaled by an exact power of two (2^200 or 2^-200) and the result by its
// square root; this covers 1e-97 < x < 1e97 and costs a multiply, where a
// fallback to IEEE double division and square root made the gather 3%
// slower even untaken.  Infinite or NaN x gives NaN.
__device__ __forceinline__ double nr_rsqrt(double x) {
  double post = 1.0;
  if (!((float)x > 1.0e-37f && (float)x < 1.0e37f)) {
    const bool small = x < 1.0;
    x *= small ? 0x1p200 : 0x1p-200;
    post = small ? 0x1p100 : 0x1p-100;
  }
  double y = (double)rsqrtf((float)x);
  const double h = 0.5 * x;
  double e = fma(-h * y, y, 0.5);
  y = fma(y, e, y);
  e = fma(-h * y, y, 0.5);
  return post * fma(y, e, y);
}

// One FP32 Jacobi rotation of the (P, Q) pair of the symmetric a[3][3]
// (reference formulas); V is updated with the same c, s in type T.
template <int P, int Q>
__device__ __forceinline__ void jacobi_rot(float (&a)[3][3], float* v, float tol, float& max_off) {
  constexpr int K = 3 - P - Q;
  const float apq = a[P][Q];
  const float aapq = fabsf(apq);
  if (aapq > max_off) max_off = aapq;
  if (aapq < tol || apq == 0.0f) return;
  const float app = a[P][P];
  const float aqq = a[Q][Q];
  float t, c, s;
  {
    // t = 1 / (theta + sgn(theta) sqrt(1 + theta^2)), theta = d / e, written
    // as sgn(d) e / (|d| + sqrt(d^2 + e^2)) with d = a_qq - a_pp, e = 2 a_pq
    // (no division by a small a_pq); c = (1 + t^2)^(-1/2), s = t c.
    float d = aqq - app;
    float e = 2.0f * apq;
    // power-of-two rescale keeps d^2 + e^2 inside the normal FP32 range
    const float m = fmaxf(fabsf(d), fabsf(e));
    const float k = m > 1.0e18f ? 0x1p-64f : (m < 1.0e-18f ? 0x1p64f : 1.0f);
    d *= k;
    e *= k;
    const float r2 = d * d + e * e;
    const float hyp = r2 * rsqrtf(r2);
    t = __fdividef(d >= 0.0f ? e : -e, fabsf(d) + hyp);
    // c = (1 + t^2)^(-1/2): the hardware seed and one Newton step, so that
    // c^2 + s^2 = 1 to FP32 rounding and the accumulated V stays orthogonal
    // (a V that drifts from orthogonality rotates F through the rebuild)
    const float h = fmaf(t, t, 1.0f);
    c = rsqrtf(h);
    c = c * fmaf(-0.5f * h * c, c, 1.5f);
    s = t * c;
  }
  a[P][P] = app - t * apq;
  a[Q][Q] = aqq + t * apq;
  a[P][Q] = 0.0f;
  a[Q][P] = 0.0f;
  {
    const float akp = a[P][K];
    const float akq = a[Q][K];
    const float nkp = c * akp - s * akq;
    const float nkq = s * akp + c * akq;
    a[P][K] = nkp;
    a[Q][K] = nkq;
    a[K][P] = nkp;
    a[K][Q] = nkq;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float vkp = v[3 * P + k];
    const float vkq = v[3 * Q + k];
    v[3 * P + k] = c * vkp - s * vkq;
    v[3 * Q + k] = s * vkp + c * vkq;
  }
}

template <class T>
__device__ __forceinline__ void svd3(const T* f, const float* f32, SvdOut<T>& o, T tol, int max_sweeps) {
  // a[col][row] of A = F^T F (FP32 form) or of A' = F^T F - I (FP64 form);
  // symmetric.  f32 is the same F in FP32.  The FP64 form builds A' in FP32
  // from E = F - I, which is exact (diagonal entries in [0.5, 2], Sterbenz;
  // off-diagonal entries unchanged): A' = E + E^T + E^T E has no cancellation,
  // so its entries keep full FP32 relative precision however small the
  // strain, as forming F^T F - I in FP64 and rounding does.
  float a[3][3];
  {
    float e[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) e[i] = (i % 4 == 0) ? f32[i] - 1.0f : f32[i];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = c; r < 3; ++r) {
        // (E^T E)_cr + E_rc + E_cr, column-major e[3 col + row]
        const float ete = e[3 * r] * e[3 * c] + e[3 * r + 1] * e[3 * c + 1] + e[3 * r + 2] * e[3 * c + 2];
        a[c][r] = (e[3 * c + r] + e[3 * r + c]) + ete;
        a[r][c] = a[c][r];
      }
  }
  float* v = o.v;
#pragma unroll
  for (int i = 0; i < 9; ++i) v[i] = (i % 4 == 0) ? 1.0f : 0.0f;
  const float ftol = (float)tol;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    float max_off = 0.0f;
    jacobi_rot<0, 1>(a, v, ftol, max_off);
    jacobi_rot<0, 2>(a, v, ftol, max_off);
    jacobi_rot<1, 2>(a, v, ftol, max_off);
    if (max_off < ftol) break;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if constexpr (sizeof(T) == 4) {
      const float x = f[0] * v[3 * i] + f[3] * v[3 * i + 1] + f[6] * v[3 * i + 2];
      const float y = f[1] * v[3 * i] + f[4] * v[3 * i + 1] + f[7] * v[3 * i + 2];
      const float z = f[2] * v[3 * i] + f[5] * v[3 * i + 1] + f[8] * v[3 * i + 2];
      const float q = x * x + y * y + z * z;
      const float s = sqrtf(q);  // correctly rounded: the stress depends on s - 1
      o.s[i] = s;
      if (s > 1.0e-12f) {
        const float inv = __frcp_rn(s);
        o.u[3 * i] = x * inv;
        o.u[3 * i + 1] = y * inv;
        o.u[3 * i + 2] = z * inv;
      } else {
        o.u[3 * i] = i == 0 ? 1.0f : 0.0f;
        o.u[3 * i + 1] = i == 1 ? 1.0f : 0.0f;
        o.u[3 * i + 2] = i == 2 ? 1.0f : 0.0f;
      }
    } else {
      // sigma_i = |F v_i| / |v_i| in FP64: a Rayleigh quotient, second order
      // in the direction error of the FP32 v_i, with the norm of v_i (1 up
      // to a few FP32 ulps) divided out: 1/|v| = 1.5 - n2/2 to O((n2-1)^2).
      const double v0 = v[3 * i], v1 = v[3 * i + 1], v2 = v[3 * i + 2];
      const double x = f[0] * v0 + f[3] * v1 + f[6] * v2;
      const double y = f[1] * v0 + f[4] * v1 + f[7] * v2;
      const double z = f[2] * v0 + f[5] * v1 + f[8] * v2;
      const double q = x * x + y * y + z * z;
      const double rq = q > 0.0 ? nr_rsqrt(q) : 0.0;  // 1 / |F v_i|
      const double rn = fma(-0.5, v0 * v0 + v1 * v1 + v2 * v2, 1.5);
      const double s = q * rq * rn;
      o.s[i] = s;
      if (s > 1.0e-12) {
        // u_i = F v_i / |F v_i|
        o.u[3 * i] = (float)(x * rq);
        o.u[3 * i + 1] = (float)(y * rq);
        o.u[3 * i + 2] = (float)(z * rq);
      } else {
        o.u[3 * i] = i == 0 ? 1.0f : 0.0f;
        o.u[3 * i + 1] = i == 1 ? 1.0f : 0.0f;
        o.u[3 * i + 2] = i == 2 ? 1.0f : 0.0f;
      }
    }
  }
  if (det3(o.u) < 0.0f) {
    // flip the column of U with the smallest (signed) sigma
    const bool m1 = o.s[1] < o.s[0];
    const T s01 = m1 ? o.s[1] : o.s[0];
    const bool m2 = o.s[2] < s01;
    const int mi = m2 ? 2 : (m1 ? 1 : 0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T sg = (i == mi) ? T(-1) : T(1);
      o.u[3 * i] *= sg;
      o.u[3 * i + 1] *= sg;
      o.u[3 * i + 2] *= sg;
      o.s[i] *= sg;
    }
  }
  // V is a product of plane rotations, so det V = +1 up to rounding: the
  // reference's flip (mpm.wgsl:457-466) never fires.  It is kept in the FP32
  // reference form and skipped in the FP64 form.
  if constexpr (sizeof(T) == 4) {
    if (det3(v) < 0.0f) {
      // flip the column of V with the smallest |sigma|
      const T a0 = o.s[0] < T(0) ? -o.s[0] : o.s[0];
      const T a1 = o.s[1] < T(0) ? -o.s[1] : o.s[1];
      const T a2 = o.s[2] < T(0) ? -o.s[2] : o.s[2];
      const bool m1 = a1 < a0;
      const T a01 = m1 ? a1 : a0;
      const bool m2 = a2 < a01;
      const int mi = m2 ? 2 : (m1 ? 1 : 0);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const float sg = (i == mi) ? -1.0f : 1.0f;
        v[3 * i] *= sg;
        v[3 * i + 1] *= sg;
        v[3 * i + 2] *= sg;
        o.s[i] *= (T)sg;
      }
    }
  }
}

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// Two independent FP32 fused multiply-adds in one instruction (sm_100
// fma.rn.f32x2): (a.x b.x + c.x, a.y b.y + c.y), each rounded once, the same
// values as two fmaf calls.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  uint64_t ua, ub, uc, r;
  memcpy(&ua, &a, 8);
  memcpy(&ub, &b, 8);
  memcpy(&uc, &c, 8);
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(ua), "l"(ub), "l"(uc));
  float2 o;
  memcpy(&o, &r, 8);
  return o;
}

// Two independent FP32 sums in one instruction (sm_100 add.rn.f32x2), each
// rounded once as __fadd_rn.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  uint64_t ua, ub, r;
  memcpy(&ua, &a, 8);
  memcpy(&ub, &b, 8);
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(ua), "l"(ub));
  float2 o;
  memcpy(&o, &r, 8);
  return o;
}

// Quadratic B-spline weights (mpm.wgsl:285-294).
__device__ __forceinline__ void quad_weights(float fx, float* w) {
  w[0] = 0.5f * (1.5f - fx) * (1.5f - fx);
  w[1] = 0.75f - (fx - 1.0f) * (fx - 1.0f);
  w[2] = 0.5f * (fx - 0.5f) * (fx - 0.5f);
}

// Fixed-corotated stress from a (U, s, V) decomposition of F, mpm.wgsl:532-599:
// s_c = clamp(s, 0.1, 10), R = U V^T, J = prod s_c, hardening h by rheology,
// P = 2 mu h (Fc - R) + lam h (J - 1) cof, S = -dt vol P Fc^T.  Returns
// B = m C + 4/dx^2 S so that a node at offset d receives w (m v + B d).
__device__ __forceinline__ void p2g_affine_principal(const SvdOut<double>& svd, const MatDev& md, float jp,
                                                     float mass, float vol, const float* C, float dt, float inv_dx,
                                                     float* B) {
  // FP64-SVD form.  With Fc = U Sc V^T, R = U V^T and cof = U diag(J/sc) V^T
  // the same stress is S = -dt vol P Fc^T = -dt vol U diag(tau) U^T,
  // tau_i = 2 mu h (sc_i - 1) sc_i + lam h (J - 1) J (Kirchhoff stress in
  // the principal frame).  sc_i - 1 and J - 1 are formed in FP64, so the
  // small-strain stress keeps full FP32 relative precision instead of
  // cancelling in Fc - R.
  double scd[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) scd[i] = fmin(fmax(svd.s[i], 0.1), 10.0);
  const double Jd = scd[0] * scd[1] * scd[2];
  const float J = (float)Jd;
  const float jm1 = (float)(Jd - 1.0);
  float h = 1.0f;
  if (md.rheo == 1) {
    h = expf(clampf(-md.hardening * jp, -3.0f, 3.0f));
  } else if (md.rheo == 0) {
    h = expf(clampf(jp, -3.0f, 3.0f));
  }
  const float k1 = 2.0f * md.mu * h;
  const float kv = md.lam * h * jm1 * J;
  float tau[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) tau[i] = k1 * (float)(scd[i] - 1.0) * (float)scd[i] + kv;
  float u[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) u[i] = svd.u[i];
  const float k = -dt * vol * 4.0f * inv_dx * inv_dx;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = c; r < 3; ++r) {
      const float S = k * (u[r] * tau[0] * u[c] + u[3 + r] * tau[1] * u[3 + c] + u[6 + r] * tau[2] * u[6 + c]);
      B[3 * c + r] = mass * C[3 * c + r] + S;
      if (r != c) B[3 * r + c] = mass * C[3 * r + c] + S;
    }
}

// Reference form (FP32 SVD); the FP64-SVD mode takes the principal form.
template <class T>
__device__ __forceinline__ void p2g_affine(const SvdOut<T>& svd, const MatDev& md, float jp, float mass, float vol,
                                           const float* C, float dt, float inv_dx, float* B) {
  if constexpr (sizeof(T) == 8) {
    p2g_affine_principal(svd, md, jp, mass, vol, C, dt, inv_dx, B);
  } else {
    float u[9], v[9], sc[3];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      u[i] = svd.u[i];
      v[i] = (float)svd.v[i];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) sc[i] = clampf((float)svd.s[i], 0.1f, 10.0f);
    float h = 1.0f;
    if (md.rheo == 1) {
      h = expf(clampf(-md.hardening * jp, -3.0f, 3.0f));
    } else if (md.rheo == 0) {
      h = expf(clampf(jp, -3.0f, 3.0f));
    }
    const float mu_h = md.mu * h;
    const float lam_h = md.lam * h;
    const float J = sc[0] * sc[1] * sc[2];
    const float cofd[3] = {sc[1] * sc[2], sc[0] * sc[2], sc[0] * sc[1]};
    float Fc[9], cof[9];
    sandwich(u, sc, v, Fc);
    sandwich(u, cofd, v, cof);
    const float k1 = 2.0f * mu_h;
    const float k2 = lam_h * (J - 1.0f);
    const float k3 = -dt * vol;
    float P[9];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        // R = U V^T
        const float Rcr = u[r] * v[c] + u[3 + r] * v[3 + c] + u[6 + r] * v[6 + c];
        P[3 * c + r] = k3 * (k1 * (Fc[3 * c + r] - Rcr) + k2 * cof[3 * c + r]);
      }
    // S = P Fc^T : S[c][r] = sum_k P[k][r] * Fc[k][c]
    const float four_inv_dx2 = 4.0f * inv_dx * inv_dx;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const float S = P[r] * Fc[c] + P[3 + r] * Fc[3 + c] + P[6 + r] * Fc[6 + c];
        B[3 * c + r] = mass * C[3 * c + r] + four_inv_dx2 * S;
      }
  }
}

// Plasticity return mapping on (U, s, V), mpm.wgsl:1366-1479.  Writes the
// projected, safety-clamped singular values into s (in place), updates jp.
// Returns false on a numerical fault.
template <class T>
__device__ __forceinline__ bool plasticity_project(SvdOut<T>& svd, const MatDev& md, float& jp, bool& changed) {
  float s[3] = {(float)svd.s[0], (float)svd.s[1], (float)svd.s[2]};
  {
    float chk[21];
#pragma unroll
    for (int a = 0; a < 3; ++a) chk[a] = s[a];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      chk[3 + 2 * i] = svd.u[i];
      chk[4 + 2 * i] = svd.v[i];
    }
    if (!all_finite(chk)) return false;
  }
  T ns[3] = {svd.s[0], svd.s[1], svd.s[2]};
  float dq = 0.0f;
  bool jp_replace = false;
  float jp_new = 0.0f;
  if (md.rheo == 1) {
    float nsf[3];
    const T lo = (T)(1.0f - md.theta_c), hi = (T)(1.0f + md.theta_s);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      T x = svd.s[a];
      x = x < lo ? lo : x;
      x = x > hi ? hi : x;
      ns[a] = x;
      nsf[a] = (float)x;
    }
    const float det_old = fmaxf(s[0] * s[1] * s[2], 1.0e-6f);
    const float det_new = fmaxf(nsf[0] * nsf[1] * nsf[2], 1.0e-6f);
    const float dlog = logf(det_old) - logf(det_new);
    jp_replace = true;
    jp_new = jp + dlog;
    if (!finitef(jp_new)) return false;
    jp_new = clampf(jp_new, -5.0f, 5.0f);
  } else if (md.rheo == 2) {
    jp_replace = true;
    jp_new = 0.0f;
  } else {
    float eps[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) eps[a] = logf(fmaxf(s[a], 1.0e-6f));
    const float tr = eps[0] + eps[1] + eps[2];
    const float mean = tr / 3.0f;
    const float dev[3] = {eps[0] - mean, eps[1] - mean, eps[2] - mean};
    const float dev_norm = sqrtf(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
    if (tr > 0.0f) {
      ns[0] = ns[1] = ns[2] = T(1);
      dq = sqrtf(eps[0] * eps[0] + eps[1] * eps[1] + eps[2] * eps[2]);
    } else if (dev_norm == 0.0f) {
      // elastic, keep s
    } else {
      const float fy = dev_norm + md.kappa * tr * md.dp_alpha;
      if (fy > 0.0f) {
        const float rc = fmaxf(0.0f, -md.dp_alpha * md.kappa * tr);
#pragma unroll
        for (int a = 0; a < 3; ++a) ns[a] = (T)expf(dev[a] * (rc / dev_norm) + mean);
        dq = fy;
      }
    }
  }
  {
    // ns comes from FP32 values (clamps of s, expf), so finite in T is finite in FP32
    const T nfs = nf_acc(nf_acc(nf_acc(T(0), ns[0]), ns[1]), ns[2]);
    const float nfq = nf_acc(nf_acc(0.0f, dq), jp + dq);
    if (!nf_ok(nfs) || !nf_ok(nfq)) return false;
  }
  changed = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T x = ns[a];
    x = x < T(0.05) ? T(0.05) : x;
    x = x > T(20) ? T(20) : x;
    changed = changed || x != svd.s[a];
    svd.s[a] = x;
  }
  jp = jp_replace ? jp_new : clampf(jp + dq, 0.0f, 5.0f);
  return true;
}

}  // namespace mpm
