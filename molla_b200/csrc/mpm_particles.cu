// mpm_particles.cu — the particle kernels of the B200 MLS-MPM substep.
//
// One substep of the reference (crates/molla-solvers/src/mpm.rs:2476-2551:
// reset_grid, p2g, grid_update, g2p, plasticity) runs as three launches
// (two for small groups, where the gather and scatter are fused):
//
//   grid_update(n)  acc[a] -> velocity, clears acc[b]               (grid sweep)
//   gather(n)       G2P(n) + F update + return mapping(n); writes the particle
//                   and, for the next substep, the APIC/stress matrix
//                   B = m C + 4/dx^2 S (S the fixed-corotated stress term)
//   scatter(n+1)    27-node deposit of mass and momentum into acc[b]
//
// Both particle kernels are persistent over a work list of (scene, tile, slot
// range) items built by the last regrouping (a stable radix sort of the
// particles by base-cell key; tiles of 4^3 base cells, cut into items of at
// most kStageMax particles).  The gather stages the 8^3-node velocity block
// around the tile in shared memory; the scatter stages the item's 64-byte
// records with one bulk copy, bins them by their current base cell and
// accumulates into an 8^3-node shared block that it flushes to HBM with one
// float4 atomic per non-empty node.  For large groups they are separate
// kernels because the gather (SVD, return mapping) needs ~128 registers per
// thread while the scatter needs fewer: split, each runs at its own
// occupancy, and the B record's round trip through HBM is cheaper than the
// fused kernel's lower occupancy.  For small groups (a few hundred items,
// about one wave) the fused k_g2p2g keeps the records in shared memory and
// saves a launch per substep.  The SVD computed
// by the return mapping is reused for the next substep's stress; the first
// substep of every step_n call runs a record-only gather that computes it
// from F.
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_device.cuh"
#include "mpm_kernels.cuh"

namespace mpm {

namespace {

struct SharedGather {
  float4 vel[kRegionNodes];
  float fallback[kGatherThreads][13];  // per-thread result slot of gather_global
};

__device__ __forceinline__ int region_index(int lx, int ly, int lz) { return lx + kRsy * ly + kRsz * lz; }

// Regroup key of a particle from its base cell: ((scene tile offset + tile)
// << 6) | cell within the tile; base clamped to the grid.
__device__ __forceinline__ uint32_t base_key(const SceneDev& sc, const int* base) {
  uint32_t t[3], c[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int b = base[a];
    b = b < 0 ? 0 : b;
    b = b > (int)sc.n - 1 ? (int)sc.n - 1 : b;
    t[a] = (uint32_t)b >> 2;
    c[a] = (uint32_t)b & 3u;
  }
  const uint32_t tile = t[0] + sc.w * (t[1] + sc.w * t[2]);
  return ((sc.key_off + tile) << kCellBits) | c[0] | (c[1] << 2) | (c[2] << 4);
}

// Gather for a particle whose stencil is not inside the staged 8^3 block
// (it left its tile since the last regrouping): 27 global reads with the
// reference's out-of-grid skip.  Kept out of line and rolled so that the
// unrolled shared-memory path stays small; it takes scalars and writes
// v (3) and G = sum w gv d^T (9) to the caller's shared-memory slot, so the
// call needs no local memory.
__device__ __noinline__ void gather_global(const float4* __restrict__ vel_pool, const SceneDev& sc,
                                           const uint32_t* __restrict__ tile_slot, float xp0, float xp1, float xp2,
                                           float* out) {
  const float xp[3] = {xp0, xp1, xp2};
  const int win[3] = {sc.winx, sc.winy, sc.winz};
  const float dx = sc.dx;
  float w[3][3], d[3][3];
  int base[3];
  for (int a = 0; a < 3; ++a) {
    const float bf = floorf(xp[a] - 0.5f);
    base[a] = (int)bf - win[a];
    const float fx = xp[a] - bf;
    quad_weights(fx, w[a]);
    for (int i = 0; i < 3; ++i) d[a][i] = ((float)i - fx) * dx;
  }
  float acc[12];
  for (int i = 0; i < 12; ++i) acc[i] = 0.f;
  for (int q = 0; q < 27; ++q) {
    const int i = q / 9, j = (q / 3) % 3, k = q % 3;
    const int64_t c = node_index(sc, tile_slot, base[0] + i, base[1] + j, base[2] + k);
    if (c < 0) continue;
    const float4 g = __ldg(&vel_pool[c]);
    const float wt = w[0][i] * w[1][j] * w[2][k];
    const float gv[3] = {wt * g.x, wt * g.y, wt * g.z};
    for (int r = 0; r < 3; ++r) {
      acc[r] += gv[r];
      acc[3 + r] += gv[r] * d[0][i];
      acc[6 + r] += gv[r] * d[1][j];
      acc[9 + r] += gv[r] * d[2][k];
    }
  }
  for (int i = 0; i < 12; ++i) out[i] = acc[i];
}

// mbarrier + bulk-copy (TMA engine) helpers for the scatter's record stage.
__device__ __forceinline__ uint32_t smem_addr(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Orders this CTA's earlier generic-proxy accesses of shared memory before
// later async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 2-D TMA tile load (box of kStageBoxRows records) at coordinates (0, row)
// of the record tensor map, completing on `bar`.
__device__ __forceinline__ void tma_load_rows(void* dst, const CUtensorMap* map, int row, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Ampere-style asynchronous 4-byte global -> shared copies (cp.async), in
// commit groups; a thread waits for its own groups.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Waits for the phase of `bar` with the given parity to complete; gives up
// (returns false) after about one second.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > 1000000000ull) return false;
  }
  return true;
}

}  // namespace

// The particle inputs the gather stages in shared memory, in order: the
// position planes, the F planes, mass, volume and J_p (planes PX..PZ and
// F0..JP in plane order), then the meta word.
constexpr int kStagedInputs = 16;
static_assert(PY == PX + 1 && PZ == PX + 2 && MASS == F0 + 9 && VOL == F0 + 10 && JP == F0 + 11,
              "the staged planes are two runs of consecutive planes");

// The CTA-uniform values of the item a gather CTA is on, kept in shared
// memory so that they hold no registers through the particle computation:
// the scene's status word, the 8^3 velocity block origin, whether this
// substep publishes v and C, and the item's slot range.
struct GatherCtx {
  uint32_t* status;
  int rx, ry, rz;
  uint32_t publish_vc;
  uint32_t start, count;
};

// One particle of an item: G2P + F update + return mapping (MODE != kRecord)
// and the scatter record (MODE != kG2P), returned in rec.  ctx holds the
// item's uniform values; vblock is the staged 8^3-node velocity block of the
// item's tile (origin node ctx.rx, ctx.ry, ctx.rz); fallback is a 12-float
// shared-memory slot of this thread for gather_global.  `in` (kStagedInputs
// words kGatherThreads apart, or null) holds the particle's inputs in the
// staged order above, copied to shared memory ahead of time (k_g2p); null
// reads them from the pool.
template <int MODE, bool WRITE_KEYS, class SR>
__device__ __forceinline__ void particle_step(const PoolDev& p, const SceneDev& sc, uint32_t s, const GatherCtx& ctx,
                                              const float4* __restrict__ vblock, float* fallback, SR stol, int sweeps,
                                              int reuse_svd, float4 (&rec)[4], const float* __restrict__ in = nullptr) {
  constexpr bool kGather = MODE != kRecord;
  constexpr bool kScatter = MODE != kG2P;
  float x, y, z, F[9], jp, mass, vol;
  uint32_t mat;
  if (in) {
    x = in[0];
    y = in[kGatherThreads];
    z = in[2 * kGatherThreads];
#pragma unroll
    for (int i = 0; i < 9; ++i) F[i] = in[(3 + i) * kGatherThreads];
    mass = in[12 * kGatherThreads];
    vol = in[13 * kGatherThreads];
    jp = in[14 * kGatherThreads];
    mat = __float_as_uint(in[15 * kGatherThreads]) & 7u;
  } else {
    x = plane(p, PX)[s];
    y = plane(p, PY)[s];
    z = plane(p, PZ)[s];
#pragma unroll
    for (int i = 0; i < 9; ++i) F[i] = plane(p, F0 + i)[s];
    jp = plane(p, JP)[s];
    mass = plane(p, MASS)[s];
    vol = plane(p, VOL)[s];
    mat = p.meta[s] & 7u;
  }
  float v[3], C[9];
  bool ok = true;
  SvdOut<SR> svd;
  if constexpr (kGather) {
    // ---- g2p (mpm.wgsl:1242-1353) ----
    const float xp[3] = {(x - sc.ox) * sc.inv_dx, (y - sc.oy) * sc.inv_dx, (z - sc.oz) * sc.inv_dx};
    const float chk[16] = {x, y, z, jp, F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8], xp[0], xp[1], xp[2]};
    if (!all_finite(chk)) {
      atomicOr(ctx.status, kFaultNumerical);
      ok = false;
    }
    if (ok) {
      float w[3][3], d[3][3];
      int base[3];
      const int win[3] = {sc.winx, sc.winy, sc.winz};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float bf = floorf(xp[a] - 0.5f);
        base[a] = (int)bf - win[a];
        const float fx = xp[a] - bf;
        quad_weights(fx, w[a]);
#pragma unroll
        for (int i = 0; i < 3; ++i) d[a][i] = ((float)i - fx) * sc.dx;
      }
      const int lx0 = base[0] - ctx.rx, ly0 = base[1] - ctx.ry, lz0 = base[2] - ctx.rz;
      const bool inside = (unsigned)lx0 <= (unsigned)(kRegion - 3) && (unsigned)ly0 <= (unsigned)(kRegion - 3) &&
                          (unsigned)lz0 <= (unsigned)(kRegion - 3);
      // Separable accumulation: v = sum w gv; G = sum (w gv) d^T.
      float vs[3] = {0.f, 0.f, 0.f};
      float G[9];
      if (inside) {
#pragma unroll
        for (int i = 0; i < 9; ++i) G[i] = 0.f;
        const float4* __restrict__ blk = &vblock[lx0 + 8 * ly0 + 64 * lz0];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          float si[3] = {0.f, 0.f, 0.f}, syi[3] = {0.f, 0.f, 0.f}, szi[3] = {0.f, 0.f, 0.f};
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            float sj[3] = {0.f, 0.f, 0.f}, szj[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
              const float4 g = blk[i + 8 * j + 64 * kk];
              const float wk = w[2][kk];
              sj[0] += wk * g.x;
              sj[1] += wk * g.y;
              sj[2] += wk * g.z;
              const float wdk = wk * d[2][kk];
              szj[0] += wdk * g.x;
              szj[1] += wdk * g.y;
              szj[2] += wdk * g.z;
            }
            const float wj = w[1][j];
            const float wdj = wj * d[1][j];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
              si[r] += wj * sj[r];
              syi[r] += wdj * sj[r];
              szi[r] += wj * szj[r];
            }
          }
          const float wi = w[0][i];
          const float wdi = wi * d[0][i];
#pragma unroll
          for (int r = 0; r < 3; ++r) {
            vs[r] += wi * si[r];
            G[r] += wdi * si[r];      // column x
            G[3 + r] += wi * syi[r];  // column y
            G[6 + r] += wi * szi[r];  // column z
          }
        }
      } else {
        float* slot = fallback;
        gather_global(p.vel, sc, p.tile_slot, xp[0], xp[1], xp[2], slot);
#pragma unroll
        for (int r = 0; r < 3; ++r) vs[r] = slot[r];
#pragma unroll
        for (int r = 0; r < 9; ++r) G[r] = slot[3 + r];
      }
      const float four_inv_dx2 = 4.0f * sc.inv_dx * sc.inv_dx;
#pragma unroll
      for (int i = 0; i < 9; ++i) C[i] = four_inv_dx2 * G[i];
      v[0] = vs[0];
      v[1] = vs[1];
      v[2] = vs[2];
      const MatDev& md = sc.mat[mat];
      if (md.rheo == 2) {
        v[0] *= md.vfac;
        v[1] *= md.vfac;
        v[2] *= md.vfac;
#pragma unroll
        for (int i = 0; i < 9; ++i) C[i] *= md.afac;
      }
      float np[3] = {x + sc.dt * v[0], y + sc.dt * v[1], z + sc.dt * v[2]};
      const float chk2[15] = {np[0], v[0], np[1], v[1], np[2], v[2], C[0], C[1], C[2],
                              C[3],  C[4], C[5],  C[6], C[7],  C[8]};
      if (!all_finite(chk2)) {
        atomicOr(ctx.status, kFaultNumerical);
        ok = false;
      }
      if (ok) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          if (np[a] < sc.lo[a] || np[a] > sc.hi[a]) v[a] = 0.f;
          np[a] = clampf(np[a], sc.lo[a], sc.hi[a]);
        }
        // F <- (I + dt C) F
        float A[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) A[i] = sc.dt * C[i] + ((i % 4 == 0) ? 1.f : 0.f);
        float Fn[9];
        matmul(A, F, Fn);
        if (!all_finite(Fn)) {
          atomicOr(ctx.status, kFaultNumerical);
          ok = false;
        } else {
          x = np[0];
          y = np[1];
          z = np[2];
#pragma unroll
          for (int i = 0; i < 9; ++i) F[i] = Fn[i];
          // ---- plasticity (mpm.wgsl:1366-1479) on the updated F ----
          SR Fs[9];
#pragma unroll
          for (int i = 0; i < 9; ++i) Fs[i] = (SR)F[i];
          svd3<SR>(Fs, F, svd, stol, sweeps);
          float jp_new = jp;
          bool changed = true;
          const SR s_trial[3] = {svd.s[0], svd.s[1], svd.s[2]};
          if (plasticity_project<SR>(svd, md, jp_new, changed)) {
            // FP32 mode rebuilds F = U s V^T every substep (the
            // reference).  The FP64-SVD mode keeps the trial F when the
            // return mapping left every singular value unchanged, and
            // otherwise adds U diag(s - s_trial) V^T to it: the same F as
            // U s V^T in exact arithmetic (F = U s_trial V^T), with the
            // FP32 rounding of U and V scaled by the (small) change in s
            // instead of by F.
            float Fr[9];
            const bool rebuild = sizeof(SR) == 4 || changed;
            if (rebuild) {
              float ds[3];
#pragma unroll
              for (int i = 0; i < 3; ++i) ds[i] = sizeof(SR) == 4 ? (float)svd.s[i] : (float)(svd.s[i] - s_trial[i]);
#pragma unroll
              for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r)
                  Fr[3 * c + r] = (sizeof(SR) == 4 ? 0.0f : F[3 * c + r]) + (svd.u[r] * ds[0]) * svd.v[c] +
                                  (svd.u[3 + r] * ds[1]) * svd.v[3 + c] + (svd.u[6 + r] * ds[2]) * svd.v[6 + c];
            }
            // the FP32 copy must be finite too (an FP64 value beyond FP32 range)
            if (!rebuild || all_finite(Fr)) {
              if (rebuild) {
#pragma unroll
                for (int i = 0; i < 9; ++i) F[i] = (float)Fr[i];
              }
              jp = jp_new;
            } else {
              atomicOr(ctx.status, kFaultNumerical);
              ok = false;
            }
          } else {
            atomicOr(ctx.status, kFaultNumerical);
            ok = false;
          }
          // G2P results are published even when the return mapping
          // faults (the reference's g2p and plasticity are separate
          // dispatches); only the plasticity update is withheld.
          // v and C are read by nothing before the next call (the next
          // gather recomputes them from the grid; the scatter takes the
          // record), so a substep that writes a record skips them unless
          // the return mapping faulted: the last substep of a call
          // publishes them.
          plane(p, PX)[s] = x;
          plane(p, PY)[s] = y;
          plane(p, PZ)[s] = z;
          if (!kScatter || !ok || ctx.publish_vc) {
            plane(p, VX)[s] = v[0];
            plane(p, VY)[s] = v[1];
            plane(p, VZ)[s] = v[2];
#pragma unroll
            for (int i = 0; i < 9; ++i) plane(p, C0 + i)[s] = C[i];
          }
#pragma unroll
          for (int i = 0; i < 9; ++i) plane(p, F0 + i)[s] = F[i];
          plane(p, JP)[s] = jp;
        }
      }
    }
  } else {
    // P2G-only: read v and C and validate the whole state (the
    // reference's g2p checks, mpm.wgsl:1247-1255, moved to the first
    // launch of the call so that a non-finite upload latches before
    // anything moves).
    v[0] = plane(p, VX)[s];
    v[1] = plane(p, VY)[s];
    v[2] = plane(p, VZ)[s];
#pragma unroll
    for (int i = 0; i < 9; ++i) C[i] = plane(p, C0 + i)[s];
    bool fin = finitef(x) && finitef(y) && finitef(z) && finitef(jp) && finitef(v[0]) && finitef(v[1]) &&
               finitef(v[2]) && finitef((x - sc.ox) * sc.inv_dx) && finitef((y - sc.oy) * sc.inv_dx) &&
               finitef((z - sc.oz) * sc.inv_dx);
#pragma unroll
    for (int i = 0; i < 9; ++i) fin = fin && finitef(F[i]) && finitef(C[i]);
    if (!fin) {
      atomicOr(ctx.status, kFaultNumerical);
      ok = false;
    }
  }
  if constexpr (kScatter) {
    // B = m C + 4/dx^2 S for the next scatter (all-zero for a particle
    // that faulted, which then deposits nothing).
    float B[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) B[i] = 0.f;
    if (ok) {
      if (!kGather || !reuse_svd) {
        SR Fs[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) Fs[i] = (SR)F[i];
        svd3<SR>(Fs, F, svd, stol, sweeps);
      }
      p2g_affine<SR>(svd, sc.mat[mat], jp, mass, vol, C, sc.dt, sc.inv_dx, B);
    }
    // Packed record (x, y, z, m), (m v, B0), (B1..B4), (B5..B8); a
    // faulted particle gets m = 0 and deposits nothing.
    const float mr = ok ? mass : 0.f;
    const float vx = ok ? mass * v[0] : 0.f, vy = ok ? mass * v[1] : 0.f, vz = ok ? mass * v[2] : 0.f;
    rec[0] = make_float4(x, y, z, mr);
    rec[1] = make_float4(vx, vy, vz, B[0]);
    rec[2] = make_float4(B[1], B[2], B[3], B[4]);
    rec[3] = make_float4(B[5], B[6], B[7], B[8]);
  }
  if constexpr (kScatter) {
    // sparse storage: the tiles this record's deposit will touch
    if (sc.tile_cap && ok) {
      const float xq[3] = {(x - sc.ox) * sc.inv_dx, (y - sc.oy) * sc.inv_dx, (z - sc.oz) * sc.inv_dx};
      mark_stencil_tiles(sc, p.tile_mark, (int)floorf(xq[0] - 0.5f) - sc.winx, (int)floorf(xq[1] - 0.5f) - sc.winy,
                         (int)floorf(xq[2] - 0.5f) - sc.winz);
    }
  }
  if constexpr (WRITE_KEYS) {
    const float xp[3] = {(x - sc.ox) * sc.inv_dx, (y - sc.oy) * sc.inv_dx, (z - sc.oz) * sc.inv_dx};
    const int win[3] = {sc.winx, sc.winy, sc.winz};
    int nbase[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) nbase[a] = (xp[a] == xp[a]) ? (int)floorf(xp[a] - 0.5f) - win[a] : 0;
    p.keys_by_id[p.orig[s]] = base_key(sc, nbase);
  }
}

// MODE: kRecord (no gather: validate the state and compute B from the SVD of
// F — the first substep of a call), kG2P (gather + return mapping, the last
// substep of a call), kG2PRecord (gather + return mapping + B for the next
// scatter, with the return mapping's SVD reused).
template <int MODE, bool WRITE_KEYS, class SR>
__global__ void __launch_bounds__(kGatherThreads, 5) k_g2p(PoolDev p, double tol, int sweeps, int reuse_svd,
                                                            int publish_all) {
  constexpr bool kGather = MODE != kRecord;
  constexpr bool kScatter = MODE != kG2P;
  __shared__ __align__(16) SceneDev s_sc;
  __shared__ __align__(16) SharedGather s_gath;
  __shared__ uint32_t s_fault;
  __shared__ GatherCtx s_ctx;
  __shared__ uint32_t s_it_next;
  // Particle inputs of this round and the next (cp.async double buffer):
  // [buffer][input][thread], the inputs in the staged order.
  __shared__ __align__(16) float s_in[2][kStagedInputs][kGatherThreads];
  // this SVD form's range of the work list: FP32-SVD items, then FP64-SVD items
  const uint32_t n32 = p.n_items[0];
  const uint32_t it_lo = sizeof(SR) == 8 ? n32 : 0u;
  const uint32_t it_hi = sizeof(SR) == 8 ? n32 + p.n_items[1] : n32;
  const SR stol = (SR)tol;
  uint32_t s_sc_scene = 0xffffffffu;  // scene whose record s_sc holds
  for (uint32_t it = it_lo + blockIdx.x; it < it_hi;) {
    const Item item = p.items[item_slot(p, n32, it)];
    // this CTA's next item, taken now and read by all after the item's work
    if (threadIdx.x == 0) s_it_next = it_lo + gridDim.x + atomicAdd(p.work, 1u);
    // A thread's particles come kGatherThreads apart; the inputs of its
    // next particle are copied to shared memory (cp.async) while it computes
    // this one, and those of its first are requested here, so that their
    // loads overlap the velocity block's.
    const uint32_t tid = threadIdx.x;
    auto fetch = [&](uint32_t k, int b, uint32_t start, uint32_t count) {
      if (k < count) {
        const uint32_t s = start + k;
        // walk the planes with one pointer: PX..PZ, then F0..JP
        const size_t cap = p.cap;
        const float* src = p.planes + s;
#pragma unroll
        for (int q = 0; q < 3; ++q, src += cap) cp_async4(&s_in[b][q][tid], src);
        src += (size_t)(F0 - 3) * cap;
#pragma unroll
        for (int q = 3; q < kStagedInputs - 1; ++q, src += cap) cp_async4(&s_in[b][q][tid], src);
        cp_async4(&s_in[b][kStagedInputs - 1][tid], p.meta + s);
      }
      cp_async_commit();
    };
    fetch(tid, 0, item.start, item.count);
    // The scene record goes to shared memory when the item's scene differs
    // from the last item's (consecutive items of a CTA mostly share one):
    // the velocity staging below reads the geometry from there, so a new
    // record is published by a barrier first.
    if (item.scene != s_sc_scene) {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(p.scenes + item.scene);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_sc);
      for (int k = threadIdx.x; k < (int)(sizeof(SceneDev) / 4); k += kGatherThreads) dst[k] = src[k];
      s_sc_scene = item.scene;
      __syncthreads();
    }
    const SceneDev& sc = s_sc;
    const uint32_t w = sc.w;
    const uint32_t tx = item.tile % w, ty = (item.tile / w) % w, tz = item.tile / (w * w);
    const int rx = 4 * (int)tx - 1, ry = 4 * (int)ty - 1, rz = 4 * (int)tz - 1;
    if (threadIdx.x == 0) {
      uint32_t* status = p.status + (size_t)sc.status * kStatusWords;
      // a latched fault, a spent substep budget or a retired scene: stand still
      s_fault = (scene_frozen(status) || !sc.live) ? 1u : 0u;
      s_ctx = GatherCtx{status, rx, ry, rz, (publish_all || budget_ends(status)) ? 1u : 0u, item.start, item.count};
    }
    if constexpr (kGather) {
      // Stage the 8^3-node velocity block (out-of-grid nodes read as zero),
      // the four loads of a thread in flight together.
      constexpr int kPer = kRegionNodes / kGatherThreads;
      static_assert(kPer * kGatherThreads == kRegionNodes, "the block splits evenly over the CTA");
      float4 g[kPer];
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int r = (int)threadIdx.x + q * kGatherThreads;
        const int64_t c = node_index(sc, p.tile_slot, rx + (r & 7), ry + ((r >> 3) & 7), rz + (r >> 6));
        g[q] = c >= 0 ? __ldg(&p.vel[c]) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int q = 0; q < kPer; ++q) s_gath.vel[(int)threadIdx.x + q * kGatherThreads] = g[q];
    }
    __syncthreads();
    const bool faulted = s_fault != 0;
    if (!faulted) {
      int b = 0;
      for (uint32_t k = tid; k < s_ctx.count; k += kGatherThreads, b ^= 1) {
        fetch(k + kGatherThreads, b ^ 1, s_ctx.start, s_ctx.count);
        cp_async_wait<1>();
        const uint32_t s = s_ctx.start + k;
        float4 rec[4];
        particle_step<MODE, WRITE_KEYS, SR>(p, sc, s, s_ctx, s_gath.vel, s_gath.fallback[threadIdx.x], stol, sweeps,
                                            reuse_svd, rec, &s_in[b][0][tid]);
        if constexpr (kScatter) {
          float4* r4 = reinterpret_cast<float4*>(p.rec) + 4 * (size_t)s;
          r4[0] = rec[0];
          r4[1] = rec[1];
          r4[2] = rec[2];
          r4[3] = rec[3];
        }
      }
    }
    cp_async_wait<0>();
    // s_it_next was published by the barrier after the staging; thread 0
    // overwrites it only after the barrier below
    const uint32_t next = s_it_next;
    __syncthreads();
    it = next;
  }
}

// Scatter of the next substep (mpm.wgsl:601-627): a particle with base =
// floor(x/dx - 0.5) and fx = x/dx - base deposits, at the node of offset
// (i,j,k), w m and w (m v + B d) with d = ((i,j,k) - fx) dx and w the
// quadratic B-spline weight.  Particles whose record mass is zero (numerical
// fault this substep) deposit nothing.
//
// Persistent CTAs over items (a tile's particles from the last regrouping,
// at most kStageMax), 192 threads.  Per item:
//  1. stage: the item's 64-byte records (contiguous slots) arrive in shared
//     memory as 2-D TMA tiles of 64 records (cp.async.bulk.tensor completing
//     on an mbarrier), issued while the previous item's block was flushed.
//     The tiles use the 64-byte swizzle: 16-byte chunk k of record j sits at
//     chunk k ^ ((j >> 1) & 3), which spreads the lanes' reads of one chunk
//     of different records over all shared-memory banks;
//  2. bin: every particle is binned by its current base cell among the 6^3
//     cells whose stencils fit the tile's 8^3-node block (a counting sort in
//     shared memory with warp-aggregated counters), so particles that moved
//     since the regrouping are grouped with their new cell-mates; one whose
//     stencil leaves the block deposits straight to HBM;
//  3. deposit: a thread takes one x-slab i of the stencil and one cell: the
//     tile's own cells as the regrouping dealt them to warps (so that a
//     warp's flush atomics fall on distinct banks, count-ordered within the
//     warp), the three slabs of a cell in adjacent lanes, then the non-empty
//     margin cells particles moved into (listed by the scan of step 2).  It
//     adds the nine slab-i node contributions of its cell's particles in
//     registers and issues 9 x 4 shared-memory atomics for the whole cell,
//     not per particle; no two lanes of a warp add to the same node;
//  4. flush: every non-empty node of the 8^3 block goes to HBM with one
//     float4 atomic and is cleared for the next item.
// Every wait on the stage is bounded (about one second); a wait that gives
// up sets kFaultDeviceWait in the scene's status word and ends the CTA after
// a second bounded wait for its copy in flight.
__device__ __noinline__ void deposit_global(float4 r0, float4 r1, float4 r2, float4 r3, float4* __restrict__ acc,
                                            uint8_t* __restrict__ touched, const SceneDev* __restrict__ scp,
                                            const uint32_t* __restrict__ tile_slot) {
  const SceneDev& sc = *scp;
  const int win[3] = {sc.winx, sc.winy, sc.winz};
  const float ox = sc.ox, oy = sc.oy, oz = sc.oz, inv_dx = sc.inv_dx, dx = sc.dx;
  const float B[9] = {r1.w, r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w};
  const float xp[3] = {(r0.x - ox) * inv_dx, (r0.y - oy) * inv_dx, (r0.z - oz) * inv_dx};
  float wgt[3][3], fx[3];
  int base[3];
  for (int a = 0; a < 3; ++a) {
    const float bf = floorf(xp[a] - 0.5f);
    base[a] = (int)bf - win[a];
    fx[a] = xp[a] - bf;
    quad_weights(fx[a], wgt[a]);
  }
  for (int q = 0; q < 27; ++q) {
    const int i = q / 9, j = (q / 3) % 3, k = q % 3;
    const int64_t c = node_index(sc, tile_slot, base[0] + i, base[1] + j, base[2] + k);
    if (c < 0) continue;
    const float wt = wgt[0][i] * wgt[1][j] * wgt[2][k];
    const float d0 = ((float)i - fx[0]) * dx, d1 = ((float)j - fx[1]) * dx, d2 = ((float)k - fx[2]) * dx;
    const float4 v = make_float4(wt * r0.w, wt * (r1.x + B[0] * d0 + B[3] * d1 + B[6] * d2),
                                 wt * (r1.y + B[1] * d0 + B[4] * d1 + B[7] * d2),
                                 wt * (r1.z + B[2] * d0 + B[5] * d1 + B[8] * d2));
    atomicAdd(&acc[c], v);
    touch(touched, c);
  }
}

constexpr int kLocalCells = 216;  // 6^3 base cells whose stencils fit the 8^3 block

// 16-byte chunk k of staged record j under the 64-byte swizzle.
__device__ __forceinline__ float4 stage_chunk(const float4* stage, uint32_t j, uint32_t k) {
  return stage[4 * j + (k ^ ((j >> 1) & 3u))];
}
__device__ __forceinline__ void stage_store(float4* stage, uint32_t j, const float4 (&rec)[4]) {
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) stage[4 * j + (k ^ ((j >> 1) & 3u))] = rec[k];
}

// Where an item's scatter lands: its scene's lattice and grid block, and the
// 8^3-node block origin (rx, ry, rz) of its tile.
struct ItemFrame {
  float ox, oy, oz, inv_dx, dx;
  int wx, wy, wz, rx, ry, rz, n;
  uint64_t grid_off;
  float4* acc;
  uint8_t* touched;
  const SceneDev* sc;         // the scene record (global memory)
  const uint32_t* tile_slot;  // sparse storage: slot of every tile key
};

__device__ __forceinline__ ItemFrame item_frame(const SceneDev& sc, const Item& item, float4* acc, uint8_t* touched,
                                                const uint32_t* tile_slot) {
  ItemFrame f;
  f.sc = &sc;
  f.tile_slot = tile_slot;
  f.ox = sc.ox;
  f.oy = sc.oy;
  f.oz = sc.oz;
  f.inv_dx = sc.inv_dx;
  f.dx = sc.dx;
  f.wx = sc.winx;
  f.wy = sc.winy;
  f.wz = sc.winz;
  const uint32_t w = sc.w;
  const uint32_t tx = item.tile % w, ty = (item.tile / w) % w, tz = item.tile / (w * w);
  f.rx = 4 * (int)tx - 1;
  f.ry = 4 * (int)ty - 1;
  f.rz = 4 * (int)tz - 1;
  f.n = (int)sc.n;
  f.grid_off = sc.grid_off;
  f.acc = acc;
  f.touched = touched;
  return f;
}

// Shared-memory working set of one scatter item.
struct ScatterShared {
  float acc[4][kRegionFloats];  // the 8^3-node block: m, p.x, p.y, p.z
  uint32_t cell[kLocalCells];   // counts, then exclusive starts
  uint16_t idx[kStageMax];      // item records sorted by local cell
  uint8_t margin[kLocalCells];  // non-empty local cells outside the tile's own 4^3
  uint32_t total, n_margin;
};

__device__ __forceinline__ bool core_cell_index(int lc) {
  const int lx = lc % 6, ly = (lc / 6) % 6, lz = lc / 36;
  return lx >= 1 && lx <= 4 && ly >= 1 && ly <= 4 && lz >= 1 && lz <= 4;
}

// Scatter step 2 (bin) for a CTA of T threads: every staged record is binned
// by its current base cell among the 6^3 local cells (counting sort with
// warp-aggregated counters); one whose stencil leaves the block deposits
// straight to HBM.  A binned record is rewritten in place in its deposit
// form (deposit_item): with fx = x/dx - base and Bd = B dx (columns Bdx,
// Bdy, Bdz for the x, y, z node offsets), the momentum the node of offset
// (i, j, k) receives per unit weight is q000 + i Bdx + j Bdy + k Bdz, where
// q000 = m v - fx0 Bdx - fx1 Bdy - fx2 Bdz (the reference's m v + B d with
// d = ((i, j, k) - fx) dx regrouped):
//   (m, q000), (Bdx, Bdy.x), (Bdy.y, Bdy.z, Bdz.x, Bdz.y), (Bdz.z, fx).
// Ends with a barrier after which cell[] holds exclusive starts and idx[]
// the sorted record indices.
template <int T>
__device__ __forceinline__ void bin_item(float4* stage, uint32_t count, bool live, const ItemFrame& f,
                                         ScatterShared& ss) {
  constexpr int kRounds = (kStageMax + T - 1) / T;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t bin[kRounds];  // local cell << 16 | rank, or 0xffffffff
#pragma unroll
  for (int q = 0; q < kRounds; ++q) {
    const uint32_t j = threadIdx.x + q * T;
    uint32_t lc = 0xffffu;
    if (live && j < count) {
      const float4 r0 = stage_chunk(stage, j, 0);
      if (r0.w != 0.f) {
        const float xp[3] = {(r0.x - f.ox) * f.inv_dx, (r0.y - f.oy) * f.inv_dx, (r0.z - f.oz) * f.inv_dx};
        const float bx = floorf(xp[0] - 0.5f), by = floorf(xp[1] - 0.5f), bz = floorf(xp[2] - 0.5f);
        const int lx = (int)bx - f.wx - f.rx;
        const int ly = (int)by - f.wy - f.ry;
        const int lz = (int)bz - f.wz - f.rz;
        if ((unsigned)lx < 6u && (unsigned)ly < 6u && (unsigned)lz < 6u) {
          lc = (uint32_t)(lx + 6 * (ly + 6 * lz));
          const float4 r1 = stage_chunk(stage, j, 1), r2 = stage_chunk(stage, j, 2), r3 = stage_chunk(stage, j, 3);
          const float fx0 = xp[0] - bx, fx1 = xp[1] - by, fx2 = xp[2] - bz;
          const float dx = f.dx;
          const float bdx[3] = {r1.w * dx, r2.x * dx, r2.y * dx};
          const float bdy[3] = {r2.z * dx, r2.w * dx, r3.x * dx};
          const float bdz[3] = {r3.y * dx, r3.z * dx, r3.w * dx};
          const float q[3] = {r1.x - fx0 * bdx[0] - fx1 * bdy[0] - fx2 * bdz[0],
                              r1.y - fx0 * bdx[1] - fx1 * bdy[1] - fx2 * bdz[1],
                              r1.z - fx0 * bdx[2] - fx1 * bdy[2] - fx2 * bdz[2]};
          const float4 t[4] = {make_float4(r0.w, q[0], q[1], q[2]), make_float4(bdx[0], bdx[1], bdx[2], bdy[0]),
                               make_float4(bdy[1], bdy[2], bdz[0], bdz[1]), make_float4(bdz[2], fx0, fx1, fx2)};
          stage_store(stage, j, t);
        } else {
          deposit_global(r0, stage_chunk(stage, j, 1), stage_chunk(stage, j, 2), stage_chunk(stage, j, 3), f.acc,
                         f.touched, f.sc, f.tile_slot);
        }
      }
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, lc);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lc != 0xffffu && lane == leader) base = atomicAdd(&ss.cell[lc], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    bin[q] = lc == 0xffffu ? 0xffffffffu : (lc << 16) | (base + __popc(peers & ((1u << lane) - 1u)));
  }
  __syncthreads();
  // exclusive scan of the 216 cell counts (warp 0, 7 cells per lane)
  if (threadIdx.x < 32) {
    uint32_t c[7], sum = 0;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const int cell = (int)lane * 7 + k;
      c[k] = cell < kLocalCells ? ss.cell[cell] : 0u;
      sum += c[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    uint32_t run = incl - sum;
    uint32_t n_margin = 0;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const int cell = (int)lane * 7 + k;
      if (cell < kLocalCells) ss.cell[cell] = run;
      run += c[k];
      // compact the non-empty margin cells (particles that left the tile's
      // own cells since the regrouping) into a short list
      const bool mar = cell < kLocalCells && c[k] != 0u && !core_cell_index(cell);
      const uint32_t ballot = __ballot_sync(0xffffffffu, mar);
      if (mar) ss.margin[n_margin + __popc(ballot & ((1u << lane) - 1u))] = (uint8_t)cell;
      n_margin += __popc(ballot);
    }
    if (lane == 31) {
      ss.total = incl;
      ss.n_margin = n_margin;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kRounds; ++q) {
    if (bin[q] != 0xffffffffu) ss.idx[ss.cell[bin[q] >> 16] + (bin[q] & 0xffffu)] = (uint16_t)(threadIdx.x + q * T);
  }
  __syncthreads();
}

// Scatter step 3 (deposit) for a CTA of T >= 192 threads.  The first 192
// threads take the (cell, x-slab) pairs of the tile's own 64 cells: each
// warp holds 10 cells from the per-item table `order` (k_item_order), which
// deals the cells so that a warp's 30 flush atomics of one node and channel
// fall on 30 different shared-memory banks, in particle-count order inside
// the warp (scatter -18% against a plain count order); the three slab
// threads of a cell sit in adjacent lanes (a quarter-warp of a 16-byte
// record load then reads about three records, not eight, and lanes reading
// the same record share a broadcast: -10%); the two spare lanes of each warp
// take the four cells of the remaining banks.  Then all T threads share
// the (margin cell, slab) pairs of the non-empty cells particles moved into
// (the compact list the scan built; scanning all 152 margin cells per item
// cost 10% of the scatter).  A thread adds the nine slab nodes of its cell's
// particles in registers and issues 9 x 4 shared-memory atomics for the whole
// cell; no two lanes of a warp add to the same node.
template <int T>
__device__ __forceinline__ void deposit_item(const float4* stage, const uint8_t* __restrict__ order,
                                             ScatterShared& ss) {
  static_assert(T >= 192, "the core cells take 6 warps of 10 cells x 3 slabs");
  const uint32_t total = ss.total;
  // per node of the slab: (p.x, p.y) and (p.z, m), accumulated in pairs
  float2 axy[9], azm[9];
  // Accumulates slab `slab` of the particles of local cell lc in registers
  // from their deposit-form records (bin_item); returns whether it had any.
  // Node (slab, j, k) gets w_slab(fx0) w_j(fx1) w_k(fx2) (m, q000 + slab Bdx +
  // j Bdy + k Bdz), the sums over j and k taken as running increments.
  auto accumulate = [&](int lc, int slab) {
#pragma unroll
    for (int q = 0; q < 9; ++q) axy[q] = azm[q] = make_float2(0.f, 0.f);
    // the slab's B-spline weight of t = fx0 - shift: 0.5 (1.5 - fx)^2,
    // 0.75 - (fx - 1)^2, 0.5 (fx - 0.5)^2
    const float shift = 1.5f - 0.5f * (float)slab;
    const bool mid = slab == 1;
    const float fslab = (float)slab;
    const uint32_t first = ss.cell[lc], end = lc == kLocalCells - 1 ? total : ss.cell[lc + 1];
    for (uint32_t t = first; t < end; ++t) {
      const uint32_t j = ss.idx[t];
      const float4 c0 = stage_chunk(stage, j, 0), c1 = stage_chunk(stage, j, 1), c2 = stage_chunk(stage, j, 2),
                   c3 = stage_chunk(stage, j, 3);
      const float ts = c3.y - shift;
      const float wi = mid ? fmaf(-ts, ts, 0.75f) : 0.5f * ts * ts;
      float wy[3], wz[3];
      quad_weights(c3.z, wy);
      quad_weights(c3.w, wz);
      // momentum at node (slab, 0, 0), paired with the mass: (q.x, q.y), (q.z, m)
      float2 qxy = make_float2(fmaf(fslab, c1.x, c0.y), fmaf(fslab, c1.y, c0.z));
      float2 qzm = make_float2(fmaf(fslab, c1.z, c0.w), c0.x);
      const float2 dyxy = make_float2(c1.w, c2.x), dzxy = make_float2(c2.z, c2.w);
      const float dyz = c2.y, dzz = c3.x;
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) {
        if (jj) {
          qxy = add2(qxy, dyxy);
          qzm.x += dyz;
        }
        const float wij = wi * wy[jj];
        float2 cxy = qxy, czm = qzm;
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
          if (kk) {
            cxy = add2(cxy, dzxy);
            czm.x += dzz;
          }
          const float wt = wij * wz[kk];
          const float2 w2 = make_float2(wt, wt);
          axy[3 * jj + kk] = fma2(w2, cxy, axy[3 * jj + kk]);
          azm[3 * jj + kk] = fma2(w2, czm, azm[3 * jj + kk]);
        }
      }
    }
    return end > first;
  };
  // Adds the accumulated slab of local cell lc to the shared block.
  auto flush = [&](int lc, int slab) {
    const int r0 = region_index(lc % 6, (lc / 6) % 6, lc / 36) + slab;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) {
        const int r = r0 + kRsy * j + kRsz * kk;
        atomicAdd(&ss.acc[0][r], azm[3 * j + kk].y);
        atomicAdd(&ss.acc[1][r], axy[3 * j + kk].x);
        atomicAdd(&ss.acc[2][r], axy[3 * j + kk].y);
        atomicAdd(&ss.acc[3][r], azm[3 * j + kk].x);
      }
  };
  // local cell (in the 6^3 frame) of slot `slot` of the item's table
  auto core_cell = [&](uint32_t slot) {
    const uint32_t c = order[slot];
    return (int)((c & 3u) + 1) + 6 * ((int)((c >> 2) & 3u) + 1 + 6 * ((int)(c >> 4) + 1));
  };
  // Warp w takes slots 10w..10w+9, the three slab threads of a cell in
  // adjacent lanes: a quarter-warp of a 16-byte record load then touches
  // about three records instead of eight, and the lanes that read the same
  // record are served by one broadcast.  The two spare lanes of each warp
  // (12 in all) take the 3 slabs of slots 60..63.
  if (threadIdx.x < 192) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t q = warp * 2u + (lane - 30u);  // spare-lane index when lane >= 30
    const uint32_t slot = lane < 30u ? warp * 10u + lane / 3u : 60u + q / 3u;
    const int slab = (int)(lane < 30u ? lane % 3u : q % 3u);
    const int lc = core_cell(slot);
    if (accumulate(lc, slab)) flush(lc, slab);
  }
  // then the (margin cell, slab) pairs of the non-empty margin cells
  const int n_margin = (int)ss.n_margin;
#pragma unroll 1
  for (int u = (int)threadIdx.x; u < 3 * n_margin; u += T) {
    const int lc = ss.margin[u % n_margin], slab = u / n_margin;
    if (accumulate(lc, slab)) flush(lc, slab);
  }
}

// Scatter step 4 (flush): every non-empty node of the 8^3 block goes to HBM
// with one float4 atomic and is cleared for the next item, as are the cell
// counters.  The caller synchronises before the block is reused.
template <int T>
__device__ __forceinline__ void flush_item(const ItemFrame& f, ScatterShared& ss) {
  for (int r = threadIdx.x; r < kRegionNodes; r += T) {
    const int lx = r & 7, ly = (r >> 3) & 7, lz = r >> 6;
    const int q = region_index(lx, ly, lz);
    const float m = ss.acc[0][q], px = ss.acc[1][q], py = ss.acc[2][q], pz = ss.acc[3][q];
    if (m != 0.f || px != 0.f || py != 0.f || pz != 0.f) {
      ss.acc[0][q] = 0.f;
      ss.acc[1][q] = 0.f;
      ss.acc[2][q] = 0.f;
      ss.acc[3][q] = 0.f;
      const int64_t c = node_index(*f.sc, f.tile_slot, f.rx + lx, f.ry + ly, f.rz + lz);
      if (c >= 0) {
        atomicAdd(&f.acc[c], make_float4(m, px, py, pz));
        touch(f.touched, (uint64_t)c);
      }
    }
  }
  for (int r = threadIdx.x; r < kLocalCells; r += T) ss.cell[r] = 0u;
}

__device__ __forceinline__ void clear_scatter_shared(ScatterShared& ss, int threads) {
  for (int r = threadIdx.x; r < 4 * kRegionFloats; r += threads) (&ss.acc[0][0])[r] = 0.f;
  for (int r = threadIdx.x; r < kLocalCells; r += threads) ss.cell[r] = 0u;
}

__global__ void __launch_bounds__(kScatterThreads, 4) k_p2g(PoolDev p, const __grid_constant__ CUtensorMap rec_map,
                                                            int acc_out) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  // the swizzle pattern repeats every 512 bytes: align the stage to 1 KiB
  float4* s_stage =
      reinterpret_cast<float4*>((reinterpret_cast<uintptr_t>(s_dyn) + 1023u) & ~static_cast<uintptr_t>(1023u));
  __shared__ ScatterShared ss;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_it_next;
  float4* __restrict__ acc = p.acc[acc_out];
  uint8_t* __restrict__ touched = p.touched[acc_out];
  const uint32_t n32 = p.n_items[0];
  const uint32_t n_items = n32 + p.n_items[1];
  clear_scatter_shared(ss, kScatterThreads);
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  // Thread 0 stages item `it` (items of 1..kStageMax particles) as
  // ceil(count / 64) tiles; rows past the item are loaded but not read.
  auto stage = [&](uint32_t it) {
    const Item nx = p.items[item_slot(p, n32, it)];
    if (nx.count - 1u < (uint32_t)kStageMax) {
      const uint32_t boxes = (nx.count + kStageBoxRows - 1) / kStageBoxRows;
      fence_proxy_async_smem();
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&s_bar)),
                   "r"(boxes * kStageBoxRows * 64u)
                   : "memory");
      for (uint32_t b = 0; b < boxes; ++b)
        tma_load_rows(s_stage + (size_t)b * kStageBoxRows * 4, &rec_map, (int)(nx.start + b * kStageBoxRows), &s_bar);
    }
  };
  if (threadIdx.x == 0 && blockIdx.x < n_items) stage(blockIdx.x);
  uint32_t parity = 0;
  for (uint32_t it = blockIdx.x; it < n_items;) {
    // this CTA's next item, taken now; its records are staged after this
    // item's deposit
    if (threadIdx.x == 0) s_it_next = gridDim.x + atomicAdd(p.work + 1, 1u);
    const uint32_t slot = item_slot(p, n32, it);
    const Item item = p.items[slot];
    const SceneDev* __restrict__ scp = p.scenes + item.scene;
    uint32_t* status = p.status + (size_t)scp->status * kStatusWords;
    // A fault latched before this launch (or a spent substep budget, or a
    // retired scene) freezes the scene; one latched by this substep's gather
    // is handled per particle (m = 0 in its record).
    const uint32_t fault0 = (scene_frozen(status) || !scp->live) ? 1u : 0u;
    const ItemFrame f = item_frame(*scp, item, acc, touched, p.tile_slot);
    const bool staged = item.count - 1u < (uint32_t)kStageMax;
    bool ok = staged;
    if (staged) {
      ok = mbar_wait_bounded(&s_bar, parity);
      parity ^= 1u;
    }
    const bool live = ok && fault0 == 0;
    bin_item<kScatterThreads>(s_stage, item.count, live, f, ss);
    if (live) deposit_item<kScatterThreads>(s_stage, p.item_order + (size_t)slot * 64, ss);
    if (__syncthreads_or(!ok)) {
      // The stage did not arrive (or the item exceeds the stage): report it,
      // wait once more (bounded) for the copy in flight and stop this CTA.
      if (threadIdx.x == 0) atomicOr(status, kFaultDeviceWait);
      if (staged) mbar_wait_bounded(&s_bar, parity ^ 1u);
      return;
    }
    // Every thread is done with the stage: the next item's copy goes now.
    // (s_it_next was published by the bin's barriers; thread 0 overwrites
    // it only after the barrier below.)
    const uint32_t next = s_it_next;
    if (threadIdx.x == 0 && next < n_items) stage(next);
    flush_item<kScatterThreads>(f, ss);
    __syncthreads();
    it = next;
  }
}

// Fused gather + scatter of one substep (non-deterministic P2G): per item,
// the CTA runs the gather of every particle (G2P, F update, return mapping,
// B record) with the record kept in shared memory instead of HBM, then bins,
// deposits and flushes the item's records as k_p2g does.  Saves the record's
// 64-byte write and read per particle and one launch, and lets the gather
// (FP32/FP64/XU pipes) of one CTA overlap the deposit (shared-memory
// atomics) of the other CTA on the SM.  Items hold at most kStageMax
// particles (the regrouping cuts them), so the records fit the stage; an
// item that does not fit latches kFaultDeviceWait and is skipped.
//
// A fault latched before an item starts freezes the item (no gather, no
// deposit); a particle that faults during the gather deposits nothing (m = 0
// in its record).  The scene is frozen from the next substep on.
template <bool WRITE_KEYS, class SR>
__global__ void __launch_bounds__(kFusedThreads, 2) k_g2p2g(PoolDev p, double tol, int sweeps, int reuse_svd,
                                                              int acc_out) {
  extern __shared__ __align__(16) float4 s_stage[];  // kStageMax records, 64-byte swizzle
  __shared__ __align__(16) SceneDev s_sc;
  __shared__ __align__(16) float4 s_vel[kRegionNodes];
  __shared__ ScatterShared ss;
  __shared__ uint32_t s_fault;
  __shared__ GatherCtx s_ctx;
  float4* __restrict__ acc = p.acc[acc_out];
  uint8_t* __restrict__ touched = p.touched[acc_out];
  // this SVD form's range of the work list: FP32-SVD items, then FP64-SVD items
  const uint32_t n32 = p.n_items[0];
  const uint32_t it_lo = sizeof(SR) == 8 ? n32 : 0u;
  const uint32_t it_hi = sizeof(SR) == 8 ? n32 + p.n_items[1] : n32;
  const SR stol = (SR)tol;
  clear_scatter_shared(ss, kFusedThreads);
  for (uint32_t it = it_lo + blockIdx.x; it < it_hi; it += gridDim.x) {
    const uint32_t slot = item_slot(p, n32, it);
    const Item item = p.items[slot];
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(p.scenes + item.scene);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_sc);
      for (int k = threadIdx.x; k < (int)(sizeof(SceneDev) / 4); k += kFusedThreads) dst[k] = src[k];
    }
    const SceneDev* __restrict__ scp = p.scenes + item.scene;
    uint32_t* status = p.status + (size_t)scp->status * kStatusWords;
    const uint32_t fault0 = (scene_frozen(status) || !scp->live) ? 1u : 0u;
    const bool publish_vc = budget_ends(status);
    const ItemFrame f = item_frame(*scp, item, acc, touched, p.tile_slot);
    const bool fits = item.count <= (uint32_t)kStageMax;
    {
      // Stage the 8^3-node velocity block (out-of-grid nodes read as zero).
      for (int r = threadIdx.x; r < kRegionNodes; r += kFusedThreads) {
        const int64_t c = node_index(*scp, p.tile_slot, f.rx + (r & 7), f.ry + ((r >> 3) & 7), f.rz + (r >> 6));
        s_vel[r] = c >= 0 ? __ldg(&p.vel[c]) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    if (threadIdx.x == 0) {
      s_fault = fault0;
      s_ctx = GatherCtx{status, f.rx, f.ry, f.rz, publish_vc ? 1u : 0u, item.start, item.count};
      if (!fits) atomicOr(status, kFaultDeviceWait);
    }
    __syncthreads();
    const bool live = s_fault == 0 && fits;
    if (live) {
      for (uint32_t k = threadIdx.x; k < item.count; k += kFusedThreads) {
        float4 rec[4];
        // the record's own stage slot is the scratch of gather_global
        particle_step<kG2PRecord, WRITE_KEYS, SR>(p, s_sc, item.start + k, s_ctx, s_vel,
                                                  reinterpret_cast<float*>(s_stage + 4 * (size_t)k), stol, sweeps,
                                                  reuse_svd, rec);
        stage_store(s_stage, k, rec);
      }
    }
    __syncthreads();
    bin_item<kFusedThreads>(s_stage, item.count, live, f, ss);
    if (live) deposit_item<kFusedThreads>(s_stage, p.item_order + (size_t)slot * 64, ss);
    __syncthreads();
    flush_item<kFusedThreads>(f, ss);
    __syncthreads();
  }
}

// Deterministic scatter (the fixed-order P2G of molla's
// mpm_deterministic_p2g.wgsl:85-150, restructured per tile).  Requires a
// regrouping after every gather, so that every particle of a tile item sits
// in its own base cell.  Thread (cell, slab) sums its cell's particles in slot
// order — (key, identity) order — in registers; the CTA then reduces the
// (cell, slab) partial sums of each of the tile's 6^3 footprint nodes in a
// fixed cell order and stores the block, without atomics.  A combine pass
// adds the blocks of the tiles covering each node, again in a fixed order.
// The result depends only on the scene's own particles and identities: it is
// bit-identical from run to run and whether or not other scenes share the
// launch.
__global__ void __launch_bounds__(kScatterThreads, 2) k_p2g_det(PoolDev p, float4* __restrict__ blocks, int acc_out) {
  __shared__ uint32_t s_first[64], s_end[64];
  __shared__ float s_part[3 * 64 * 9 * 4];
  __shared__ uint32_t s_fault;
  const float4* __restrict__ rec = reinterpret_cast<const float4*>(p.rec);
  const uint32_t n32 = p.n_items[0];
  const uint32_t n_items = n32 + p.n_items[1];
  const int cell = threadIdx.x & 63;
  const int slab = threadIdx.x >> 6;
  for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
    const uint32_t slot = item_slot(p, n32, it);
    const Item item = p.items[slot];
    const SceneDev* __restrict__ scp = p.scenes + item.scene;
    const uint32_t w = scp->w;
    const float ox = scp->ox, oy = scp->oy, oz = scp->oz, inv_dx = scp->inv_dx, dx = scp->dx;
    const int winx = scp->winx, winy = scp->winy, winz = scp->winz;
    uint32_t* status = p.status + (size_t)scp->status * kStatusWords;
    const uint32_t tx = item.tile % w, ty = (item.tile / w) % w, tz = item.tile / (w * w);
    if (threadIdx.x == 0) s_fault = (scene_frozen(status) || !scp->live) ? 1u : 0u;
    if (threadIdx.x < 64) {
      s_first[threadIdx.x] = 0;
      s_end[threadIdx.x] = 0;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < item.count; k += blockDim.x) {
      const uint32_t s = item.start + k;
      const uint32_t c = p.slot_key[s] & 63u;
      if (k == 0 || (p.slot_key[s - 1] & 63u) != c) s_first[c] = s;
      if (k + 1 == item.count || (p.slot_key[s + 1] & 63u) != c) s_end[c] = s + 1;
    }
    __syncthreads();
    float am[9], apx[9], apy[9], apz[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) am[q] = apx[q] = apy[q] = apz[q] = 0.f;
    if (s_fault == 0) {
      const int cx = cell & 3, cy = (cell >> 2) & 3, cz = cell >> 4;
      const int bx = 4 * (int)tx + cx, by = 4 * (int)ty + cy, bz = 4 * (int)tz + cz;  // this cell's base
      const int win[3] = {winx, winy, winz};
      for (uint32_t s = s_first[cell]; s < s_end[cell]; ++s) {
        const float4 r0 = __ldg(&rec[4 * (size_t)s]);
        if (r0.w == 0.f) continue;
        const float4 r1 = __ldg(&rec[4 * (size_t)s + 1]);
        const float4 r2 = __ldg(&rec[4 * (size_t)s + 2]);
        const float4 r3 = __ldg(&rec[4 * (size_t)s + 3]);
        const float mass = r0.w;
        const float B[9] = {r1.w, r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w};
        const float xp[3] = {(r0.x - ox) * inv_dx, (r0.y - oy) * inv_dx, (r0.z - oz) * inv_dx};
        float wgt[3][3], fx[3];
        int base[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float bf = floorf(xp[a] - 0.5f);
          base[a] = (int)bf - win[a];
          fx[a] = xp[a] - bf;
          quad_weights(fx[a], wgt[a]);
        }
        const float wi = slab == 0 ? wgt[0][0] : (slab == 1 ? wgt[0][1] : wgt[0][2]);
        const float di = ((float)slab - fx[0]) * dx;
        const float qx[3] = {r1.x + B[0] * di, r1.y + B[1] * di, r1.z + B[2] * di};
        const bool own = base[0] == bx && base[1] == by && base[2] == bz;
        if (!own && slab == 0 && threadIdx.x < 64) atomicOr(status, kFaultNondeterministic);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float wij = wi * wgt[1][j];
          const float dj = ((float)j - fx[1]) * dx;
          const float qy[3] = {qx[0] + B[3] * dj, qx[1] + B[4] * dj, qx[2] + B[5] * dj};
#pragma unroll
          for (int kk = 0; kk < 3; ++kk) {
            const float wt = wij * wgt[2][kk];
            const float dk = ((float)kk - fx[2]) * dx;
            const float dm = wt * mass;
            const float px = wt * (qy[0] + B[6] * dk);
            const float py = wt * (qy[1] + B[7] * dk);
            const float pz = wt * (qy[2] + B[8] * dk);
            if (own) {
              am[3 * j + kk] += dm;
              apx[3 * j + kk] += px;
              apy[3 * j + kk] += py;
              apz[3 * j + kk] += pz;
            } else {
              // Not in its cell (positions set from outside the grid since
              // the last regrouping): deposited with an atomic that the
              // combine pass adds to, outside the fixed order; flagged in
              // the status word.
              const int64_t c = node_index(*scp, p.tile_slot, base[0] + slab, base[1] + j, base[2] + kk);
              if (c >= 0) {
                atomicAdd(&p.acc[acc_out][c], make_float4(dm, px, py, pz));
                touch(p.touched[acc_out], (uint64_t)c);
              }
            }
          }
        }
      }
    }
    {
      float* dst = s_part + ((slab * 64 + cell) * 9) * 4;
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        dst[4 * q] = am[q];
        dst[4 * q + 1] = apx[q];
        dst[4 * q + 2] = apy[q];
        dst[4 * q + 3] = apz[q];
      }
    }
    __syncthreads();
    // Node (nx, ny, nz) of the 6^3 footprint receives, from cell (cx, cy, cz)
    // with 0 <= n - c <= 2 per axis, the partial sum stored by thread
    // (cell, slab = nx - cx) at index 3 (ny - cy) + (nz - cz).
    float4* blk = blocks + (size_t)slot * kTileNodes;
    for (int q = threadIdx.x; q < kTileNodes; q += blockDim.x) {
      const int nx = q % 6, ny = (q / 6) % 6, nz = q / 36;
      float sm = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
      for (int cz = max(0, nz - 2); cz <= min(3, nz); ++cz)
        for (int cy = max(0, ny - 2); cy <= min(3, ny); ++cy)
          for (int cx = max(0, nx - 2); cx <= min(3, nx); ++cx) {
            const float* src = s_part + (((nx - cx) * 64 + (cx + 4 * cy + 16 * cz)) * 9 + 3 * (ny - cy) + (nz - cz)) * 4;
            sm += src[0];
            sx += src[1];
            sy += src[2];
            sz += src[3];
          }
      blk[q] = make_float4(sm, sx, sy, sz);
    }
    __syncthreads();
  }
}

// Combine pass of the deterministic scatter: node g of a scene receives the
// blocks of the (up to 8) occupied tiles whose footprint [4t, 4t+5] contains
// it, summed in (tz, ty, tx) order by the first such tile's thread.
__global__ void k_combine_det(PoolDev p, const float4* __restrict__ blocks, const uint32_t* __restrict__ tile_item,
                              int acc_out) {
  const uint32_t n32 = p.n_items[0];
  if (blockIdx.x >= n32 + p.n_items[1]) return;
  const uint32_t it = item_slot(p, n32, blockIdx.x);  // the item's slot, as tile_item holds it
  const Item item = p.items[it];
  const SceneDev* __restrict__ scp = p.scenes + item.scene;
  const int w = (int)scp->w, n = (int)scp->n;
  const uint32_t key_off = scp->key_off;
  const int tx = (int)(item.tile % (uint32_t)w), ty = (int)((item.tile / (uint32_t)w) % (uint32_t)w),
            tz = (int)(item.tile / (uint32_t)(w * w));
  for (int q = threadIdx.x; q < kTileNodes; q += blockDim.x) {
    const int g[3] = {4 * tx + q % 6, 4 * ty + (q / 6) % 6, 4 * tz + q / 36};
    if (g[0] >= n || g[1] >= n || g[2] >= n) continue;
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      hi[a] = g[a] / 4;
      lo[a] = max(0, (g[a] - 5 + 3) / 4);  // smallest t with 4t + 5 >= g
      hi[a] = min(hi[a], w - 1);
    }
    bool mine = false, found = false;
    float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int cz = lo[2]; cz <= hi[2]; ++cz)
      for (int cy = lo[1]; cy <= hi[1]; ++cy)
        for (int cx = lo[0]; cx <= hi[0]; ++cx) {
          const uint32_t key = key_off + (uint32_t)(cx + w * (cy + w * cz));
          const uint32_t other = tile_item[key];
          if (other == 0xffffffffu) continue;
          if (!found) {
            found = true;
            mine = other == it;
            if (!mine) break;
          }
          const int l = (g[0] - 4 * cx) + 6 * ((g[1] - 4 * cy) + 6 * (g[2] - 4 * cz));
          const float4 b = blocks[(size_t)other * kTileNodes + l];
          sum.x += b.x;
          sum.y += b.y;
          sum.z += b.z;
          sum.w += b.w;
        }
    const int64_t c = mine ? node_index(*scp, p.tile_slot, g[0], g[1], g[2]) : -1;
    if (c >= 0) {
      // One writer per node; the cell holds zero or out-of-order deposits.
      float4& a = p.acc[acc_out][c];
      const float4 old = a;
      a = make_float4(old.x + sum.x, old.y + sum.y, old.z + sum.z, old.w + sum.w);
      touch(p.touched[acc_out], (uint64_t)c);
    }
  }
}

// ---------------------------------------------------------------------------

template <int MODE, bool KEYS, class SR>
static cudaError_t launch_gather_t(const PoolDev& p, double tol, int sweeps, int reuse, int grid, cudaStream_t st,
                                   bool publish_all) {
  const cudaError_t e = cudaMemsetAsync(p.work, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  k_g2p<MODE, KEYS, SR><<<grid, kGatherThreads, 0, st>>>(p, tol, sweeps, reuse, publish_all ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_gather(int mode, bool write_keys, bool svd_fp64, const PoolDev& p, double tol, int sweeps,
                          int reuse, int grid, cudaStream_t st, bool publish_all) {
#define MPM_DISPATCH(M)                                                                          \
  if (mode == M) {                                                                               \
    if (svd_fp64) {                                                                              \
      return write_keys ? launch_gather_t<M, true, double>(p, tol, sweeps, reuse, grid, st, publish_all) \
                        : launch_gather_t<M, false, double>(p, tol, sweeps, reuse, grid, st, publish_all); \
    }                                                                                            \
    return write_keys ? launch_gather_t<M, true, float>(p, tol, sweeps, reuse, grid, st, publish_all) \
                      : launch_gather_t<M, false, float>(p, tol, sweeps, reuse, grid, st, publish_all); \
  }
  MPM_DISPATCH(kRecord)
  MPM_DISPATCH(kG2P)
  MPM_DISPATCH(kG2PRecord)
#undef MPM_DISPATCH
  return cudaErrorInvalidValue;
}

constexpr size_t kFusedStageBytes = (size_t)kStageMax * 64;

template <bool KEYS, class SR>
static cudaError_t launch_fused_t(const PoolDev& p, double tol, int sweeps, int reuse, int acc_out, int grid,
                                  cudaStream_t st) {
  k_g2p2g<KEYS, SR><<<grid, kFusedThreads, kFusedStageBytes, st>>>(p, tol, sweeps, reuse, acc_out);
  return cudaGetLastError();
}

cudaError_t launch_fused(bool write_keys, bool svd_fp64, const PoolDev& p, double tol, int sweeps, int reuse,
                         int acc_out, int grid, cudaStream_t st) {
  if (svd_fp64)
    return write_keys ? launch_fused_t<true, double>(p, tol, sweeps, reuse, acc_out, grid, st)
                      : launch_fused_t<false, double>(p, tol, sweeps, reuse, acc_out, grid, st);
  return write_keys ? launch_fused_t<true, float>(p, tol, sweeps, reuse, acc_out, grid, st)
                    : launch_fused_t<false, float>(p, tol, sweeps, reuse, acc_out, grid, st);
}

// stage tiles plus 1 KiB for the alignment of the swizzled stage
constexpr size_t kStageBytes = (size_t)kStageMax * 64 + 1024;
static_assert(kStageMax % kStageBoxRows == 0, "the stage holds whole TMA tiles");

bool make_record_map(CUtensorMap* out, const float* rec, uint32_t cap, std::string* err) {
  using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      if (err) *err = "cuTensorMapEncodeTiled is not available from the driver";
      return false;
    }
    encode = reinterpret_cast<EncodeFn>(fn);
  }
  // records: rows of 16 floats (64 bytes), cap rows; tiles of 64 rows
  const cuuint64_t dims[2] = {16, cap ? cap : 1};
  const cuuint64_t strides[1] = {64};
  const cuuint32_t box[2] = {16, (cuuint32_t)kStageBoxRows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(rec), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    if (err) *err = "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r);
    return false;
  }
  return true;
}

// Self-test of the scatter's bounded stage wait: one warp waits, through the
// same mbar_wait_bounded, on an mbarrier phase that nothing completes (one
// expected arrival, none made), then reports the way k_p2g does
// (kFaultDeviceWait in the status word) and records how long it waited.  No
// copy is in flight, so the CTA may end there.
__global__ void __launch_bounds__(32) k_selftest_wait(uint32_t* status, unsigned long long* waited_ns) {
  __shared__ __align__(8) uint64_t s_bar;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t t0 = global_ns();
  const bool ok = mbar_wait_bounded(&s_bar, 0u);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) {
    atomicOr(status, kFaultDeviceWait);
    *waited_ns = global_ns() - t0;
  }
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&s_bar)) : "memory");
}

cudaError_t launch_selftest_wait(uint32_t* status, unsigned long long* waited_ns, cudaStream_t st) {
  k_selftest_wait<<<1, 32, 0, st>>>(status, waited_ns);
  return cudaGetLastError();
}

cudaError_t launch_scatter(const PoolDev& p, const CUtensorMap& rec_map, int acc_out, int grid, cudaStream_t st) {
  const cudaError_t e = cudaMemsetAsync(p.work + 1, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  k_p2g<<<grid, kScatterThreads, kStageBytes, st>>>(p, rec_map, acc_out);
  return cudaGetLastError();
}

cudaError_t launch_scatter_det(const PoolDev& p, float4* blocks, int acc_out, int grid, cudaStream_t st) {
  k_p2g_det<<<grid, kScatterThreads, 0, st>>>(p, blocks, acc_out);
  return cudaGetLastError();
}

cudaError_t launch_combine_det(const PoolDev& p, const float4* blocks, const uint32_t* tile_item, uint32_t max_items,
                               int acc_out, cudaStream_t st) {
  if (!max_items) return cudaSuccess;
  k_combine_det<<<max_items, 128, 0, st>>>(p, blocks, tile_item, acc_out);
  return cudaGetLastError();
}

static int persistent(const void* fn, int threads, size_t dyn_smem = 0) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, dyn_smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  if (sms < 1) sms = 148;
  return sms * per_sm;
}

int gather_grid_size(bool svd_fp64) {
  return svd_fp64 ? persistent((const void*)k_g2p<kG2PRecord, false, double>, kGatherThreads)
                  : persistent((const void*)k_g2p<kG2PRecord, false, float>, kGatherThreads);
}

int fused_grid_size(bool svd_fp64) {
  // the record stage needs more than the default 48 KB of dynamic shared memory
  const void* fns[4] = {(const void*)k_g2p2g<false, double>, (const void*)k_g2p2g<true, double>,
                        (const void*)k_g2p2g<false, float>, (const void*)k_g2p2g<true, float>};
  for (const void* fn : fns)
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedStageBytes);
  return persistent(svd_fp64 ? fns[0] : fns[2], kFusedThreads, kFusedStageBytes);
}

int scatter_grid_size() {
  // the record stage needs more than the default 48 KB of dynamic shared memory
  cudaFuncSetAttribute((const void*)k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageBytes);
  return persistent((const void*)k_p2g, kScatterThreads, kStageBytes);
}

}  // namespace mpm
