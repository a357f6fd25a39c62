// mpm_kernels.cu — the substep kernels of the B200 MLS-MPM path.
//
// One substep of the reference (crates/molla-solvers/src/mpm.rs:2476-2551:
// reset_grid, p2g, grid_update, g2p, plasticity) runs here as two launches:
//
//   grid_update(n)            acc[a] -> velocity, clears acc[b]   (HBM sweep)
//   particles(n)              G2P(n) + plasticity(n) + P2G(n+1) into acc[b]
//
// The particle kernel is persistent over a work list of (scene, tile, slot
// range) items produced by the last regrouping sort: each CTA takes an item,
// accumulates the item's P2G contributions in a 9^3-node shared-memory block
// around the tile, and flushes the non-empty nodes to HBM with one float4
// atomic each.  The particle state of the next step stays in registers
// between the gather and the scatter, so each particle is read once and
// written once per substep, and the SVD computed by the plasticity return
// mapping is reused for the next step's stress (F was rebuilt from exactly
// that U, diag(s), V).  The first substep of every step_n call runs a
// P2G-only launch that computes the SVD from F.
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

// Adds one node contribution to the shared block or, outside it, to HBM.
__device__ __forceinline__ void deposit(float (*s_acc)[kRegionNodes], int rx, int ry, int rz, int ix, int iy,
                                        int iz, int n, float4* __restrict__ acc, uint64_t grid_off, float dm,
                                        float px, float py, float pz) {
  const unsigned lx = (unsigned)(ix - rx), ly = (unsigned)(iy - ry), lz = (unsigned)(iz - rz);
  if (lx < (unsigned)kRegion && ly < (unsigned)kRegion && lz < (unsigned)kRegion) {
    const int r = (int)lx + kRegion * ((int)ly + kRegion * (int)lz);
    atomicAdd(&s_acc[0][r], dm);
    atomicAdd(&s_acc[1][r], px);
    atomicAdd(&s_acc[2][r], py);
    atomicAdd(&s_acc[3][r], pz);
  } else if ((unsigned)ix < (unsigned)n && (unsigned)iy < (unsigned)n && (unsigned)iz < (unsigned)n) {
    const uint64_t c = grid_off + (uint64_t)ix + (uint64_t)n * ((uint64_t)iy + (uint64_t)n * (uint64_t)iz);
    atomicAdd(&acc[c], make_float4(dm, px, py, pz));
  }
}

// 27-node APIC scatter of one particle (mpm.wgsl:601-627): node at offset
// (i,j,k) from base receives w*m and w*(m v + B d), d = ((i,j,k) - fx) dx.
__device__ __forceinline__ void scatter_particle(float (*s_acc)[kRegionNodes], int rx, int ry, int rz,
                                                 const SceneDev& sc, float4* __restrict__ acc, float x, float y,
                                                 float z, float mass, const float* v, const float* B) {
  const float xp[3] = {(x - sc.ox) * sc.inv_dx, (y - sc.oy) * sc.inv_dx, (z - sc.oz) * sc.inv_dx};
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
  const float mv[3] = {mass * v[0], mass * v[1], mass * v[2]};
  const int n = (int)sc.n;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    // B d = B[:,0] dx_i + B[:,1] dy_j + B[:,2] dz_k, split by axis.
    const float qx[3] = {mv[0] + B[0] * d[0][i], mv[1] + B[1] * d[0][i], mv[2] + B[2] * d[0][i]};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float wij = w[0][i] * w[1][j];
      const float qy[3] = {qx[0] + B[3] * d[1][j], qx[1] + B[4] * d[1][j], qx[2] + B[5] * d[1][j]};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float wt = wij * w[2][k];
        const float px = wt * (qy[0] + B[6] * d[2][k]);
        const float py = wt * (qy[1] + B[7] * d[2][k]);
        const float pz = wt * (qy[2] + B[8] * d[2][k]);
        deposit(s_acc, rx, ry, rz, base[0] + i, base[1] + j, base[2] + k, n, acc, sc.grid_off, wt * mass, px, py,
                pz);
      }
    }
  }
}

template <class T>
__device__ __forceinline__ T svd_tol_cast(double t) {
  return (T)t;
}

}  // namespace

// ---------------------------------------------------------------------------
// The particle kernel.  MODE: kP2G (scatter only, SVD from F), kG2P (gather +
// plasticity, no scatter: the last substep of a call), kG2P2G (gather +
// plasticity + scatter of the next substep with the reused SVD).
template <int MODE, bool WRITE_KEYS, class SR>
__global__ void __launch_bounds__(kParticleThreads) k_particles(PoolDev p, int acc_out, double tol, int sweeps,
                                                                int reuse_svd) {
  constexpr bool kGather = MODE != kP2G;
  constexpr bool kScatter = MODE != kG2P;
  __shared__ float s_acc[kScatter ? 4 : 1][kScatter ? kRegionNodes : 1];
  __shared__ uint32_t s_fault;
  float4* __restrict__ acc = p.acc[acc_out];
  const uint32_t n_items = *p.n_items;
  const SR stol = svd_tol_cast<SR>(tol);
  for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item item = p.items[it];
    const SceneDev& sc = p.scenes[item.scene];
    uint32_t* status = p.status + (size_t)sc.status * kStatusWords;
    if (threadIdx.x == 0) s_fault = *(volatile uint32_t*)status;
    const uint32_t tx = item.tile % sc.w, ty = (item.tile / sc.w) % sc.w, tz = item.tile / (sc.w * sc.w);
    const int rx = 4 * (int)tx - 2, ry = 4 * (int)ty - 2, rz = 4 * (int)tz - 2;
    if constexpr (kScatter) {
      for (int r = threadIdx.x; r < kRegionNodes; r += blockDim.x) {
        s_acc[0][r] = 0.f;
        s_acc[1][r] = 0.f;
        s_acc[2][r] = 0.f;
        s_acc[3][r] = 0.f;
      }
    }
    __syncthreads();
    const bool faulted = s_fault != 0;
    if (!faulted) {
      for (uint32_t k = threadIdx.x; k < item.count; k += blockDim.x) {
        const uint32_t s = item.start + k;
        float x = plane(p, PX)[s], y = plane(p, PY)[s], z = plane(p, PZ)[s];
        float F[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) F[i] = plane(p, F0 + i)[s];
        float jp = plane(p, JP)[s];
        const float mass = plane(p, MASS)[s];
        const float vol = plane(p, VOL)[s];
        const uint32_t meta = p.meta[s];
        const MatDev& md = sc.mat[meta & 7u];
        float v[3], C[9];
        bool ok = true;
        SvdOut<SR> svd;
        if constexpr (kGather) {
          // ---- g2p (mpm.wgsl:1242-1353) ----
          bool fin = finitef(x) && finitef(y) && finitef(z) && finitef(jp);
#pragma unroll
          for (int i = 0; i < 9; ++i) fin = fin && finitef(F[i]);
          const float xp[3] = {(x - sc.ox) * sc.inv_dx, (y - sc.oy) * sc.inv_dx, (z - sc.oz) * sc.inv_dx};
          fin = fin && finitef(xp[0]) && finitef(xp[1]) && finitef(xp[2]);
          if (!fin) {
            atomicOr(status, kFaultNumerical);
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
            // Separable accumulation: v = sum w gv; G = sum (w gv) d^T.
            float vs[3] = {0.f, 0.f, 0.f};
            float G[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) G[i] = 0.f;
            const int n = (int)sc.n;
            const float4* __restrict__ gvel = p.vel + sc.grid_off;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
              const int ix = base[0] + i;
              float si[3] = {0.f, 0.f, 0.f}, syi[3] = {0.f, 0.f, 0.f}, szi[3] = {0.f, 0.f, 0.f};
#pragma unroll
              for (int j = 0; j < 3; ++j) {
                const int iy = base[1] + j;
                float sj[3] = {0.f, 0.f, 0.f}, szj[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                  const int iz = base[2] + k;
                  if ((unsigned)ix < (unsigned)n && (unsigned)iy < (unsigned)n && (unsigned)iz < (unsigned)n) {
                    const float4 g = __ldg(&gvel[(size_t)ix + (size_t)n * ((size_t)iy + (size_t)n * (size_t)iz)]);
                    const float wk = w[2][k];
                    sj[0] += wk * g.x;
                    sj[1] += wk * g.y;
                    sj[2] += wk * g.z;
                    const float wdk = wk * d[2][k];
                    szj[0] += wdk * g.x;
                    szj[1] += wdk * g.y;
                    szj[2] += wdk * g.z;
                  }
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
            const float four_inv_dx2 = 4.0f * sc.inv_dx * sc.inv_dx;
#pragma unroll
            for (int i = 0; i < 9; ++i) C[i] = four_inv_dx2 * G[i];
            v[0] = vs[0];
            v[1] = vs[1];
            v[2] = vs[2];
            if (md.rheo == 2) {
              v[0] *= md.vfac;
              v[1] *= md.vfac;
              v[2] *= md.vfac;
#pragma unroll
              for (int i = 0; i < 9; ++i) C[i] *= md.afac;
            }
            float np[3] = {x + sc.dt * v[0], y + sc.dt * v[1], z + sc.dt * v[2]};
            bool fin2 = finitef(np[0]) && finitef(np[1]) && finitef(np[2]) && finitef(v[0]) && finitef(v[1]) &&
                        finitef(v[2]);
#pragma unroll
            for (int i = 0; i < 9; ++i) fin2 = fin2 && finitef(C[i]);
            if (!fin2) {
              atomicOr(status, kFaultNumerical);
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
              bool fin3 = true;
#pragma unroll
              for (int i = 0; i < 9; ++i) fin3 = fin3 && finitef(Fn[i]);
              if (!fin3) {
                atomicOr(status, kFaultNumerical);
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
                svd3<SR>(Fs, svd, stol, sweeps);
                float jp_new = jp;
                if (plasticity_project<SR>(svd, md, jp_new)) {
                  SR Fr[9];
                  sandwich(svd.u, svd.s, svd.v, Fr);
                  bool fin4 = true;
#pragma unroll
                  for (int i = 0; i < 9; ++i) fin4 = fin4 && finitef((float)Fr[i]);
                  if (fin4) {
#pragma unroll
                    for (int i = 0; i < 9; ++i) F[i] = (float)Fr[i];
                    jp = jp_new;
                  } else {
                    atomicOr(status, kFaultNumerical);
                    ok = false;
                  }
                } else {
                  atomicOr(status, kFaultNumerical);
                  ok = false;
                }
                // G2P results are published even when the return mapping
                // faults (the reference's g2p and plasticity are separate
                // dispatches); only the plasticity update is withheld.
                plane(p, PX)[s] = x;
                plane(p, PY)[s] = y;
                plane(p, PZ)[s] = z;
                plane(p, VX)[s] = v[0];
                plane(p, VY)[s] = v[1];
                plane(p, VZ)[s] = v[2];
#pragma unroll
                for (int i = 0; i < 9; ++i) plane(p, C0 + i)[s] = C[i];
#pragma unroll
                for (int i = 0; i < 9; ++i) plane(p, F0 + i)[s] = F[i];
                plane(p, JP)[s] = jp;
              }
            }
          }
        } else {
          // P2G-only: read v, C; validate the whole state (the reference's
          // g2p checks, mpm.wgsl:1247-1255, moved to the first launch of the
          // call so that a non-finite upload latches before anything moves).
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
            atomicOr(status, kFaultNumerical);
            ok = false;
          }
        }
        if constexpr (kScatter) {
          if (ok) {
            if (!kGather || !reuse_svd) {
              SR Fs[9];
#pragma unroll
              for (int i = 0; i < 9; ++i) Fs[i] = (SR)F[i];
              svd3<SR>(Fs, svd, stol, sweeps);
            }
            float B[9];
            p2g_affine<SR>(svd, md, jp, mass, vol, C, sc.dt, sc.inv_dx, B);
            scatter_particle(s_acc, rx, ry, rz, sc, acc, x, y, z, mass, v, B);
          }
        }
        if constexpr (WRITE_KEYS) {
          p.keys_by_id[p.orig[s]] = sc.key_off + tile_key_of(sc, x, y, z);
        }
      }
    }
    if constexpr (kScatter) {
      __syncthreads();
      if (!faulted) {
        const int n = (int)sc.n;
        for (int r = threadIdx.x; r < kRegionNodes; r += blockDim.x) {
          const float m = s_acc[0][r], px = s_acc[1][r], py = s_acc[2][r], pz = s_acc[3][r];
          if (m != 0.f || px != 0.f || py != 0.f || pz != 0.f) {
            const int ix = rx + r % kRegion, iy = ry + (r / kRegion) % kRegion, iz = rz + r / (kRegion * kRegion);
            if ((unsigned)ix < (unsigned)n && (unsigned)iy < (unsigned)n && (unsigned)iz < (unsigned)n) {
              const uint64_t c =
                  sc.grid_off + (uint64_t)ix + (uint64_t)n * ((uint64_t)iy + (uint64_t)n * (uint64_t)iz);
              atomicAdd(&acc[c], make_float4(m, px, py, pz));
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

// grid_update (mpm.wgsl:1013-1058) over the grid pool, clearing the other
// accumulator for the next scatter and counting completed substeps.
__global__ void __launch_bounds__(kCellThreads) k_grid_update(PoolDev p, const uint32_t* __restrict__ block_scene,
                                                              uint64_t total_cells, int acc_in, int count_substep) {
  const uint64_t g = (uint64_t)blockIdx.x * kCellThreads + threadIdx.x;
  if (g >= total_cells) return;
  const float4 a = p.acc[acc_in][g];
  p.acc[acc_in ^ 1][g] = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t sid = block_scene[g / kCellBlock];
  if (sid == 0xffffffffu) return;
  const SceneDev& sc = p.scenes[sid];
  const uint64_t local = g - sc.grid_off;
  const uint32_t n = sc.n;
  if (local >= (uint64_t)n * n * n) return;
  if (count_substep && local == 0) {
    uint32_t* status = p.status + (size_t)sc.status * kStatusWords;
    if (*(volatile uint32_t*)status == 0u) atomicAdd(status + 1, 1u);
  }
  const float m = a.x;
  if (m <= 1.0e-9f || !(m == m)) {
    p.vel[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  float v[3] = {a.y / m, a.z / m, a.w / m};
  v[1] = v[1] + sc.dt * sc.gy;
  const int ix = (int)(local % n), iy = (int)((local / n) % n), iz = (int)(local / ((uint64_t)n * n));
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

// Sort keys of the live slots (tile_keys, mpm_particle_order.wgsl:11-25)
// written at the particle's identity.
__global__ void k_keys(PoolDev p, uint32_t n_slots) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const SceneDev& sc = p.scenes[p.meta[s] >> 8];
  // Particles of a removed scene sort behind every live key.
  p.keys_by_id[p.orig[s]] =
      sc.live ? sc.key_off + tile_key_of(sc, plane(p, PX)[s], plane(p, PY)[s], plane(p, PZ)[s]) : 0xffffffffu;
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
                          const uint32_t* __restrict__ ids, uint32_t n_live) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_live) return;
  const uint32_t id = ids[s];
  const uint32_t old = slot_of[id];
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) dst[(size_t)k * cap + s] = src[(size_t)k * cap + old];
  meta_dst[s] = meta_src[old];
  orig_dst[s] = id;
  slot_of[id] = s;
}

// tile_start[t] = first sorted position whose key is >= t, for t in [0, K].
__global__ void k_tile_start(const uint32_t* __restrict__ sorted_keys, uint32_t n_live, uint32_t K,
                             uint32_t* __restrict__ tile_start) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > K) return;
  uint32_t lo = 0, hi = n_live;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (sorted_keys[mid] < t) lo = mid + 1;
    else hi = mid;
  }
  tile_start[t] = lo;
}

// Work items: every occupied tile, cut into chunks of at most `chunk` slots.
// scene_of_tile is found by a search over the scene key offsets.
__global__ void k_items(const uint32_t* __restrict__ tile_start, uint32_t K, const uint32_t* __restrict__ key_offs,
                        uint32_t n_scenes, const uint32_t* __restrict__ scene_ids, uint32_t chunk,
                        Item* __restrict__ items, uint32_t* __restrict__ n_items) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= K) return;
  const uint32_t a = tile_start[t], b = tile_start[t + 1];
  if (b <= a) return;
  // last scene whose key offset is <= t
  uint32_t lo = 0, hi = n_scenes;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (key_offs[mid] <= t) lo = mid;
    else hi = mid;
  }
  const uint32_t cnt = b - a;
  const uint32_t pieces = (cnt + chunk - 1) / chunk;
  const uint32_t base = atomicAdd(n_items, pieces);
  for (uint32_t i = 0; i < pieces; ++i) {
    Item it;
    it.start = a + i * chunk;
    it.count = min(chunk, cnt - i * chunk);
    it.scene = scene_ids[lo];
    it.tile = t - key_offs[lo];
    items[base + i] = it;
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

template <int MODE, bool KEYS, class SR>
static cudaError_t launch_particles_t(const PoolDev& p, int acc_out, double tol, int sweeps, int reuse, int grid,
                                      cudaStream_t st) {
  k_particles<MODE, KEYS, SR><<<grid, kParticleThreads, 0, st>>>(p, acc_out, tol, sweeps, reuse);
  return cudaGetLastError();
}

cudaError_t launch_particles(int mode, bool write_keys, bool svd_fp64, const PoolDev& p, int acc_out, double tol,
                             int sweeps, int reuse, int grid, cudaStream_t st) {
#define MPM_DISPATCH(M)                                                                            \
  if (mode == M) {                                                                                 \
    if (svd_fp64) {                                                                                \
      return write_keys ? launch_particles_t<M, true, double>(p, acc_out, tol, sweeps, reuse, grid, st)  \
                        : launch_particles_t<M, false, double>(p, acc_out, tol, sweeps, reuse, grid, st); \
    }                                                                                              \
    return write_keys ? launch_particles_t<M, true, float>(p, acc_out, tol, sweeps, reuse, grid, st)     \
                      : launch_particles_t<M, false, float>(p, acc_out, tol, sweeps, reuse, grid, st);    \
  }
  MPM_DISPATCH(kP2G)
  MPM_DISPATCH(kG2P)
  MPM_DISPATCH(kG2P2G)
#undef MPM_DISPATCH
  return cudaErrorInvalidValue;
}

int particle_grid_size(int mode, bool write_keys, bool svd_fp64) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaErrorInvalidValue;
#define MPM_OCC(M, K, T)                                                                                     \
  if (mode == M && write_keys == K && svd_fp64 == (sizeof(T) == 8))                                         \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_particles<M, K, T>, kParticleThreads, 0);
  MPM_OCC(kP2G, false, float) MPM_OCC(kP2G, true, float) MPM_OCC(kP2G, false, double) MPM_OCC(kP2G, true, double)
  MPM_OCC(kG2P, false, float) MPM_OCC(kG2P, true, float) MPM_OCC(kG2P, false, double) MPM_OCC(kG2P, true, double)
  MPM_OCC(kG2P2G, false, float) MPM_OCC(kG2P2G, true, float) MPM_OCC(kG2P2G, false, double)
  MPM_OCC(kG2P2G, true, double)
#undef MPM_OCC
  if (e != cudaSuccess || per_sm < 1) per_sm = 1;
  if (sms < 1) sms = 148;
  return sms * per_sm;
}

cudaError_t launch_grid_update(const PoolDev& p, const uint32_t* block_scene, uint64_t total_cells, int acc_in,
                               int count_substep, cudaStream_t st) {
  const uint64_t blocks = (total_cells + kCellThreads - 1) / kCellThreads;
  if (blocks == 0) return cudaSuccess;
  k_grid_update<<<(unsigned)blocks, kCellThreads, 0, st>>>(p, block_scene, total_cells, acc_in, count_substep);
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
                           uint32_t* orig_dst, uint32_t* slot_of, const uint32_t* ids, uint32_t n_live,
                           cudaStream_t st) {
  if (!n_live) return cudaSuccess;
  k_reorder<<<(n_live + 255) / 256, 256, 0, st>>>(src, dst, cap, meta_src, meta_dst, orig_dst, slot_of, ids, n_live);
  return cudaGetLastError();
}

cudaError_t launch_items(const uint32_t* sorted_keys, uint32_t n_live, uint32_t K, uint32_t* tile_start,
                         const uint32_t* key_offs, uint32_t n_scenes, const uint32_t* scene_ids, uint32_t chunk,
                         Item* items, uint32_t* n_items, cudaStream_t st) {
  cudaMemsetAsync(n_items, 0, sizeof(uint32_t), st);
  k_tile_start<<<(K + 1 + 255) / 256, 256, 0, st>>>(sorted_keys, n_live, K, tile_start);
  if (K > 0)
    k_items<<<(K + 255) / 256, 256, 0, st>>>(tile_start, K, key_offs, n_scenes, scene_ids, chunk, items, n_items);
  return cudaGetLastError();
}

cudaError_t launch_gather_xyz(const PoolDev& p, int first, const uint32_t* slot_of, uint32_t id_base, uint32_t n,
                              float* out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_gather_xyz<<<(n + 255) / 256, 256, 0, st>>>(p, first, slot_of, id_base, n, out);
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
