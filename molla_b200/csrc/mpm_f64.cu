// mpm_f64.cu — the all-FP64 substep on the GPU, for precision studies.
//
// FP64 particle state and FP64 grid, one thread per particle or node, in the
// reference dispatch order (crates/molla-solvers/src/mpm.rs:2476-2551):
// reset, p2g (mpm.wgsl:495-628), grid_update (:1013-1058), g2p (:1242-1353),
// plasticity (:1366-1479), with the reference's two-sided Jacobi SVD
// (:349-468) run in FP64 to a tight tolerance.  Nothing here is tuned: this
// path exists to measure how far the FP32 and FP32 + FP64-SVD modes drift
// from an all-FP64 run of the same step on the same device.
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_f64.cuh"

namespace mpm {

namespace {

constexpr uint32_t kFault = 2u;  // mpm.wgsl:229

__device__ __forceinline__ bool fin(double x) { return isfinite(x); }

__device__ __forceinline__ double det3d(const double* a) {
  return a[0] * (a[4] * a[8] - a[7] * a[5]) - a[3] * (a[1] * a[8] - a[7] * a[2]) + a[6] * (a[1] * a[5] - a[4] * a[2]);
}

// o = u diag(d) v^T, column-major 3x3.
__device__ __forceinline__ void sandwich64(const double* u, const double* d, const double* v, double* o) {
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o[3 * c + r] = u[r] * d[0] * v[c] + u[3 + r] * d[1] * v[3 + c] + u[6 + r] * d[2] * v[6 + c];
}

// Two-sided Jacobi SVD of F (column-major) on A = F^T F, cyclic over
// (0,1), (0,2), (1,2), the reference's rotation formulas and sign fixes, all
// in FP64.  u, v column-major; s may carry one negative sign.
__device__ void svd_ref64(const double* f, double* u, double* s, double* v, double tol, int sweeps) {
  double a[3][3];  // a[col][row]
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) a[c][r] = f[3 * r] * f[3 * c] + f[3 * r + 1] * f[3 * c + 1] + f[3 * r + 2] * f[3 * c + 2];
  for (int i = 0; i < 9; ++i) v[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int sw = 0; sw < sweeps; ++sw) {
    double max_off = 0.0;
    for (int pq = 0; pq < 3; ++pq) {
      const int P = pq == 2 ? 1 : 0, Q = pq == 0 ? 1 : 2, K = 3 - P - Q;
      const double apq = a[Q][P];
      max_off = fmax(max_off, fabs(apq));
      if (fabs(apq) < tol) continue;
      const double app = a[P][P], aqq = a[Q][Q];
      const double theta = (aqq - app) / (2.0 * apq);
      const double t = theta >= 0.0 ? 1.0 / (theta + sqrt(1.0 + theta * theta))
                                    : 1.0 / (theta - sqrt(1.0 + theta * theta));
      const double c = 1.0 / sqrt(1.0 + t * t);
      const double sn = t * c;
      a[P][P] = app - t * apq;
      a[Q][Q] = aqq + t * apq;
      a[Q][P] = 0.0;
      a[P][Q] = 0.0;
      const double akp = a[P][K], akq = a[Q][K];
      a[P][K] = c * akp - sn * akq;
      a[Q][K] = sn * akp + c * akq;
      a[K][P] = a[P][K];
      a[K][Q] = a[Q][K];
      for (int k = 0; k < 3; ++k) {
        const double vkp = v[3 * P + k], vkq = v[3 * Q + k];
        v[3 * P + k] = c * vkp - sn * vkq;
        v[3 * Q + k] = sn * vkp + c * vkq;
      }
    }
    if (max_off < tol) break;
  }
  for (int i = 0; i < 3; ++i) {
    double m[3];
    for (int r = 0; r < 3; ++r) m[r] = f[r] * v[3 * i] + f[3 + r] * v[3 * i + 1] + f[6 + r] * v[3 * i + 2];
    const double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    s[i] = len;
    for (int r = 0; r < 3; ++r) u[3 * i + r] = len > 1.0e-12 ? m[r] / len : (i == r ? 1.0 : 0.0);
  }
  if (det3d(u) < 0.0) {
    int mi = 0;
    if (s[1] < s[mi]) mi = 1;
    if (s[2] < s[mi]) mi = 2;
    for (int r = 0; r < 3; ++r) u[3 * mi + r] = -u[3 * mi + r];
    s[mi] = -s[mi];
  }
  if (det3d(v) < 0.0) {
    int mi = 0;
    if (fabs(s[1]) < fabs(s[mi])) mi = 1;
    if (fabs(s[2]) < fabs(s[mi])) mi = 2;
    for (int r = 0; r < 3; ++r) v[3 * mi + r] = -v[3 * mi + r];
    s[mi] = -s[mi];
  }
}

__device__ __forceinline__ void weights64(double fx, double* w) {
  w[0] = 0.5 * (1.5 - fx) * (1.5 - fx);
  w[1] = 0.75 - (fx - 1.0) * (fx - 1.0);
  w[2] = 0.5 * (fx - 0.5) * (fx - 0.5);
}

__device__ __forceinline__ bool latched(const State64& st) { return *(volatile const uint32_t*)st.status != 0u; }

__global__ void k64_p2g(Scene64 sc, State64 st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= st.n || latched(st)) return;
  const double* pos = st.pos + 3 * i;
  const double xp[3] = {(pos[0] - sc.o[0]) * sc.inv_dx, (pos[1] - sc.o[1]) * sc.inv_dx, (pos[2] - sc.o[2]) * sc.inv_dx};
  for (int a = 0; a < 3; ++a)
    if (!(fabs(xp[a]) < 1.0e9)) return;
  int base[3];
  double fx[3], w[3][3];
  for (int a = 0; a < 3; ++a) {
    const double bf = floor(xp[a] - 0.5);
    base[a] = (int)bf - sc.win[a];
    fx[a] = xp[a] - bf;
    weights64(fx[a], w[a]);
  }
  const double* F = st.F + 9 * i;
  double u[9], s[3], v[9];
  svd_ref64(F, u, s, v, sc.tol, sc.sweeps);
  const Mat64 md = sc.mat[st.mat[i] < (uint32_t)sc.n_mat ? st.mat[i] : 0];
  double h = 1.0;
  if (md.rheo == 1) h = exp(fmin(fmax(-md.hardening * st.jp[i], -3.0), 3.0));
  else if (md.rheo == 0) h = exp(fmin(fmax(st.jp[i], -3.0), 3.0));
  double scl[3];
  for (int k = 0; k < 3; ++k) scl[k] = fmin(fmax(s[k], 0.1), 10.0);
  const double J = scl[0] * scl[1] * scl[2];
  const double cofd[3] = {scl[1] * scl[2], scl[0] * scl[2], scl[0] * scl[1]};
  double Fc[9], cof[9], P[9], S[9];
  sandwich64(u, scl, v, Fc);
  sandwich64(u, cofd, v, cof);
  const double k1 = 2.0 * md.mu * h, k2 = md.lam * h * (J - 1.0), k3 = -sc.dt * st.vol[i];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      const double Rcr = u[r] * v[c] + u[3 + r] * v[3 + c] + u[6 + r] * v[6 + c];
      P[3 * c + r] = k3 * (k1 * (Fc[3 * c + r] - Rcr) + k2 * cof[3 * c + r]);
    }
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) S[3 * c + r] = P[r] * Fc[c] + P[3 + r] * Fc[3 + c] + P[6 + r] * Fc[6 + c];
  const double* C = st.C + 9 * i;
  const double* vel = st.vel + 3 * i;
  const double m = st.mass[i];
  const double k4 = 4.0 * sc.inv_dx * sc.inv_dx;
  for (int q = 0; q < 27; ++q) {
    const int a = q / 9, b = (q / 3) % 3, c = q % 3;
    const int ix = base[0] + a, iy = base[1] + b, iz = base[2] + c;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= sc.n || iy >= sc.n || iz >= sc.n) continue;
    const double wt = w[0][a] * w[1][b] * w[2][c];
    const double d[3] = {((double)a - fx[0]) * sc.dx, ((double)b - fx[1]) * sc.dx, ((double)c - fx[2]) * sc.dx};
    const size_t cell = (size_t)ix + (size_t)sc.n * ((size_t)iy + (size_t)sc.n * (size_t)iz);
    const double wm = wt * m;
    for (int r = 0; r < 3; ++r) {
      const double aff = C[r] * d[0] + C[3 + r] * d[1] + C[6 + r] * d[2];
      const double sf = S[r] * d[0] + S[3 + r] * d[1] + S[6 + r] * d[2];
      atomicAdd(&st.gmom[3 * cell + r], wm * (vel[r] + aff) + wt * (sf * k4));
    }
    atomicAdd(&st.gmass[cell], wm);
  }
}

__global__ void k64_grid(Scene64 sc, State64 st) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n3 = (size_t)sc.n * sc.n * sc.n;
  if (c >= n3 || latched(st)) return;
  if (c == 0) atomicAdd(st.status + 1, 1u);
  const double m = st.gmass[c];
  double* v = st.gvel + 3 * c;
  if (m <= 1.0e-9 || !(m == m)) {
    v[0] = v[1] = v[2] = 0.0;
    return;
  }
  double vv[3] = {st.gmom[3 * c] / m, st.gmom[3 * c + 1] / m, st.gmom[3 * c + 2] / m};
  vv[1] = vv[1] + sc.dt * sc.gy;
  const int n = sc.n, pad = sc.pad;
  const int ix = (int)(c % n), iy = (int)((c / n) % n), iz = (int)(c / ((size_t)n * n));
  const double f = sc.friction;
  if (sc.sticky) {
    if (ix < pad || ix >= n - pad || iy < pad || iy >= n - pad || iz < pad || iz >= n - pad) vv[0] = vv[1] = vv[2] = 0.0;
  } else {
    if (ix < pad) { vv[0] = fmax(vv[0], 0.0); vv[1] *= f; vv[2] *= f; }
    if (ix >= n - pad) { vv[0] = fmin(vv[0], 0.0); vv[1] *= f; vv[2] *= f; }
    if (iy < pad) { vv[1] = fmax(vv[1], 0.0); vv[0] *= f; vv[2] *= f; }
    if (iy >= n - pad) { vv[1] = fmin(vv[1], 0.0); vv[0] *= f; vv[2] *= f; }
    if (iz < pad) { vv[2] = fmax(vv[2], 0.0); vv[0] *= f; vv[1] *= f; }
    if (iz >= n - pad) { vv[2] = fmin(vv[2], 0.0); vv[0] *= f; vv[1] *= f; }
  }
  v[0] = vv[0];
  v[1] = vv[1];
  v[2] = vv[2];
}

__global__ void k64_g2p(Scene64 sc, State64 st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= st.n || latched(st)) return;
  double* pos = st.pos + 3 * i;
  double* vel = st.vel + 3 * i;
  double* C = st.C + 9 * i;
  double* F = st.F + 9 * i;
  bool ok = fin(st.jp[i]);
  for (int k = 0; k < 3; ++k) ok = ok && fin(pos[k]) && fin(vel[k]);
  for (int k = 0; k < 9; ++k) ok = ok && fin(C[k]) && fin(F[k]);
  double xp[3];
  for (int a = 0; a < 3; ++a) {
    xp[a] = (pos[a] - sc.o[a]) * sc.inv_dx;
    ok = ok && fin(xp[a]);
  }
  if (!ok) {
    atomicOr(st.status, kFault);
    return;
  }
  int base[3];
  double fx[3], w[3][3];
  for (int a = 0; a < 3; ++a) {
    const double bf = floor(xp[a] - 0.5);
    base[a] = (int)bf - sc.win[a];
    fx[a] = xp[a] - bf;
    weights64(fx[a], w[a]);
  }
  double vn[3] = {0.0, 0.0, 0.0}, Cn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 27; ++q) {
    const int a = q / 9, b = (q / 3) % 3, c = q % 3;
    const int ix = base[0] + a, iy = base[1] + b, iz = base[2] + c;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= sc.n || iy >= sc.n || iz >= sc.n) continue;
    const double wt = w[0][a] * w[1][b] * w[2][c];
    const double* gv = st.gvel + 3 * ((size_t)ix + (size_t)sc.n * ((size_t)iy + (size_t)sc.n * (size_t)iz));
    const double d[3] = {((double)a - fx[0]) * sc.dx, ((double)b - fx[1]) * sc.dx, ((double)c - fx[2]) * sc.dx};
    const double scale = 4.0 * wt * sc.inv_dx * sc.inv_dx;
    for (int r = 0; r < 3; ++r) vn[r] = vn[r] + wt * gv[r];
    for (int col = 0; col < 3; ++col)
      for (int row = 0; row < 3; ++row) Cn[3 * col + row] = Cn[3 * col + row] + scale * gv[row] * d[col];
  }
  const Mat64 md = sc.mat[st.mat[i] < (uint32_t)sc.n_mat ? st.mat[i] : 0];
  if (md.rheo == 2) {
    const double vd = exp(-fmax(md.vdamp, 0.0) * sc.dt), ad = exp(-fmax(md.adamp, 0.0) * sc.dt);
    for (int r = 0; r < 3; ++r) vn[r] *= vd;
    for (int k = 0; k < 9; ++k) Cn[k] *= ad;
  }
  double np[3];
  bool ok2 = true;
  for (int a = 0; a < 3; ++a) {
    np[a] = pos[a] + sc.dt * vn[a];
    ok2 = ok2 && fin(np[a]) && fin(vn[a]);
  }
  for (int k = 0; k < 9; ++k) ok2 = ok2 && fin(Cn[k]);
  if (!ok2) {
    atomicOr(st.status, kFault);
    return;
  }
  for (int a = 0; a < 3; ++a) {
    if (np[a] < sc.lo[a] || np[a] > sc.hi[a]) vn[a] = 0.0;
    np[a] = fmin(fmax(np[a], sc.lo[a]), sc.hi[a]);
  }
  double Fn[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += ((r == k ? 1.0 : 0.0) + sc.dt * Cn[3 * k + r]) * F[3 * c + k];
      Fn[3 * c + r] = acc;
    }
  for (int k = 0; k < 9; ++k)
    if (!fin(Fn[k])) {
      atomicOr(st.status, kFault);
      return;
    }
  for (int a = 0; a < 3; ++a) {
    pos[a] = np[a];
    vel[a] = vn[a];
  }
  for (int k = 0; k < 9; ++k) {
    C[k] = Cn[k];
    F[k] = Fn[k];
  }
}

__global__ void k64_plasticity(Scene64 sc, State64 st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= st.n || latched(st)) return;
  double* F = st.F + 9 * i;
  double jp = st.jp[i];
  bool ok = fin(jp);
  for (int k = 0; k < 9; ++k) ok = ok && fin(F[k]);
  double u[9], s[3], v[9];
  if (ok) svd_ref64(F, u, s, v, sc.tol, sc.sweeps);
  for (int k = 0; k < 3 && ok; ++k) ok = fin(s[k]);
  for (int k = 0; k < 9 && ok; ++k) ok = fin(u[k]) && fin(v[k]);
  if (!ok) {
    atomicOr(st.status, kFault);
    return;
  }
  const Mat64 md = sc.mat[st.mat[i] < (uint32_t)sc.n_mat ? st.mat[i] : 0];
  double ns[3] = {s[0], s[1], s[2]}, dq = 0.0, jp_new = 0.0;
  bool replace = false;
  if (md.rheo == 1) {
    for (int a = 0; a < 3; ++a) ns[a] = fmin(fmax(s[a], 1.0 - md.theta_c), 1.0 + md.theta_s);
    const double det_old = fmax(s[0] * s[1] * s[2], 1.0e-6), det_new = fmax(ns[0] * ns[1] * ns[2], 1.0e-6);
    replace = true;
    jp_new = jp + (log(det_old) - log(det_new));
    if (!fin(jp_new)) {
      atomicOr(st.status, kFault);
      return;
    }
    jp_new = fmin(fmax(jp_new, -5.0), 5.0);
  } else if (md.rheo == 2) {
    replace = true;
  } else {
    double eps[3];
    for (int a = 0; a < 3; ++a) eps[a] = log(fmax(s[a], 1.0e-6));
    const double tr = eps[0] + eps[1] + eps[2], mean = tr / 3.0;
    const double dev[3] = {eps[0] - mean, eps[1] - mean, eps[2] - mean};
    const double dn = sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
    if (tr > 0.0) {
      ns[0] = ns[1] = ns[2] = 1.0;
      dq = sqrt(eps[0] * eps[0] + eps[1] * eps[1] + eps[2] * eps[2]);
    } else if (dn != 0.0) {
      const double fy = dn + md.kappa * tr * md.dp_alpha;
      if (fy > 0.0) {
        const double rc = fmax(0.0, -md.dp_alpha * md.kappa * tr);
        for (int a = 0; a < 3; ++a) ns[a] = exp(dev[a] * (rc / dn) + mean);
        dq = fy;
      }
    }
  }
  if (!fin(ns[0]) || !fin(ns[1]) || !fin(ns[2]) || !fin(dq) || !fin(jp + dq)) {
    atomicOr(st.status, kFault);
    return;
  }
  for (int a = 0; a < 3; ++a) ns[a] = fmin(fmax(ns[a], 0.05), 20.0);
  double Fr[9];
  sandwich64(u, ns, v, Fr);
  for (int k = 0; k < 9; ++k)
    if (!fin(Fr[k])) {
      atomicOr(st.status, kFault);
      return;
    }
  for (int k = 0; k < 9; ++k) F[k] = Fr[k];
  st.jp[i] = replace ? jp_new : fmin(fmax(jp + dq, 0.0), 5.0);
}

// Grid totals of the last P2G: out[0] mass, out[1..3] momentum.
__global__ void k64_totals(Scene64 sc, State64 st, double* out) {
  const size_t n3 = (size_t)sc.n * sc.n * sc.n;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += (size_t)gridDim.x * blockDim.x) {
    acc[0] += st.gmass[c];
    acc[1] += st.gmom[3 * c];
    acc[2] += st.gmom[3 * c + 1];
    acc[3] += st.gmom[3 * c + 2];
  }
  for (int k = 0; k < 4; ++k) {
    double x = acc[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[k], x);
  }
}

}  // namespace

cudaError_t launch_step64(const Scene64& sc, const State64& st, uint32_t substeps, cudaStream_t s) {
  const size_t n3 = (size_t)sc.n * sc.n * sc.n;
  const unsigned pb = (unsigned)((st.n + 127) / 128), gb = (unsigned)((n3 + 255) / 256);
  for (uint32_t k = 0; k < substeps; ++k) {
    cudaMemsetAsync(st.gmass, 0, n3 * sizeof(double), s);
    cudaMemsetAsync(st.gmom, 0, 3 * n3 * sizeof(double), s);
    if (st.n) k64_p2g<<<pb, 128, 0, s>>>(sc, st);
    k64_grid<<<gb, 256, 0, s>>>(sc, st);
    if (st.n) {
      k64_g2p<<<pb, 128, 0, s>>>(sc, st);
      k64_plasticity<<<pb, 128, 0, s>>>(sc, st);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_totals64(const Scene64& sc, const State64& st, double* out4, cudaStream_t s) {
  cudaMemsetAsync(out4, 0, 4 * sizeof(double), s);
  k64_totals<<<592, 256, 0, s>>>(sc, st, out4);
  return cudaGetLastError();
}

}  // namespace mpm
