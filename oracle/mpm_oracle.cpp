// mpm_oracle.cpp — CPU oracle for the explicit MLS-MPM substep.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA product
// path is compared against; it is never linked into the product library and
// nothing in molla_b200/ calls it. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load the shared object built from it.
//
// It restates, in plain C++17, the arithmetic of molla's WGSL MPM step
// (crates/molla-solvers/shaders/mpm.wgsl) and of its particle-ordering pass
// (crates/molla-solvers/shaders/mpm_particle_order.wgsl plus the stable radix
// sort contract of crates/molla-compute-primitives/src/radix_sort.rs:20-30).
// Every function cites the reference lines it follows. The step is templated
// on the state precision and, separately, on the SVD precision, which gives
// the three oracle forms used by the tests:
//   * <float,  float>  — FP32, the reference's own precision;
//   * <float,  double> — FP32 state with an FP64 SVD/polar decomposition;
//   * <double, double> — FP64 everywhere (the accuracy reference).
// Grid accumulation runs in particle-index order (the WGSL accumulation order
// is unspecified because it uses atomics). An OpenMP form of the FP32 step is
// the timed CPU baseline; it accumulates with atomics and is not used for
// bit-level comparisons.
//
// Parity pins: the sort key/permutation is pinned bit-exactly by the
// reference's own host formula in crates/molla-solvers/src/mpm_particle_order_tests.rs:33-42
// and its stable-sort reference (crates/molla-compute-primitives/tests/radix_sort_gpu.rs:299-305).
// The floating-point step is pinned by the reference's known-answer tests
// (material oracles, G2P affine exactness, free fall, mass sums); bit-level
// parity of the float step is not pinnable because the reference's rounding
// is decided by naga/wgpu and the vendor driver.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// Column-major 3x3 matrix, m[col][row], the WGSL mat3x3 convention.
template <class R> struct M3 {
  R m[3][3];
};

template <class R> static inline M3<R> zero3() {
  M3<R> a;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) a.m[c][r] = R(0);
  return a;
}
template <class R> static inline M3<R> ident3() {
  M3<R> a = zero3<R>();
  a.m[0][0] = a.m[1][1] = a.m[2][2] = R(1);
  return a;
}
// (A*B)[c][r] = sum_k A[k][r] * B[c][k]
template <class R> static inline M3<R> mul(const M3<R>& a, const M3<R>& b) {
  M3<R> o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      R s = a.m[0][r] * b.m[c][0];
      s = s + a.m[1][r] * b.m[c][1];
      s = s + a.m[2][r] * b.m[c][2];
      o.m[c][r] = s;
    }
  return o;
}
template <class R> static inline M3<R> transpose(const M3<R>& a) {
  M3<R> o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o.m[c][r] = a.m[r][c];
  return o;
}
template <class R> static inline void mulv(const M3<R>& a, const R v[3], R out[3]) {
  for (int r = 0; r < 3; ++r) {
    R s = a.m[0][r] * v[0];
    s = s + a.m[1][r] * v[1];
    s = s + a.m[2][r] * v[2];
    out[r] = s;
  }
}
template <class R> static inline M3<R> diag_sandwich(const M3<R>& u, const R d[3], const M3<R>& v) {
  // u * diag(d) * transpose(v), evaluated left to right as in mpm.wgsl:577-587.
  M3<R> dm = zero3<R>();
  dm.m[0][0] = d[0];
  dm.m[1][1] = d[1];
  dm.m[2][2] = d[2];
  return mul(mul(u, dm), transpose(v));
}
template <class R> static inline R det3(const M3<R>& a) {
  // WGSL determinant(): expansion along the first column.
  const R a00 = a.m[0][0], a01 = a.m[1][0], a02 = a.m[2][0];
  const R a10 = a.m[0][1], a11 = a.m[1][1], a12 = a.m[2][1];
  const R a20 = a.m[0][2], a21 = a.m[1][2], a22 = a.m[2][2];
  return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
}
template <class R> static inline R length3(const R v[3]) {
  return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}
template <class R> static inline R clampr(R x, R lo, R hi) { return std::min(std::max(x, lo), hi); }

template <class R> static inline bool finite_bits(R x) { return std::isfinite(x); }
template <class R> static inline bool finite_m(const M3<R>& a) {
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r)
      if (!std::isfinite(a.m[c][r])) return false;
  return true;
}

template <class R> struct Svd {
  M3<R> u;
  R s[3];
  M3<R> v;
};

// Two-sided Jacobi SVD: eigen-decompose A = F^T F by cyclic Jacobi rotations,
// sigma_i = |F v_i|, u_i = F v_i / sigma_i, then sign fixes so that det(U) and
// det(V) are +1.  Follows crates/molla-solvers/shaders/mpm.wgsl:365-468
// (max 16 sweeps, absolute off-diagonal tolerance 1e-7 in the reference).
template <class R> Svd<R> svd3_jacobi(const M3<R>& f, R tol, int max_sweeps) {
  M3<R> v = ident3<R>();
  M3<R> a = mul(transpose(f), f);
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    R max_off = R(0);
    for (int p = 0; p < 3; ++p) {
      for (int q = p + 1; q < 3; ++q) {
        const R apq = a.m[q][p];
        if (std::fabs(apq) > max_off) max_off = std::fabs(apq);
        if (std::fabs(apq) < tol) continue;
        const R app = a.m[p][p];
        const R aqq = a.m[q][q];
        const R theta = (aqq - app) / (R(2) * apq);
        R t;
        if (theta >= R(0)) {
          t = R(1) / (theta + std::sqrt(R(1) + theta * theta));
        } else {
          t = R(1) / (theta - std::sqrt(R(1) + theta * theta));
        }
        const R c = R(1) / std::sqrt(R(1) + t * t);
        const R s = t * c;
        a.m[p][p] = app - t * apq;
        a.m[q][q] = aqq + t * apq;
        a.m[q][p] = R(0);
        a.m[p][q] = R(0);
        for (int k = 0; k < 3; ++k) {
          if (k != p && k != q) {
            const R akp = a.m[p][k];
            const R akq = a.m[q][k];
            a.m[p][k] = c * akp - s * akq;
            a.m[q][k] = s * akp + c * akq;
            a.m[k][p] = a.m[p][k];
            a.m[k][q] = a.m[q][k];
          }
        }
        for (int k = 0; k < 3; ++k) {
          const R vkp = v.m[p][k];
          const R vkq = v.m[q][k];
          v.m[p][k] = c * vkp - s * vkq;
          v.m[q][k] = s * vkp + c * vkq;
        }
      }
    }
    if (max_off < tol) break;
  }
  Svd<R> out;
  out.u = zero3<R>();
  for (int i = 0; i < 3; ++i) {
    const R vi[3] = {v.m[i][0], v.m[i][1], v.m[i][2]};
    R mvi[3];
    mulv(f, vi, mvi);
    const R s = length3(mvi);
    out.s[i] = s;
    if (s > R(1.0e-12)) {
      out.u.m[i][0] = mvi[0] / s;
      out.u.m[i][1] = mvi[1] / s;
      out.u.m[i][2] = mvi[2] / s;
    } else {
      out.u.m[i][0] = i == 0 ? R(1) : R(0);
      out.u.m[i][1] = i == 1 ? R(1) : R(0);
      out.u.m[i][2] = i == 2 ? R(1) : R(0);
    }
  }
  if (det3(out.u) < R(0)) {
    int mi = 0;
    if (out.s[1] < out.s[mi]) mi = 1;
    if (out.s[2] < out.s[mi]) mi = 2;
    for (int r = 0; r < 3; ++r) out.u.m[mi][r] = -out.u.m[mi][r];
    out.s[mi] = -out.s[mi];
  }
  if (det3(v) < R(0)) {
    int mi = 0;
    if (std::fabs(out.s[1]) < std::fabs(out.s[mi])) mi = 1;
    if (std::fabs(out.s[2]) < std::fabs(out.s[mi])) mi = 2;
    for (int r = 0; r < 3; ++r) v.m[mi][r] = -v.m[mi][r];
    out.s[mi] = -out.s[mi];
  }
  out.v = v;
  return out;
}

}  // namespace orc

extern "C" {

// One row of the material table (crates/molla-solvers/src/mpm.rs:662-686,
// WGSL MpmMaterialRow mpm.wgsl:134-146): rheology 0 sand, 1 snow, 2 viscous.
// youngs/poisson > 0 override the scene-wide values for this row; that
// per-row modulus is an extension (the reference has global E and nu only,
// crates/molla-solvers/shaders/mpm.wgsl:98-99) and is 0 in reference mode.
typedef struct orc_material {
  uint32_t rheology;
  float dp_alpha;
  float theta_c;
  float theta_s;
  float hardening;
  float velocity_damping;
  float affine_damping;
  float youngs;
  float poisson;
} orc_material;

// Per-substep constants (WGSL Uniforms, mpm.wgsl:82-121; packing
// crates/molla-solvers/src/mpm.rs:2355-2404).  boundary_pad is 2 in the
// reference (mpm.wgsl:1049, :1327); sticky != 0 selects the no-slip
// extension in which every velocity component in the pad layer is zeroed.
typedef struct orc_scene {
  uint32_t grid_size;
  float cell_size;
  float inv_cell_size;  // f32 1/cell_size computed on the host, as mpm.rs:2389
  float origin[3];
  int32_t window[3];
  float dt;
  float gravity_y;
  float youngs;
  float poisson;
  float boundary_friction;
  uint32_t boundary_pad;
  uint32_t sticky;
  uint32_t n_materials;
  orc_material materials[8];
  double svd_tol;        // 1e-7 in the reference
  uint32_t svd_sweeps;   // 16 in the reference
  uint32_t jacobi_iters; // MpmTimeStep::Implicit sweeps per substep (0: explicit)
  uint32_t n_rigid;      // rigid spheres (set_rigid_spheres, mpm.rs:1521-1565)
  float rigid[8][7];     // center xyz, radius, velocity xyz
  double wrench[8][6];   // out: force xyz, torque xyz of the last substep
} orc_scene;

}  // extern "C"

namespace orc {

enum : uint32_t { FAULT_NUMERICAL = 2u };

template <class R> struct Params {
  int n;
  R dx, inv_dx, ox, oy, oz;
  int wx, wy, wz;
  R dt, gy, friction;
  int pad;
  bool sticky;
  R youngs, poisson;
};

template <class R> static Params<R> params_of(const orc_scene& s) {
  Params<R> p;
  p.n = (int)s.grid_size;
  p.dx = (R)s.cell_size;
  p.inv_dx = (R)s.inv_cell_size;
  p.ox = (R)s.origin[0];
  p.oy = (R)s.origin[1];
  p.oz = (R)s.origin[2];
  p.wx = s.window[0];
  p.wy = s.window[1];
  p.wz = s.window[2];
  p.dt = (R)s.dt;
  p.gy = (R)s.gravity_y;
  p.friction = (R)s.boundary_friction;
  p.pad = s.boundary_pad ? (int)s.boundary_pad : 2;
  p.sticky = s.sticky != 0;
  p.youngs = (R)s.youngs;
  p.poisson = (R)s.poisson;
  return p;
}

// Quadratic B-spline weights, mpm.wgsl:285-294.
template <class R> static inline void quad_weights(R fx, R w[3]) {
  w[0] = R(0.5) * (R(1.5) - fx) * (R(1.5) - fx);
  w[1] = R(0.75) - (fx - R(1)) * (fx - R(1));
  w[2] = R(0.5) * (fx - R(0.5)) * (fx - R(0.5));
}

template <class R> struct MatConst {
  int rheo;
  R mu, lam, dp_alpha, theta_c, theta_s, hardening, vdamp, adamp;
};

template <class R> static MatConst<R> mat_const(const orc_scene& s, uint32_t id, const Params<R>& p) {
  const orc_material& m = s.materials[id < s.n_materials ? id : 0];
  MatConst<R> c;
  // u32(mrow.p0.x + 0.5) in mpm.wgsl:556-557 is the integer rheology id.
  c.rheo = (int)m.rheology;
  const R e = m.youngs > 0.f ? (R)m.youngs : p.youngs;
  const R nu = m.youngs > 0.f ? (R)m.poisson : p.poisson;
  // mpm.wgsl:550-551
  c.mu = e / (R(2) * (R(1) + nu));
  c.lam = e * nu / ((R(1) + nu) * (R(1) - R(2) * nu));
  c.dp_alpha = (R)m.dp_alpha;
  c.theta_c = (R)m.theta_c;
  c.theta_s = (R)m.theta_s;
  c.hardening = (R)m.hardening;
  c.vdamp = (R)m.velocity_damping;
  c.adamp = (R)m.affine_damping;
  return c;
}

template <class R> struct State {
  int n;
  R* pos;   // 3n
  R* vel;   // 3n
  R* C;     // 9n, column-major per particle
  R* F;     // 9n
  R* mass;  // n
  R* vol;   // n
  R* jp;    // n
  const uint32_t* mat;
};

template <class R> static inline M3<R> load_m(const R* a) {
  M3<R> m;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) m.m[c][r] = a[3 * c + r];
  return m;
}
template <class R> static inline void store_m(R* a, const M3<R>& m) {
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) a[3 * c + r] = m.m[c][r];
}

// Convert between precisions (used for the FP64-SVD form of the FP32 step).
template <class D, class S> static inline M3<D> cvt(const M3<S>& a) {
  M3<D> o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o.m[c][r] = (D)a.m[c][r];
  return o;
}
template <class D, class S> static inline Svd<D> cvt_svd(const Svd<S>& a) {
  Svd<D> o;
  o.u = cvt<D>(a.u);
  o.v = cvt<D>(a.v);
  for (int i = 0; i < 3; ++i) o.s[i] = (D)a.s[i];
  return o;
}

template <class R, class SR> static inline Svd<R> svd_in(const M3<R>& f, const orc_scene& sc) {
  const int sweeps = sc.svd_sweeps ? (int)sc.svd_sweeps : 16;
  const SR tol = sc.svd_tol > 0 ? (SR)sc.svd_tol : (SR)1.0e-7;
  return cvt_svd<R>(svd3_jacobi<SR>(cvt<SR>(f), tol, sweeps));
}

// Grid accumulators for one substep.
template <class R> struct Grid {
  int n;
  std::vector<R> mass, mom;  // n^3, 3 n^3
  std::vector<R> vel;        // 3 n^3 (post grid_update)
  std::vector<uint8_t> rigid;  // n^3: node stamped by a rigid sphere this substep
};

// The P2G body (mpm.wgsl:495-628 and :734-893): per-particle fixed-corotated
// stress from the clamped SVD, then the 27-node APIC scatter.  Calls `add`
// with (cell index, dm, mom[3]) for every in-bounds node.
template <class R, class SR, class Add>
static void p2g_particle(const orc_scene& sc, const Params<R>& p, const State<R>& st, int pid, Add&& add) {
  const R pos[3] = {st.pos[3 * pid], st.pos[3 * pid + 1], st.pos[3 * pid + 2]};
  const R vel[3] = {st.vel[3 * pid], st.vel[3 * pid + 1], st.vel[3 * pid + 2]};
  const R mass = st.mass[pid];
  const R vol = st.vol[pid];
  const M3<R> F = load_m(st.F + 9 * pid);
  const M3<R> C = load_m(st.C + 9 * pid);
  const R o[3] = {p.ox, p.oy, p.oz};
  const int win[3] = {p.wx, p.wy, p.wz};
  R xp[3], bf[3], fx[3], w[3][3];
  int base[3];
  for (int a = 0; a < 3; ++a) xp[a] = (pos[a] - o[a]) * p.inv_dx;
  // Non-finite or far out-of-grid positions deposit nothing here; the g2p
  // pass of the same substep latches the fault for non-finite state.
  for (int a = 0; a < 3; ++a)
    if (!(std::fabs(xp[a]) < R(1.0e9))) return;
  for (int a = 0; a < 3; ++a) {
    bf[a] = std::floor(xp[a] - R(0.5));
    base[a] = (int)bf[a] - win[a];
    fx[a] = xp[a] - bf[a];
    quad_weights(fx[a], w[a]);
  }
  const MatConst<R> mc = mat_const<R>(sc, st.mat[pid], p);
  R h = R(1);
  if (mc.rheo == 1) {
    h = std::exp(clampr(-mc.hardening * st.jp[pid], R(-3), R(3)));
  } else if (mc.rheo == 0) {
    h = std::exp(clampr(st.jp[pid], R(-3), R(3)));
  }
  M3<R> stress;
  if constexpr (sizeof(SR) > sizeof(R)) {
    // FP32 state with the FP64 SVD: the same stress in the principal frame,
    // S = -dt vol U diag(tau) U^T with tau_i = 2 mu h (sc_i - 1) sc_i +
    // lam h (J - 1) J, evaluated in FP64 and rounded once (the product's
    // FP64-SVD mode; identical to the PK1 form below in exact arithmetic).
    const int sweeps = sc.svd_sweeps ? (int)sc.svd_sweeps : 16;
    const Svd<SR> sv = svd3_jacobi<SR>(cvt<SR>(F), sc.svd_tol > 0 ? (SR)sc.svd_tol : (SR)1.0e-7, sweeps);
    SR scd[3];
    for (int i = 0; i < 3; ++i) scd[i] = clampr(sv.s[i], SR(0.1), SR(10));
    const SR J = scd[0] * scd[1] * scd[2];
    SR tau[3];
    for (int i = 0; i < 3; ++i)
      tau[i] = SR(2) * SR(mc.mu) * SR(h) * (scd[i] - SR(1)) * scd[i] + SR(mc.lam) * SR(h) * (J - SR(1)) * J;
    const SR k = -SR(p.dt) * SR(vol);
    M3<SR> sd;
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r)
        sd.m[c][r] = k * (sv.u.m[0][r] * tau[0] * sv.u.m[0][c] + sv.u.m[1][r] * tau[1] * sv.u.m[1][c] +
                          sv.u.m[2][r] * tau[2] * sv.u.m[2][c]);
    stress = cvt<R>(sd);
  } else {
  Svd<R> svd = svd_in<R, SR>(F, sc);
  R sc3[3];
  for (int i = 0; i < 3; ++i) sc3[i] = clampr(svd.s[i], R(0.1), R(10));
  const M3<R> Rm = mul(svd.u, transpose(svd.v));
  const R J = sc3[0] * sc3[1] * sc3[2];
  const R mu_h = mc.mu * h;
  const R lam_h = mc.lam * h;
  const M3<R> Fc = diag_sandwich(svd.u, sc3, svd.v);
  const R cofd[3] = {sc3[1] * sc3[2], sc3[0] * sc3[2], sc3[0] * sc3[1]};
  const M3<R> cof = diag_sandwich(svd.u, cofd, svd.v);
  M3<R> pk1;
  const R k1 = R(2) * mu_h;
  const R k2 = lam_h * (J - R(1));
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) pk1.m[c][r] = k1 * (Fc.m[c][r] - Rm.m[c][r]) + k2 * cof.m[c][r];
  M3<R> spk;
  const R k3 = -p.dt * vol;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) spk.m[c][r] = k3 * pk1.m[c][r];
  stress = mul(spk, transpose(Fc));
  }
  const R dx = p.dx;
  const R inv_dx2 = p.inv_dx * p.inv_dx;
  const R four_inv_dx2 = R(4) * inv_dx2;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        const R wgt = w[0][i] * w[1][j] * w[2][k];
        const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
        if (ix < 0 || iy < 0 || iz < 0 || ix >= p.n || iy >= p.n || iz >= p.n) continue;
        const R d[3] = {((R)i - fx[0]) * dx, ((R)j - fx[1]) * dx, ((R)k - fx[2]) * dx};
        R aff[3], sf[3];
        mulv(C, d, aff);
        mulv(stress, d, sf);
        R mom[3];
        const R wm = wgt * mass;
        for (int a = 0; a < 3; ++a) mom[a] = wm * (vel[a] + aff[a]) + wgt * (sf[a] * four_inv_dx2);
        add((size_t)ix + (size_t)p.n * ((size_t)iy + (size_t)p.n * (size_t)iz), wm, mom);
      }
}

// grid_update, mpm.wgsl:1013-1058 (dense grid, no rigid mask).
template <class R> static void grid_update(const Params<R>& p, Grid<R>& g, int nthreads) {
  const int n = p.n;
#pragma omp parallel for num_threads(nthreads > 1 ? nthreads : 1) schedule(static) if (nthreads > 1)
  for (int iz = 0; iz < n; ++iz)
    for (int iy = 0; iy < n; ++iy)
      for (int ix = 0; ix < n; ++ix) {
        const size_t c = (size_t)ix + (size_t)n * ((size_t)iy + (size_t)n * (size_t)iz);
        const R m = g.mass[c];
        R* v = &g.vel[3 * c];
        if (m <= R(1.0e-9) || !(m == m)) {
          v[0] = v[1] = v[2] = R(0);
          continue;
        }
        v[0] = g.mom[3 * c] / m;
        v[1] = g.mom[3 * c + 1] / m;
        v[2] = g.mom[3 * c + 2] / m;
        if (!g.rigid.empty() && g.rigid[c]) continue;  // rigid-imprinted: no gravity, no walls
        v[1] = v[1] + p.dt * p.gy;
        const int pad = p.pad;
        const R f = p.friction;
        if (p.sticky) {
          // Extension: no-slip walls, every component zero in the pad layer.
          if (ix < pad || ix >= n - pad || iy < pad || iy >= n - pad || iz < pad || iz >= n - pad)
            v[0] = v[1] = v[2] = R(0);
          continue;
        }
        if (ix < pad) { v[0] = std::max(v[0], R(0)); v[1] = v[1] * f; v[2] = v[2] * f; }
        if (ix >= n - pad) { v[0] = std::min(v[0], R(0)); v[1] = v[1] * f; v[2] = v[2] * f; }
        if (iy < pad) { v[1] = std::max(v[1], R(0)); v[0] = v[0] * f; v[2] = v[2] * f; }
        if (iy >= n - pad) { v[1] = std::min(v[1], R(0)); v[0] = v[0] * f; v[2] = v[2] * f; }
        if (iz < pad) { v[2] = std::max(v[2], R(0)); v[0] = v[0] * f; v[1] = v[1] * f; }
        if (iz >= n - pad) { v[2] = std::min(v[2], R(0)); v[0] = v[0] * f; v[1] = v[1] * f; }
      }
}

// rigid_imprint (mpm.wgsl:939-1003) for legacy spheres: a node inside the
// first sphere that contains it takes the sphere velocity with the heavy
// mass 1e6; its sand mass and momentum give the reaction -(m v - p) / dt
// (dt floored at 1e-6) and its torque about the center.
template <class R> static void rigid_imprint(orc_scene& sc, const Params<R>& p, Grid<R>& g) {
  const int n = p.n;
  const R o[3] = {p.ox, p.oy, p.oz};
  const int win[3] = {p.wx, p.wy, p.wz};
  for (int iz = 0; iz < n; ++iz)
    for (int iy = 0; iy < n; ++iy)
      for (int ix = 0; ix < n; ++ix) {
        const size_t c = (size_t)ix + (size_t)n * ((size_t)iy + (size_t)n * (size_t)iz);
        const int idx[3] = {ix, iy, iz};
        R node[3];
        for (int a = 0; a < 3; ++a) node[a] = o[a] + (R)(idx[a] + win[a]) * p.dx;
        for (uint32_t r = 0; r < sc.n_rigid; ++r) {
          const float* q = sc.rigid[r];
          const R arm[3] = {node[0] - (R)q[0], node[1] - (R)q[1], node[2] - (R)q[2]};
          if (!(std::sqrt(arm[0] * arm[0] + arm[1] * arm[1] + arm[2] * arm[2]) < (R)q[3])) continue;
          const R m_old = g.mass[c];
          const R mom_old[3] = {g.mom[3 * c], g.mom[3 * c + 1], g.mom[3 * c + 2]};
          const R v[3] = {(R)q[4], (R)q[5], (R)q[6]};
          const R stamp = R(1.0e6);
          g.mass[c] = stamp;
          for (int a = 0; a < 3; ++a) g.mom[3 * c + a] = stamp * v[a];
          g.rigid[c] = 1;
          if (m_old > R(1.0e-9)) {
            const R inv_dt = R(1) / std::max(p.dt, R(1.0e-6));
            R f[3];
            for (int a = 0; a < 3; ++a) f[a] = -(m_old * v[a] - mom_old[a]) * inv_dt;
            const R t[3] = {arm[1] * f[2] - arm[2] * f[1], arm[2] * f[0] - arm[0] * f[2], arm[0] * f[1] - arm[1] * f[0]};
            for (int a = 0; a < 3; ++a) {
              sc.wrench[r][a] += (double)f[a];
              sc.wrench[r][3 + a] += (double)t[a];
            }
          }
          break;
        }
      }
}

// mpm_rigid_force_integrate (mpm.wgsl:1175-1228): non-rigid nodes with sand
// mass within radius + dx react with -(m w / dt) (v_sphere - v_node), w
// tapered linearly over the outer cell.
template <class R> static void rigid_shell(orc_scene& sc, const Params<R>& p, const Grid<R>& g) {
  const int n = p.n;
  const R o[3] = {p.ox, p.oy, p.oz};
  const int win[3] = {p.wx, p.wy, p.wz};
  for (int iz = 0; iz < n; ++iz)
    for (int iy = 0; iy < n; ++iy)
      for (int ix = 0; ix < n; ++ix) {
        const size_t c = (size_t)ix + (size_t)n * ((size_t)iy + (size_t)n * (size_t)iz);
        const R m = g.mass[c];
        if (m <= R(1.0e-9) || !(m == m) || g.rigid[c]) continue;
        const int idx[3] = {ix, iy, iz};
        R node[3];
        for (int a = 0; a < 3; ++a) node[a] = o[a] + (R)(idx[a] + win[a]) * p.dx;
        for (uint32_t r = 0; r < sc.n_rigid; ++r) {
          const float* q = sc.rigid[r];
          const R arm[3] = {node[0] - (R)q[0], node[1] - (R)q[1], node[2] - (R)q[2]};
          const R d = std::sqrt(arm[0] * arm[0] + arm[1] * arm[1] + arm[2] * arm[2]);
          if (d > (R)q[3] + p.dx) continue;
          R w = R(1);
          if (d > (R)q[3]) w = std::max(R(0), R(1) - (d - (R)q[3]) / p.dx);
          const R k = -(m * w / std::max(p.dt, R(1.0e-6)));
          R f[3];
          for (int a = 0; a < 3; ++a) f[a] = k * ((R)q[4 + a] - g.vel[3 * c + a]);
          const R t[3] = {arm[1] * f[2] - arm[2] * f[1], arm[2] * f[0] - arm[0] * f[2], arm[0] * f[1] - arm[1] * f[0]};
          for (int a = 0; a < 3; ++a) {
            sc.wrench[r][a] += (double)f[a];
            sc.wrench[r][3 + a] += (double)t[a];
          }
        }
      }
}

// mpm_implicit_apply + mpm_implicit_swap (mpm.wgsl:1060-1173): jacobi_iters
// sweeps on the grid velocity; a node with mass blends with the mean of its
// face neighbours that carry mass, at the rate a = dt^2 m (E / 1500) / dx^2.
template <class R> static void implicit_sweeps(const orc_scene& sc, const Params<R>& p, Grid<R>& g, int nthreads) {
  const int n = p.n;
  const size_t n3 = (size_t)n * n * n;
  std::vector<R> next(3 * n3);
  const R c2 = p.youngs / R(1500);
  for (uint32_t it = 0; it < sc.jacobi_iters; ++it) {
#pragma omp parallel for num_threads(nthreads > 1 ? nthreads : 1) schedule(static) if (nthreads > 1)
    for (int iz = 0; iz < n; ++iz)
      for (int iy = 0; iy < n; ++iy)
        for (int ix = 0; ix < n; ++ix) {
          const size_t c = (size_t)ix + (size_t)n * ((size_t)iy + (size_t)n * (size_t)iz);
          const R m = g.mass[c];
          const R* v = &g.vel[3 * c];
          R* o = &next[3 * c];
          if (m <= R(1.0e-9) || !(m == m) || (!g.rigid.empty() && g.rigid[c])) {
            o[0] = v[0];
            o[1] = v[1];
            o[2] = v[2];
            continue;
          }
          const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
          R avg[3] = {R(0), R(0), R(0)};
          R count = R(0);
          for (int k = 0; k < 6; ++k) {
            const int nx = ix + off[k][0], ny = iy + off[k][1], nz = iz + off[k][2];
            if (nx < 0 || ny < 0 || nz < 0 || nx >= n || ny >= n || nz >= n) continue;
            const size_t nc = (size_t)nx + (size_t)n * ((size_t)ny + (size_t)n * (size_t)nz);
            const R nm = g.mass[nc];
            if (nm <= R(1.0e-9) || !(nm == nm)) continue;
            for (int a = 0; a < 3; ++a) avg[a] = avg[a] + g.vel[3 * nc + a];
            count = count + R(1);
          }
          for (int a = 0; a < 3; ++a) avg[a] = count > R(0) ? avg[a] / count : v[a];
          const R alpha = p.dt * p.dt * m * c2 * p.inv_dx * p.inv_dx;
          const R denom = m + alpha;
          R vn[3];
          bool nan = false;
          for (int a = 0; a < 3; ++a) {
            vn[a] = (m * v[a] + alpha * avg[a]) / denom;
            nan = nan || !(vn[a] == vn[a]);
          }
          for (int a = 0; a < 3; ++a) o[a] = nan ? v[a] : vn[a];
        }
    g.vel.swap(next);
  }
}

template <class R> static inline bool finite_vec(const R* v) {
  return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

// g2p, mpm.wgsl:1242-1353.  Returns false on a numerical fault (state of the
// particle untouched).
template <class R> static bool g2p_particle(const orc_scene& sc, const Params<R>& p, const Grid<R>& g,
                                            State<R>& st, int pid) {
  R* pos = st.pos + 3 * pid;
  R* vel = st.vel + 3 * pid;
  const M3<R> Cold = load_m(st.C + 9 * pid);
  const M3<R> Fold = load_m(st.F + 9 * pid);
  if (!finite_vec(pos) || !finite_vec(vel) || !finite_m(Cold) || !finite_m(Fold) || !std::isfinite(st.jp[pid]))
    return false;
  const R o[3] = {p.ox, p.oy, p.oz};
  const int win[3] = {p.wx, p.wy, p.wz};
  R xp[3], bf[3], fx[3], w[3][3];
  int base[3];
  for (int a = 0; a < 3; ++a) xp[a] = (pos[a] - o[a]) * p.inv_dx;
  if (!finite_vec(xp)) return false;
  for (int a = 0; a < 3; ++a) {
    bf[a] = std::floor(xp[a] - R(0.5));
    base[a] = (int)bf[a] - win[a];
    fx[a] = xp[a] - bf[a];
    quad_weights(fx[a], w[a]);
  }
  R vn[3] = {0, 0, 0};
  M3<R> Cn = zero3<R>();
  const R inv_dx = p.inv_dx, dx = p.dx;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        const R wgt = w[0][i] * w[1][j] * w[2][k];
        const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
        if (ix < 0 || iy < 0 || iz < 0 || ix >= p.n || iy >= p.n || iz >= p.n) continue;
        const size_t c = (size_t)ix + (size_t)p.n * ((size_t)iy + (size_t)p.n * (size_t)iz);
        const R* gv = &g.vel[3 * c];
        for (int a = 0; a < 3; ++a) vn[a] = vn[a] + wgt * gv[a];
        const R d[3] = {((R)i - fx[0]) * dx, ((R)j - fx[1]) * dx, ((R)k - fx[2]) * dx};
        const R scale = R(4) * wgt * inv_dx * inv_dx;
        for (int col = 0; col < 3; ++col)
          for (int row = 0; row < 3; ++row) Cn.m[col][row] = Cn.m[col][row] + scale * gv[row] * d[col];
      }
  const MatConst<R> mc = mat_const<R>(sc, st.mat[pid], p);
  if (mc.rheo == 2) {
    const R vd = std::exp(-std::max(mc.vdamp, R(0)) * p.dt);
    const R ad = std::exp(-std::max(mc.adamp, R(0)) * p.dt);
    for (int a = 0; a < 3; ++a) vn[a] = vn[a] * vd;
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) Cn.m[c][r] = Cn.m[c][r] * ad;
  }
  R np[3];
  for (int a = 0; a < 3; ++a) np[a] = pos[a] + p.dt * vn[a];
  if (!finite_vec(np) || !finite_vec(vn) || !finite_m(Cn)) return false;
  const int pad = p.pad;
  for (int a = 0; a < 3; ++a) {
    const R lo = o[a] + (R)(win[a] + pad) * p.dx;
    const R hi = o[a] + (R)(win[a] + (p.n - pad - 1)) * p.dx;
    if (np[a] < lo || np[a] > hi) vn[a] = R(0);
    np[a] = clampr(np[a], lo, hi);
  }
  M3<R> A = ident3<R>();
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) A.m[c][r] = A.m[c][r] + p.dt * Cn.m[c][r];
  const M3<R> Fn = mul(A, Fold);
  if (!finite_m(Fn)) return false;
  for (int a = 0; a < 3; ++a) {
    pos[a] = np[a];
    vel[a] = vn[a];
  }
  store_m(st.C + 9 * pid, Cn);
  store_m(st.F + 9 * pid, Fn);
  return true;
}

// plasticity, mpm.wgsl:1366-1479.  Returns false on a numerical fault.
template <class R, class SR>
static bool plasticity_particle(const orc_scene& sc, const Params<R>& p, State<R>& st, int pid) {
  const MatConst<R> mc = mat_const<R>(sc, st.mat[pid], p);
  const M3<R> F = load_m(st.F + 9 * pid);
  if (!finite_m(F) || !std::isfinite(st.jp[pid])) return false;
  const Svd<R> svd = svd_in<R, SR>(F, sc);
  const R* s = svd.s;
  if (!finite_vec(s) || !finite_m(svd.u) || !finite_m(svd.v)) return false;
  R ns[3] = {s[0], s[1], s[2]};
  R dq = R(0);
  bool jp_replace = false;
  R jp_new = R(0);
  if (mc.rheo == 1) {
    for (int a = 0; a < 3; ++a) ns[a] = clampr(s[a], R(1) - mc.theta_c, R(1) + mc.theta_s);
    const R det_old = std::max(s[0] * s[1] * s[2], R(1.0e-6));
    const R det_new = std::max(ns[0] * ns[1] * ns[2], R(1.0e-6));
    const R dlog = std::log(det_old) - std::log(det_new);
    jp_replace = true;
    jp_new = st.jp[pid] + dlog;
    if (!std::isfinite(jp_new)) return false;
    jp_new = clampr(jp_new, R(-5), R(5));
  } else if (mc.rheo == 2) {
    jp_replace = true;
    jp_new = R(0);
  } else {
    const R d = R(3);
    R eps[3];
    for (int a = 0; a < 3; ++a) eps[a] = std::log(std::max(s[a], R(1.0e-6)));
    const R tr = eps[0] + eps[1] + eps[2];
    const R mean = tr / d;
    R dev[3];
    for (int a = 0; a < 3; ++a) dev[a] = eps[a] - mean;
    const R dev_norm = length3(dev);
    const R kappa = (d * mc.lam + R(2) * mc.mu) / (R(2) * mc.mu);
    if (tr > R(0)) {
      ns[0] = ns[1] = ns[2] = R(1);
      dq = length3(eps);
    } else if (dev_norm == R(0)) {
      // keep s
    } else {
      const R fy = dev_norm + kappa * tr * mc.dp_alpha;
      if (fy <= R(0)) {
        // keep s
      } else {
        const R rc = std::max(R(0), -mc.dp_alpha * kappa * tr);
        R ne[3];
        for (int a = 0; a < 3; ++a) {
          ne[a] = dev[a] * (rc / dev_norm) + mean;
          ns[a] = std::exp(ne[a]);
        }
        dq = fy;
      }
    }
  }
  if (!finite_vec(ns) || !std::isfinite(dq) || !std::isfinite(st.jp[pid] + dq)) return false;
  R ss[3];
  bool changed = false;
  for (int a = 0; a < 3; ++a) {
    ss[a] = clampr(ns[a], R(0.05), R(20));
    changed = changed || ss[a] != s[a];
  }
  // The FP64-SVD mode keeps the trial F when no singular value moved; the
  // reference (FP32 and FP64 runs) rebuilds F = U s V^T every substep.
  if (sizeof(SR) == sizeof(R) || changed) {
    const M3<R> Fn = diag_sandwich(svd.u, ss, svd.v);
    if (!finite_m(Fn)) return false;
    store_m(st.F + 9 * pid, Fn);
  }
  if (jp_replace) {
    st.jp[pid] = jp_new;
  } else {
    st.jp[pid] = clampr(st.jp[pid] + dq, R(0), R(5));
  }
  return true;
}

// One or more substeps in the reference dispatch order (mpm.rs:2476-2551):
// reset, p2g, grid_update, g2p, plasticity.  status[0] holds the fault bits
// (FAULT_NUMERICAL = 2 as in mpm.wgsl:229), status[1] the completed-substep
// count (mpm.wgsl:1246).  Once the latch is set, later kernels are no-ops
// (grid_valid(), mpm.wgsl:213-215).
template <class R, class SR>
static void step(orc_scene& sc, State<R>& st, R* out_mass, R* out_mom, uint32_t* status, int substeps,
                 int nthreads) {
  const Params<R> p = params_of<R>(sc);
  Grid<R> g;
  g.n = p.n;
  const size_t cells = (size_t)p.n * p.n * p.n;
  g.mass.assign(cells, R(0));
  g.mom.assign(3 * cells, R(0));
  g.vel.assign(3 * cells, R(0));
  if (sc.n_rigid) g.rigid.assign(cells, 0);
  for (int s = 0; s < substeps; ++s) {
    if (status[0] != 0) break;
    if (sc.n_rigid) {
      std::fill(g.rigid.begin(), g.rigid.end(), (uint8_t)0);
      for (uint32_t r = 0; r < sc.n_rigid; ++r)
        for (int k = 0; k < 6; ++k) sc.wrench[r][k] = 0.0;
    }
    {
      const long long nc = (long long)g.mass.size();
      R* gm = g.mass.data();
      R* gp = g.mom.data();
#pragma omp parallel for num_threads(nthreads > 1 ? nthreads : 1) schedule(static) if (nthreads > 1)
      for (long long c = 0; c < nc; ++c) {
        gm[c] = R(0);
        gp[3 * c] = gp[3 * c + 1] = gp[3 * c + 2] = R(0);
      }
    }
    if (nthreads <= 1) {
      for (int pid = 0; pid < st.n; ++pid) {
        p2g_particle<R, SR>(sc, p, st, pid, [&](size_t c, R dm, const R* mom) {
          g.mass[c] += dm;
          g.mom[3 * c] += mom[0];
          g.mom[3 * c + 1] += mom[1];
          g.mom[3 * c + 2] += mom[2];
        });
      }
    } else {
#pragma omp parallel for num_threads(nthreads) schedule(static)
      for (int pid = 0; pid < st.n; ++pid) {
        p2g_particle<R, SR>(sc, p, st, pid, [&](size_t c, R dm, const R* mom) {
#pragma omp atomic
          g.mass[c] += dm;
#pragma omp atomic
          g.mom[3 * c] += mom[0];
#pragma omp atomic
          g.mom[3 * c + 1] += mom[1];
#pragma omp atomic
          g.mom[3 * c + 2] += mom[2];
        });
      }
    }
    if (sc.n_rigid) rigid_imprint(sc, p, g);
    grid_update(p, g, nthreads);
    if (sc.jacobi_iters) implicit_sweeps(sc, p, g, nthreads);
    if (sc.n_rigid) rigid_shell(sc, p, g);
    status[1] += 1;
    bool fault = false;
    if (nthreads <= 1) {
      for (int pid = 0; pid < st.n; ++pid)
        if (!g2p_particle(sc, p, g, st, pid)) fault = true;
    } else {
      int f = 0;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(| : f)
      for (int pid = 0; pid < st.n; ++pid)
        if (!g2p_particle(sc, p, g, st, pid)) f = 1;
      fault = f != 0;
    }
    if (fault) {
      status[0] |= FAULT_NUMERICAL;
      break;
    }
    if (nthreads <= 1) {
      for (int pid = 0; pid < st.n; ++pid)
        if (!plasticity_particle<R, SR>(sc, p, st, pid)) fault = true;
    } else {
      int f = 0;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(| : f)
      for (int pid = 0; pid < st.n; ++pid)
        if (!plasticity_particle<R, SR>(sc, p, st, pid)) f = 1;
      fault = f != 0;
    }
    if (fault) {
      status[0] |= FAULT_NUMERICAL;
      break;
    }
  }
  if (out_mass) std::copy(g.mass.begin(), g.mass.end(), out_mass);
  if (out_mom) std::copy(g.mom.begin(), g.mom.end(), out_mom);
}

}  // namespace orc

extern "C" {

// FP32 state; svd_fp64 != 0 runs the SVD in FP64 (the north-star precision).
// nthreads > 1 selects the OpenMP form (atomic accumulation; the timed CPU
// baseline).  grid_mass/grid_mom (n^3 and 3 n^3) receive the last substep's
// P2G result and may be null.
int orc_step_f32(orc_scene* sc, int n, float* pos, float* vel, float* C, float* F, float* mass,
                 float* vol, float* jp, const uint32_t* mat, float* grid_mass, float* grid_mom,
                 uint32_t* status, int substeps, int svd_fp64, int nthreads) {
  orc::State<float> st{n, pos, vel, C, F, mass, vol, jp, mat};
  if (svd_fp64)
    orc::step<float, double>(*sc, st, grid_mass, grid_mom, status, substeps, nthreads);
  else
    orc::step<float, float>(*sc, st, grid_mass, grid_mom, status, substeps, nthreads);
  return 0;
}

// FP64 everywhere (the accuracy reference).
int orc_step_f64(orc_scene* sc, int n, double* pos, double* vel, double* C, double* F, double* mass,
                 double* vol, double* jp, const uint32_t* mat, double* grid_mass, double* grid_mom,
                 uint32_t* status, int substeps, int nthreads) {
  orc::State<double> st{n, pos, vel, C, F, mass, vol, jp, mat};
  orc::step<double, double>(*sc, st, grid_mass, grid_mom, status, substeps, nthreads);
  return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// svd3_jacobi on one matrix (column-major F[9]); mpm.wgsl:365-468.
void orc_svd3_f32(const float* F, float* U, float* s, float* V, double tol, int sweeps) {
  orc::M3<float> f = orc::load_m(F);
  orc::Svd<float> r = orc::svd3_jacobi<float>(f, (float)tol, sweeps);
  orc::store_m(U, r.u);
  orc::store_m(V, r.v);
  for (int i = 0; i < 3; ++i) s[i] = r.s[i];
}
void orc_svd3_f64(const double* F, double* U, double* s, double* V, double tol, int sweeps) {
  orc::M3<double> f = orc::load_m(F);
  orc::Svd<double> r = orc::svd3_jacobi<double>(f, tol, sweeps);
  orc::store_m(U, r.u);
  orc::store_m(V, r.v);
  for (int i = 0; i < 3; ++i) s[i] = r.s[i];
}

// The plasticity kernel body of the step (mpm.wgsl:1366-1479) on one
// particle, FP64.  Returns 1 on success, 0 on a numerical fault.
int orc_plasticity_f64(const orc_scene* sc, double* F, double* jp, uint32_t mat) {
  orc::Params<double> p = orc::params_of<double>(*sc);
  orc::State<double> st{1, nullptr, nullptr, nullptr, F, nullptr, nullptr, jp, &mat};
  return orc::plasticity_particle<double, double>(*sc, p, st, 0) ? 1 : 0;
}

// G2P gather of a prescribed node-velocity field (4 doubles per node, xyz + pad),
// mpm_gather_oracle.rs:3-41 (f64) — the same arithmetic as the step's g2p.
void orc_gather_f64(const orc_scene* sc, const double* pos, const double* grid_vel4, double* v_out, double* C_out) {
  orc::Params<double> p = orc::params_of<double>(*sc);
  const double o[3] = {p.ox, p.oy, p.oz};
  double xp[3], bf[3], fx[3], w[3][3];
  int base[3];
  for (int a = 0; a < 3; ++a) {
    xp[a] = (pos[a] - o[a]) / p.dx;
    bf[a] = std::floor(xp[a] - 0.5);
    base[a] = (int)bf[a];
    fx[a] = xp[a] - bf[a];
    orc::quad_weights(fx[a], w[a]);
  }
  double v[3] = {0, 0, 0};
  double Cm[9] = {0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
        if (ix < 0 || iy < 0 || iz < 0 || ix >= p.n || iy >= p.n || iz >= p.n) continue;
        const size_t c = (size_t)ix + (size_t)p.n * ((size_t)iy + (size_t)p.n * (size_t)iz);
        const double* gv = grid_vel4 + 4 * c;
        const double wgt = w[0][i] * w[1][j] * w[2][k];
        const double d[3] = {((double)i - fx[0]) * p.dx, ((double)j - fx[1]) * p.dx, ((double)k - fx[2]) * p.dx};
        for (int a = 0; a < 3; ++a) v[a] += wgt * gv[a];
        for (int col = 0; col < 3; ++col)
          for (int row = 0; row < 3; ++row) Cm[3 * col + row] += gv[row] * d[col] * (4.0 * wgt / (p.dx * p.dx));
      }
  for (int a = 0; a < 3; ++a) v_out[a] = v[a];
  for (int a = 0; a < 9; ++a) C_out[a] = Cm[a];
}

// tile_keys, mpm_particle_order.wgsl:11-25, followed by the stable ascending
// sort of (key, identity) pairs (radix_sort.rs:20-30; radix_sort_gpu.rs:299-305).
// positions: 3 floats per particle (count of them); keys/ids: capacity entries.
// Entries at or beyond `count` get key 0xFFFFFFFF and keep their identity.
void orc_particle_order(const orc_scene* sc, uint32_t count, uint32_t capacity, const float* positions,
                        uint32_t* keys, uint32_t* ids) {
  const uint32_t n = sc->grid_size;
  const uint32_t width = (n + 3u) / 4u;
  std::vector<std::pair<uint32_t, uint32_t>> kv(capacity);
  for (uint32_t id = 0; id < capacity; ++id) {
    uint32_t key = 0xffffffffu;
    if (id < count) {
      uint32_t tile[3];
      for (int a = 0; a < 3; ++a) {
        const float x = (positions[3 * id + a] - sc->origin[a]) * sc->inv_cell_size;
        const float fl = std::floor(x);
        // i32(f32) conversion saturates in WGSL; clamp the float first.
        int32_t cell;
        if (!(fl == fl)) cell = 0;
        else if (fl >= 2147483520.0f) cell = 2147483647;
        else if (fl <= -2147483648.0f) cell = (int32_t)(-2147483647 - 1);
        else cell = (int32_t)fl;
        cell -= sc->window[a];
        if (cell < 0) cell = 0;
        if (cell > (int32_t)(n - 1u)) cell = (int32_t)(n - 1u);
        tile[a] = (uint32_t)cell / 4u;
      }
      key = tile[0] + width * (tile[1] + width * tile[2]);
    }
    kv[id] = {key, id};
  }
  std::stable_sort(kv.begin(), kv.end(),
                   [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                     return a.first < b.first;
                   });
  for (uint32_t i = 0; i < capacity; ++i) {
    keys[i] = kv[i].first;
    ids[i] = kv[i].second;
  }
}

// Stable sort of (u32 key, u32 value) pairs by key: the CPU reference of
// crates/molla-compute-primitives/tests/radix_sort_gpu.rs:299-305.
void orc_sort_pairs(uint32_t n, uint32_t* keys, uint32_t* values) {
  std::vector<std::pair<uint32_t, uint32_t>> kv(n);
  for (uint32_t i = 0; i < n; ++i) kv[i] = {keys[i], values[i]};
  std::stable_sort(kv.begin(), kv.end(),
                   [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                     return a.first < b.first;
                   });
  for (uint32_t i = 0; i < n; ++i) {
    keys[i] = kv[i].first;
    values[i] = kv[i].second;
  }
}

// material_row dp_alpha in f32 (crates/molla-solvers/src/mpm.rs:662-668):
// sqrt(2/3) * (2 sin(phi)) / (3 - sin(phi)), no 1-degree floor on this path.
float orc_dp_alpha_f32(float phi) {
  const float sp = std::sin(phi);
  return std::sqrt(2.0f / 3.0f) * (2.0f * sp) / (3.0f - sp);
}

// ---- f64 material twins: crates/molla-solvers/src/mpm_oracle.rs:174-359 ----

// drucker_prager_alpha, mpm_oracle.rs:251-256 (phi >= 1 degree).
double orc_dp_alpha_f64(double phi) {
  const double pi = 3.14159265358979323846;
  phi = std::max(phi, 1.0 * pi / 180.0);
  const double sp = std::sin(phi);
  return std::sqrt(2.0 / 3.0) * (2.0 * sp) / (3.0 - sp);
}

// snow_clamp_singular_values, mpm_oracle.rs:174-195.
void orc_snow_clamp_f64(const double* s, double jp, double theta_c, double theta_s, double* out_s, double* out_jp) {
  const double lo = 1.0 - theta_c, hi = 1.0 + theta_s;
  for (int a = 0; a < 3; ++a) out_s[a] = std::min(std::max(s[a], lo), hi);
  const double det_old = std::max(s[0] * s[1] * s[2], 1.0e-6);
  const double det_new = std::max(out_s[0] * out_s[1] * out_s[2], 1.0e-6);
  const double v = jp + (std::log(det_old) - std::log(det_new));
  *out_jp = std::min(std::max(v, -5.0), 5.0);
}

// sand_project_singular_values, mpm_oracle.rs:316-359.
void orc_sand_project_f64(const double* s, double jp, double youngs, double poisson, double phi, double* out_s,
                          double* out_jp) {
  const double mu = youngs / (2.0 * (1.0 + poisson));
  const double lam = youngs * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
  const double d = 3.0;
  const double alpha = orc_dp_alpha_f64(phi);
  double eps[3];
  for (int a = 0; a < 3; ++a) eps[a] = std::log(std::max(s[a], 1.0e-6));
  const double tr = eps[0] + eps[1] + eps[2];
  const double mean = tr / d;
  double dev[3];
  for (int a = 0; a < 3; ++a) dev[a] = eps[a] - mean;
  const double dn = std::sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const double kappa = (d * lam + 2.0 * mu) / (2.0 * mu);
  double dq = 0.0;
  for (int a = 0; a < 3; ++a) out_s[a] = s[a];
  if (tr > 0.0) {
    for (int a = 0; a < 3; ++a) out_s[a] = 1.0;
    dq = std::sqrt(eps[0] * eps[0] + eps[1] * eps[1] + eps[2] * eps[2]);
  } else if (dn == 0.0) {
  } else {
    const double fy = dn + kappa * tr * alpha;
    if (fy > 0.0) {
      const double rc = std::max(-alpha * kappa * tr, 0.0);
      for (int a = 0; a < 3; ++a) out_s[a] = std::exp(dev[a] * (rc / dn) + mean);
      dq = fy;
    }
  }
  *out_jp = std::min(std::max(jp + dq, 0.0), 5.0);
}

// viscous_damping_step, mpm_oracle.rs:137-157.
void orc_viscous_damping_f64(const double* v, const double* C, double dt, double vd, double ad, double* out_v,
                             double* out_C, double* factors) {
  const double fv = std::exp(-std::max(vd, 0.0) * std::max(dt, 0.0));
  const double fa = std::exp(-std::max(ad, 0.0) * std::max(dt, 0.0));
  for (int a = 0; a < 3; ++a) out_v[a] = v[a] * fv;
  for (int a = 0; a < 9; ++a) out_C[a] = C[a] * fa;
  factors[0] = fv;
  factors[1] = fa;
}

}  // extern "C"
