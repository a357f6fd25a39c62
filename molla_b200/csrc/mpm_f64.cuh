// mpm_f64.cuh — the all-FP64 substep (precision studies): scene constants,
// state pointers and launchers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {

struct Mat64 {
  int rheo;  // 0 sand, 1 snow, 2 viscous
  double mu, lam, kappa, dp_alpha, theta_c, theta_s, hardening, vdamp, adamp;
};

struct Scene64 {
  int n;
  double dx, inv_dx, o[3];
  int win[3];
  double dt, gy, friction;
  int pad, sticky;
  double lo[3], hi[3];  // position clamp box (mpm.wgsl:1327-1340)
  double tol;
  int sweeps;
  int n_mat;
  Mat64 mat[8];
};

struct State64 {
  int n;
  double *pos, *vel, *C, *F, *mass, *vol, *jp;  // 3n, 3n, 9n, 9n, n, n, n
  const uint32_t* mat;
  double *gmass, *gmom, *gvel;  // n^3, 3 n^3, 3 n^3
  uint32_t* status;             // fault word, completed substeps
};

// `substeps` reference substeps (reset, p2g, grid update, g2p, plasticity).
cudaError_t launch_step64(const Scene64& sc, const State64& st, uint32_t substeps, cudaStream_t s);
// Grid mass and momentum totals of the last P2G into out4 (device).
cudaError_t launch_totals64(const Scene64& sc, const State64& st, double* out4, cudaStream_t s);

}  // namespace mpm
