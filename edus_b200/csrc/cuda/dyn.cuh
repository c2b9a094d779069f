// dyn.cuh — adaptive time step on the device (Source_Main/dyn_dt_evolution.cpp).
//
// The reference's adaptive loop (dyn_dt_evolution.cpp:1-183) keeps its clock,
// step and field on the host and reduces the step's largest population change
// over all ranks before it picks the next step (:64-133). Here those scalars
// live in one DynStep in device memory: k_dyn_begin opens a step (stops the
// run at t_fin, decides the output instant and the snapshot slot, evaluates
// the stage fields and the integrator's coefficients), the stage kernels read
// them from it, the last stage's max reduction lands in it, and k_dyn_end
// picks the next step and advances the clock. A whole adaptive run is then a
// chain of captured kernels with no host round trip per step; the host only
// watches the `active` flag, a few chunks behind.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "../../../include/edus_b200.h"
#include "dev.cuh"

namespace edus {

struct DynStep {
  // configuration (fixed for the run)
  edus_laser pump[EDUS_MAX_PUMPS];
  edus_laser probe;
  int n_pumps;
  int taylor;       // 0: RK4 (Source_Main/RungeKutta.cpp), 1: Taylor (Taylor_DE_solver_deriv_Polynom.cpp)
  int order;        // Taylor order
  int res;          // it_resolution: an output instant every res steps
  int log_cap;      // records the log holds
  int snap_on;      // PrintPopulation / Print_new_band_dispersion snapshot switch
  int snap_cap;     // per-k snapshot slots (0: times only)
  int snap_tcap;    // entries of snap_t
  double print_start, print_end, print_step;
  double t_fin, eps, dt0;
  const double* pcmax;  // P_cond_max, n_cond of the last output instant (observable kernel outputs)
  const double* ncond;
  double* snap_t;       // [snap_tcap] snapshot times (fs)
  // loop state (the reference's scalars)
  double t, dt;
  int it, nlog, icont;
  int active;           // 1 while t < t_fin; never set back by the device
  int fault;            // 0, or kDynFault*
  int e_non0;
  double EF_last[2][3];  // field of the last evaluation, recorded with the next output instant
  double dt_prev[kMaxOrder];
  // this step
  int obs_now;           // the step begins with an output instant
  int snap_slot;         // its snapshot slot, -1 none
  double EF[3][2][3];    // RK4: fields at t, t + dt/2, t + dt; Taylor: at t
  double c[4][2];        // RK4 stage coefficients (c1, c2)
  double tinv[kMaxOrder * kMaxOrder];  // Taylor tau^-1 (scaled)
  double tpow[kMaxOrder];              // dt^(i+1)
  unsigned long long maxdp;            // max population change of the step (FP64 bits)
};

constexpr int kDynFaultSnapshots = 1;  // a snapshot past the allocated slots
constexpr int kDynFaultTaylor = 2;     // singular Taylor tau matrix

// Electric field of one laser at time t (headers/Laser.h:56-76,128-144:
// Gaussian, sin^2 and piecewise-linear envelopes times sin / cos carriers on
// two polarisations).
// Host and device run this same function.
__host__ __device__ inline void laser_field(const edus_laser& L, double t, double E[3]) {
  double env = 0.;
  if (L.envelope_kind == EDUS_ENV_GAUSS) {
    const double d = t - L.t0;
    env = (d * d < 40 * L.sigma * L.sigma) ? L.E0 * exp(-d * d / (2 * L.sigma * L.sigma)) : 0.;
  } else if (L.envelope_kind == EDUS_ENV_SIN2) {
    if (t >= L.t0 && t <= L.tf) {
      const double s = sin(3.14159265358979323846 * (t - L.t0) / (L.tf - L.t0));
      env = L.E0 * (s * s);
    }
  } else if (L.envelope_kind == EDUS_ENV_PW) {
    double tr = 0.;
    if (t >= L.t0 && t < L.w1)
      tr = (t - L.t0) / (L.w1 - L.t0);
    else if (t >= L.w1 && t < L.w2)
      tr = 1.;
    else if (t >= L.w2 && t <= L.tf)
      tr = (t - L.tf) / (L.w2 - L.tf);
    env = L.E0 * tr;
  }
  const double p1 = L.envelope_only ? 1. : sin(L.wl * (t - L.t0) + L.phase);
  const double p2 = L.envelope_only ? 1. : cos(L.wl * (t - L.t0) + L.phase);
  for (int i = 0; i < 3; i++) E[i] = env * (p1 * L.pol1[i] + p2 * L.pol2[i]);
}

// Pump sum and half the probe (Source_Main/RungeKutta.cpp:24-30).
__host__ __device__ inline void field_sum(const edus_laser* pump, int n_pumps, const edus_laser& probe, double t,
                                          double EF[2][3]) {
  for (int i = 0; i < 3; i++) EF[0][i] = 0.;
  for (int ip = 0; ip < n_pumps; ip++) {
    double e[3];
    laser_field(pump[ip], t, e);
    for (int i = 0; i < 3; i++) EF[0][i] += e[i];
  }
  double e2[3];
  laser_field(probe, t, e2);
  for (int i = 0; i < 3; i++) EF[1][i] = .5 * e2[i];
}

__host__ __device__ inline bool field_is_nonzero(const double EF[2][3]) {
  double s = 0;
  for (int a = 0; a < 2; a++)
    for (int i = 0; i < 3; i++) s += EF[a][i] * EF[a][i];
  return sqrt(s) > 1e-20;
}

// Inverse of an m x m matrix (m < kMaxOrder) by Gauss-Jordan elimination with
// partial pivoting; false when a pivot is zero.
__host__ __device__ inline bool inv_small(int m, const double* A, double* Ainv) {
  double a[kMaxOrder][2 * kMaxOrder];
  for (int i = 0; i < m; i++)
    for (int j = 0; j < 2 * m; j++) a[i][j] = (j < m) ? A[i * m + j] : (j - m == i ? 1.0 : 0.0);
  for (int c = 0; c < m; c++) {
    int piv = c;
    for (int r = c + 1; r < m; r++)
      if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
    if (a[piv][c] == 0.0) return false;
    if (piv != c)
      for (int j = 0; j < 2 * m; j++) {
        const double t = a[c][j];
        a[c][j] = a[piv][j];
        a[piv][j] = t;
      }
    const double d = a[c][c];
    for (int j = 0; j < 2 * m; j++) a[c][j] /= d;
    for (int r = 0; r < m; r++) {
      if (r == c) continue;
      const double f = a[r][c];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * m; j++) a[r][j] -= f * a[c][j];
    }
  }
  for (int i = 0; i < m; i++)
    for (int j = 0; j < m; j++) Ainv[i * m + j] = a[i][m + j];
  return true;
}

// One-thread kernels around every step (dyn.cu).
cudaError_t launch_dyn_begin(DynStep* d, cudaStream_t s);
cudaError_t launch_dyn_end(DynStep* d, cudaStream_t s);

}  // namespace edus
