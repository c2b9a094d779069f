// dyn.cu — the two one-thread kernels of the device-side adaptive time step
// (Source_Main/dyn_dt_evolution.cpp:1-183).
#include "dyn.cuh"

namespace edus {
namespace {

constexpr double kAuFs = 0.02418884326505;  // fs per a.u. of time

// Open a step: the loop test (dyn_dt_evolution.cpp: while time_loop < t_fin),
// the output instant every res steps and its snapshot switch
// (Source_Main/if_resolution.cpp:18-33), the stage fields at t, t + dt/2,
// t + dt and the RK4 coefficients dt/6, dt/3, dt/2 (Source_Main/RungeKutta.cpp),
// or the Taylor step's tau^-1 and dt powers from the last TO - 1 steps
// (Source_Main/Taylor_DE_solver_deriv_Polynom.cpp:1-177). Clears the max.
__global__ void k_dyn_begin(DynStep* d) {
  // one warp: lane 0 keeps the loop state; the stage fields, the tau entries
  // and the Gauss-Jordan row operations are spread over the lanes
  __shared__ double a[kMaxOrder][2 * kMaxOrder];
  __shared__ int stop, piv_s;
  pdl_wait();
  const int lane = threadIdx.x;
  if (lane == 0) {
    stop = 0;
    d->obs_now = 0;
    d->snap_slot = -1;
    d->maxdp = 0ull;
    if (!d->active) {
      stop = 1;
    } else if (!(d->t < d->t_fin)) {
      d->active = 0;
      stop = 1;
    } else if (d->it % d->res == 0) {
      d->obs_now = 1;
      const double t = d->t;
      if (d->snap_on && t > d->print_start + d->icont * d->print_step && t < d->print_end) {
        d->icont++;
        // slots exist when snap_cap > 0; without them only the time is kept
        if (d->icont >= d->snap_tcap || (d->snap_cap > 0 && d->icont >= d->snap_cap)) {
          d->fault = kDynFaultSnapshots;
          d->active = 0;
          d->obs_now = 0;
          stop = 1;
        } else {
          d->snap_t[d->icont] = t * kAuFs;
          if (d->snap_cap > 0) d->snap_slot = d->icont;
        }
      }
    }
  }
  __syncwarp();
  if (stop) return;
  const double t = d->t, dt = d->dt;
  if (!d->taylor) {
    const double dt2 = dt / 2.0;
    if (lane < 3) field_sum(d->pump, d->n_pumps, d->probe, lane == 0 ? t : (lane == 1 ? t + dt2 : t + dt), d->EF[lane]);
    if (lane == 0) {
      const double dt6 = dt / 6.0, dt3 = dt / 3.0;
      d->c[0][0] = dt6;
      d->c[0][1] = dt2;
      d->c[1][0] = dt3;
      d->c[1][1] = dt2;
      d->c[2][0] = dt3;
      d->c[2][1] = dt;
      d->c[3][0] = dt6;
      d->c[3][1] = 0.;
    }
    return;
  }
  // Taylor: tau_iq = 1e7 ti^(q+1) with ti the sums of the last steps, its
  // inverse by Gauss-Jordan elimination with partial pivoting (as the host
  // loop's inv_gj), and dt^(i+1)
  const int TO = d->order, m = TO - 1;
  if (lane == 31) {
    field_sum(d->pump, d->n_pumps, d->probe, t, d->EF[0]);
    d->e_non0 = field_is_nonzero(d->EF[0]);
  }
  const double scale = 1.0e7;
  for (int q = lane; q < m * m; q += 32) {
    const int i = q / m, c = q - i * m;
    double ti = d->dt_prev[0];
    for (int r = 1; r <= i; r++) ti += d->dt_prev[r - 1];
    a[i][c] = scale * pow(ti, (double)(c + 1));
  }
  for (int q = lane; q < m * m; q += 32) {
    const int i = q / m, c = q - i * m;
    a[i][m + c] = (c == i) ? 1.0 : 0.0;
  }
  if (lane < TO) d->tpow[lane] = pow(dt, (double)(lane + 1));
  __syncwarp();
  for (int c = 0; c < m; c++) {
    if (lane == 0) {
      int piv = c;
      for (int r = c + 1; r < m; r++)
        if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
      piv_s = a[piv][c] == 0.0 ? -1 : piv;
    }
    __syncwarp();
    const int piv = piv_s;
    if (piv < 0) {
      if (lane == 0) {
        d->fault = kDynFaultTaylor;
        d->active = 0;
        d->obs_now = 0;
        d->snap_slot = -1;
      }
      return;
    }
    if (piv != c && lane < 2 * m) {
      const double x = a[c][lane];
      a[c][lane] = a[piv][lane];
      a[piv][lane] = x;
    }
    __syncwarp();
    const double pv = a[c][c];
    __syncwarp();
    if (lane < 2 * m) a[c][lane] /= pv;
    __syncwarp();
    // every other row r: a[r][j] -= a[r][c] a[c][j] (the multiplier read before the row changes)
    for (int q = lane; q < m * 2 * m; q += 32) {
      const int r = q / (2 * m), j = q - r * 2 * m;
      if (r == c) continue;
      const double f = a[r][c];
      if (f == 0.0) continue;
      if (j != c) a[r][j] -= f * a[c][j];
    }
    __syncwarp();
    for (int r = lane; r < m; r += 32)
      if (r != c) a[r][c] -= a[r][c] * a[c][c];
    __syncwarp();
  }
  for (int q = lane; q < m * m; q += 32) {
    const int i = q / m, c = q - i * m;
    d->tinv[q] = a[i][m + c] * scale;
  }
}

// Close a step: the next step from the largest population change
// (dyn_dt_evolution.cpp:100-124: shrink by eps / max above eps while dt > 0.01,
// else grow by 2 % up to dt0), the Taylor step history, the clock advanced by
// the new step as the reference does, and the step and output counters.
__global__ void k_dyn_end(DynStep* d) {
  pdl_wait();
  if (threadIdx.x != 0 || !d->active) return;
  const double mx = __longlong_as_double((long long)d->maxdp);
  double dt = d->dt;
  if ((mx > d->eps) && (dt > 0.01))
    dt *= d->eps / mx;
  else if (dt < d->dt0)
    dt *= 1.02;
  d->dt = dt;
  const int last = d->taylor ? 0 : 2;
  for (int a = 0; a < 2; a++)
    for (int i = 0; i < 3; i++) d->EF_last[a][i] = d->EF[last][a][i];
  if (d->taylor) {
    for (int i = d->order - 1; i > 0; i--) d->dt_prev[i] = d->dt_prev[i - 1];
    d->dt_prev[0] = dt;
  } else {
    d->e_non0 = field_is_nonzero(d->EF[2]);
  }
  if (d->obs_now) d->nlog++;
  d->t += dt;
  d->it++;
}

}  // namespace

cudaError_t launch_dyn_begin(DynStep* d, cudaStream_t s) { return launch_pdl(k_dyn_begin, dim3(1), dim3(32), 0, s, d); }
cudaError_t launch_dyn_end(DynStep* d, cudaStream_t s) { return launch_pdl(k_dyn_end, dim3(1), dim3(32), 0, s, d); }

}  // namespace edus
