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
  pdl_wait();
  if (threadIdx.x != 0) return;
  d->obs_now = 0;
  d->snap_slot = -1;
  d->maxdp = 0ull;
  if (!d->active) return;
  if (!(d->t < d->t_fin)) {
    d->active = 0;
    return;
  }
  const double t = d->t, dt = d->dt;
  if (d->it % d->res == 0) {
    d->obs_now = 1;
    if (d->snap_on && t > d->print_start + d->icont * d->print_step && t < d->print_end) {
      d->icont++;
      // slots exist when snap_cap > 0; without them only the time is kept
      if (d->icont >= d->snap_tcap || (d->snap_cap > 0 && d->icont >= d->snap_cap)) {
        d->fault = kDynFaultSnapshots;
        d->active = 0;
        d->obs_now = 0;
        return;
      }
      d->snap_t[d->icont] = t * kAuFs;
      if (d->snap_cap > 0) d->snap_slot = d->icont;
    }
  }
  if (!d->taylor) {
    const double dt6 = dt / 6.0, dt3 = dt / 3.0, dt2 = dt / 2.0;
    field_sum(d->pump, d->n_pumps, d->probe, t, d->EF[0]);
    field_sum(d->pump, d->n_pumps, d->probe, t + dt2, d->EF[1]);
    field_sum(d->pump, d->n_pumps, d->probe, t + dt, d->EF[2]);
    d->c[0][0] = dt6;
    d->c[0][1] = dt2;
    d->c[1][0] = dt3;
    d->c[1][1] = dt2;
    d->c[2][0] = dt3;
    d->c[2][1] = dt;
    d->c[3][0] = dt6;
    d->c[3][1] = 0.;
  } else {
    field_sum(d->pump, d->n_pumps, d->probe, t, d->EF[0]);
    d->e_non0 = field_is_nonzero(d->EF[0]);
    const int TO = d->order, m = TO - 1;
    double ti[kMaxOrder], tau[kMaxOrder * kMaxOrder];
    ti[0] = d->dt_prev[0];
    for (int i = 1; i < m; i++) ti[i] = ti[i - 1] + d->dt_prev[i - 1];
    const double scale = 1.0e7;
    for (int i = 0; i < m; i++)
      for (int q = 0; q < m; q++) tau[i * m + q] = scale * pow(ti[i], (double)(q + 1));
    if (!inv_small(m, tau, d->tinv)) {
      d->fault = kDynFaultTaylor;
      d->active = 0;
      d->obs_now = 0;
      d->snap_slot = -1;
      return;
    }
    for (int i = 0; i < m * m; i++) d->tinv[i] *= scale;
    for (int i = 0; i < TO; i++) d->tpow[i] = pow(dt, (double)(i + 1));
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
