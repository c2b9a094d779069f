// capi.cu — the C ABI: problem objects, device context, time loop, outputs.
//
// The time loop reproduces Source_Main/const_dt_evolution.cpp:1-54 and
// Source_Main/dyn_dt_evolution.cpp:1-183 of the reference: output instants
// before the step at it % it_resolution == 0, RK4 with the stage-3 field reuse
// and the E_non0 bookkeeping of Source_Main/RungeKutta.cpp:151-163, AB with a
// zero derivative history (headers/ODE_solver.h:40-62), Taylor with its tau
// matrix (Source_Main/Taylor_DE_solver_deriv_Polynom.cpp:100-123), adaptive dt.
// All kernel launches go to one stream and nothing synchronises with the host
// inside a constant-dt run; the observable log stays on the device until read.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <mutex>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "ctx_hooks.hpp"
#include "cuda/kernels.hpp"
#include "cuda/tc_contract.hpp"
#include "cuda/dyn.cuh"
#include "host/problem.hpp"

namespace edus {
namespace {

#define CK(x)                                                                             \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) return fail(EDUS_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

// Source_Main/RungeKutta.cpp:24-30 (laser_field: headers/Laser.h:56-76,128-144)
void field_at(const edus_params& p, double t, double EF[2][3]) { field_sum(p.pump, p.n_pumps, p.probe, t, EF); }

static bool field_nonzero(const double EF[2][3]) {
  double Emax = 0;
  for (int a = 0; a < 2; a++)
    for (int i = 0; i < 3; i++) Emax += EF[a][i] * EF[a][i];
  return std::sqrt(Emax) > 1e-20;
}

}  // namespace edus

using namespace edus;

struct edus_ctx {
  Problem P;
  int device = 0;
  cudaStream_t stream = nullptr;
  int n = 0, ntri = 0, nk = 0;
  size_t plane = 0;  // ntri * nk
  DevTables tb{};
  DevConsts hc{};
  DevConsts* d_cst = nullptr;
  std::vector<void*> allocs;
  double2 *d_P0 = nullptr, *d_P1 = nullptr, *d_Pa = nullptr, *d_Pb = nullptr, *d_ring = nullptr, *d_hr = nullptr;
  double2 *d_h = nullptr, *d_X0 = nullptr;
  // Coulomb in the diagonal basis: the state in the eigenbasis and the rotated term
  bool diagb = false;
  double2 *d_pdiag = nullptr, *d_xw = nullptr;
  CoulDev cd{};
  void* d_part = nullptr;
  unsigned int* d_done = nullptr;
  int* d_err = nullptr;  // device error word set by bounded waits
  edus_obs* d_log = nullptr;
  edus_obs* d_obs_one = nullptr;  // record of edus_observables, allocated on its first call
  size_t dev_bytes = 0;            // device memory the context holds
  long long async_l0 = 0;          // launch count at the start of an asynchronous whole run
  int log_cap = 0, nlog = 0;
  double* d_ncond = nullptr;
  double* d_pcmax = nullptr;
  // per-k snapshots (PrintPopulation / Print_new_band_dispersion): icont and
  // the times as the reference counts them; with PrintPopulation, slot m of
  // d_snap holds snapshot m's three eigenbasis elements [3][nk]; with the
  // Coulomb mean field, slot m of d_edia its band energies [n][nk]
  bool snap_on = false;
  int icont = -1, snap_cap = 0, snap_ic = 0, snap_jc = 0;
  double2* d_snap = nullptr;
  double* d_edia = nullptr;
  std::vector<double> snap_t;
  unsigned long long* d_maxdp = nullptr;
  // adaptive step on the device (whole runs): the step scalars, a pinned copy
  // of their active flag, the snapshot times, and the captured chunk of steps
  // with the host state it was captured from
  DynStep* d_dyn = nullptr;
  int* h_active = nullptr;
  double* d_snapt = nullptr;
  int snapt_cap = 0;
  cudaGraph_t dyn_graph = nullptr;
  cudaGraphExec_t dyn_exec = nullptr;
  long long dyn_chunk_launches = 0;
  int dyn_K = 0, dyn_phase = -1;
  double2* dyn_P0 = nullptr;
  int dyn_ring[kMaxOrder]{};
  cudaEvent_t dyn_ev[2]{};
  // loop state (host mirror of the reference's scalars)
  int it = 0, itfi = 0, res = 1;
  double time_loop = 0, dt = 0, dt0 = 0;
  double EF[2][3]{};
  bool e_non0 = true;
  int ring_idx[kMaxOrder]{};
  double dt_prev[kMaxOrder]{};
  double P_cond_max = 0, n_cond = 0;
  int solver = 0, order = 0;
  bool dyn = false, coul = false;
  // velocity gauge: the model tables tb.H, tb.D hold H, D at k + A(t) of the
  // last stage; A(t) = -int E_pump dt tracked on the host up to time vg_t
  bool vg = false;
  VgArgs vga{};
  // velocity gauge with the stage contraction on the tensor cores (precision
  // EDUS_PREC_MIXED): exact-slice GEMM, FP64 planes
  bool vg_tc = false;
  batch::TcVgArgs vgt{};
  double vg_t = 0, vg_A[3] = {0, 0, 0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
  long long launches = 0, last_launches = 0;
  // per-kernel event timing
  bool profiling = false;
  int prof_reps = 1;  // back-to-back repeats of each idempotent RHS launch under edus_profile_ex
  cudaEvent_t prof_open[2]{};
  struct ProfPair {
    int kind;
    cudaEvent_t a, b;
    int reps;
  };
  std::vector<ProfPair> prof_pairs;
  // CUDA graph of the whole constant-dt loop from it = 0 (captured once, replayed after edus_reset)
  bool use_graphs = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  long long graph_launches = 0;
  double2* d_Pinit = nullptr;
  double2 *P0_start = nullptr, *Pa_start = nullptr;
  struct HostClock {
    int it, nlog;
    double time_loop, dt;
    double EF[2][3];
    bool e_non0;
    int ring_idx[kMaxOrder];
    double2 *P0, *Pa;
    int icont;
    std::vector<double> snap_t;
    double vg_t, vg_A[3];
  } after_graph{};
};

namespace {

template <class T>
int dalloc(edus_ctx* c, T** p, size_t count) {
  void* v = nullptr;
  cudaError_t e = cudaMalloc(&v, sizeof(T) * (count ? count : 1));
  if (e != cudaSuccess) return fail(EDUS_ENOMEM, "cudaMalloc(%zu bytes): %s", sizeof(T) * count, cudaGetErrorString(e));
  c->allocs.push_back(v);
  c->dev_bytes += sizeof(T) * (count ? count : 1);
  *p = (T*)v;
  return 0;
}

// reference layout [k][n][n] -> upper-triangle planes [e][k]
void to_planes(const cd* src, int nk, int n, int comps, std::vector<double2>& dst) {
  int nt = n * (n + 1) / 2;
  dst.assign((size_t)comps * nt * nk, make_double2(0, 0));
  for (int k = 0; k < nk; k++)
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++)
        for (int x = 0; x < comps; x++) {
          cd v = src[(((size_t)k * n + i) * n + j) * comps + x];
          dst[((size_t)x * nt + tri_index(i, j, n)) * nk + k] = make_double2(v.real(), v.imag());
        }
}

int upload(edus_ctx* c, double2* d, const std::vector<double2>& h) {
  CK(cudaMemcpyAsync(d, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice, c->stream));
  return 0;
}

int state_to_dev(edus_ctx* c, const double* rho, double2* d) {
  std::vector<double2> pl;
  to_planes((const cd*)rho, c->nk, c->n, 1, pl);
  int rc = upload(c, d, pl);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int state_from_dev(edus_ctx* c, const double2* d, double* rho) {
  std::vector<double2> pl(c->plane);
  CK(cudaMemcpyAsync(pl.data(), d, sizeof(double2) * c->plane, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int n = c->n, nk = c->nk;
  cd* out = (cd*)rho;
  for (int k = 0; k < nk; k++)
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++) {
        double2 v = pl[(size_t)tri_index(i, j, n) * nk + k];
        out[((size_t)k * n + i) * n + j] = cd(v.x, v.y);
        if (i != j) out[((size_t)k * n + j) * n + i] = cd(v.x, -v.y);
      }
  return 0;
}

double2* slot_ptr(edus_ctx* c, int slot) {
  switch (slot) {
    case EDUS_SLOT_P0: return c->d_P0;
    case EDUS_SLOT_P1: return c->d_P1;
    case EDUS_SLOT_P2: return c->d_Pa;
    case EDUS_SLOT_PV: return c->d_Pb;
  }
  return nullptr;
}

StageArgs base_args(edus_ctx* c) {
  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.wx2 = c->P.p.probe.wl;
  a.order = c->order;
  a.dt = c->dt;
  a.xw = c->diagb ? c->d_xw : nullptr;
  return a;
}

// Per-kernel event timing (edus_profile): kind 0 = RHS + stage update, 1 = Coulomb transform pair.
int prof_mark(edus_ctx* c, int kind, bool begin) {
  if (!c->profiling) return 0;
  cudaEvent_t ev;
  CK(cudaEventCreate(&ev));
  CK(cudaEventRecord(ev, c->stream));
  if (begin)
    c->prof_open[kind] = ev;
  else
    c->prof_pairs.push_back({kind, c->prof_open[kind], ev, 1});
  return 0;
}

int run_coulomb(edus_ctx* c, const double2* src) {
  if (!c->coul) return 0;
  int rc = prof_mark(c, 1, true);
  if (rc) return rc;
  if (c->diagb) {
    // headers/RungeKutta.h:35-55: coefficients of the state in the eigenbasis,
    // then the screened term of that basis rotated back (:96-123)
    CK(launch_pdiag(c->tb, src, c->d_pdiag, c->stream));
    CK(launch_coulomb(c->tb, c->cd, c->d_pdiag, c->d_h, nullptr, c->d_X0, c->stream));
    CK(launch_coulomb_xw(c->tb, c->d_cst, c->d_pdiag, c->d_xw, c->stream));
    c->launches += 4;
  } else {
    CK(launch_coulomb(c->tb, c->cd, src, c->d_h, nullptr, c->d_X0, c->stream));
    c->launches += 2;
  }
  return prof_mark(c, 1, false);
}

int rhs(edus_ctx* c, StageArgs& a) {
  int rc = run_coulomb(c, a.src);
  if (rc) return rc;
  if ((rc = prof_mark(c, 0, true))) return rc;
  // profiling: repeat launches whose result does not depend on their own
  // output (Pv, the AB and Taylor updates: dst and the ring slot are written
  // from src and the older ring slots) to time the kernel back to back
  const bool idem = a.op == OP_PV || a.op == OP_AB || a.op == OP_TAYLOR;
  const int reps = (c->profiling && idem && a.dst != a.src) ? c->prof_reps : 1;
  for (int r = 0; r < reps; r++) {
    CK(launch_rhs(c->tb, c->d_cst, a, c->stream));
    c->launches++;
  }
  if ((rc = prof_mark(c, 0, false))) return rc;
  if (c->profiling) c->prof_pairs.back().reps = reps;
  return 0;
}

void set_ef(StageArgs& a, const double EF[2][3]) {
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 3; j++) a.EF[i][j] = EF[i][j];
}

int observe(edus_ctx* c) {
  edus_obs rec;
  memset(&rec, 0, sizeof(rec));
  rec.t = c->time_loop;
  for (int i = 0; i < 3; i++) {
    rec.EF_pump[i] = c->EF[0][i];
    rec.EF_probe[i] = c->EF[1][i];
  }
  rec.dt = c->dt;
  edus_obs* slot = nullptr;
  if (c->nlog < c->log_cap) slot = c->d_log + c->nlog;
  double scaleJ = c->P.dk[0] * c->P.dk[1] * c->P.dk[2] / c->P.det_a;
  double scaleTA = std::fabs(c->P.jac) * c->P.dk[0] * c->P.dk[1] * c->P.dk[2];
  // velocity gauge: the populations in the eigenbasis of H(k + A) and J1 from
  // the stencil gradient of H(k + A), as with a renormalised H
  const double2* hr = c->vg ? c->vga.H : (c->coul ? c->d_hr : nullptr);
  CK(launch_observables(c->tb, c->d_cst, c->d_P0, hr, c->P.p.current, c->P.p.tabs, c->d_part, c->d_done, scaleJ, scaleTA,
                        rec, slot, c->d_ncond, c->d_pcmax, c->stream));
  c->launches += 1;
  c->nlog++;
  return 0;
}

// Velocity gauge: A(t) = -int_t0^t E_pump dt by 4-point Gauss-Legendre panels of
// at most 0.5 a.u. from the tracked time (one panel per RK4 half step).
void vg_advance_A(edus_ctx* c, double t) {
  static const double gx[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
  static const double gw[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
  if (t < c->vg_t) {
    c->vg_t = c->P.t_start;
    c->vg_A[0] = c->vg_A[1] = c->vg_A[2] = 0.;
  }
  const int panels = (int)std::ceil((t - c->vg_t) / 0.5);
  const double t0 = c->vg_t;
  for (int q = 0; q < panels; q++) {
    const double a = t0 + (t - t0) * q / panels, b = t0 + (t - t0) * (q + 1) / panels;
    const double h = 0.5 * (b - a), m = 0.5 * (a + b);
    for (int g = 0; g < 4; g++) {
      double EF[2][3];
      field_at(c->P.p, m + h * gx[g], EF);
      for (int x = 0; x < 3; x++) c->vg_A[x] -= h * gw[g] * EF[0][x];
    }
  }
  c->vg_t = t;
}

// H, D at k + A(t) into the model tables (FP64 sums on CUDA cores, or the
// exact-slice GEMM on the tensor cores)
int vg_tables(edus_ctx* c, double t) {
  vg_advance_A(c, t);
  for (int i = 0; i < 3; i++) c->vga.A[i] = c->P.MI[i][0] * c->vg_A[0] + c->P.MI[i][1] * c->vg_A[1] + c->P.MI[i][2] * c->vg_A[2];
  if (c->vg_tc) {
    for (int i = 0; i < 3; i++) c->vgt.A[i] = c->vga.A[i];
    CK(batch::tc_vg_stage(c->vgt, c->stream));
    c->launches += 3;
  } else {
    CK(launch_vg_tables(c->vga, c->stream));
    c->launches++;
  }
  return 0;
}

bool want_hr(edus_ctx* c) { return c->coul && ((c->it + 1) % c->res == 0); }

// Source_Main/RungeKutta.cpp (one RK4 step)
int step_rk4(edus_ctx* c, bool startup_ring) {
  const double dt = c->dt, dt6 = dt / 6.0, dt3 = dt / 3.0, dt2 = dt / 2.0;
  const double t = c->time_loop;
  StageArgs a = base_args(c);
  // velocity gauge: no k-gradient term; H, D at k + A of each stage
  a.e_non0 = c->vg ? false : c->e_non0;
  field_at(c->P.p, t, c->EF);
  set_ef(a, c->EF);
  a.src = c->d_P0;
  a.base = c->d_P0;
  a.acc = c->d_P1;
  a.dst = c->d_Pa;
  a.op = OP_RK_FIRST;
  a.c1 = dt6;
  a.c2 = dt2;
  if (startup_ring) {
    a.ring = c->d_ring;
    for (int s = 0; s < c->order; s++) a.ring_idx[s] = c->ring_idx[s];
  }
  int rc = c->vg ? vg_tables(c, t) : 0;
  if (rc) return rc;
  if ((rc = rhs(c, a))) return rc;
  a.ring = nullptr;
  field_at(c->P.p, t + dt2, c->EF);
  if (c->vg && (rc = vg_tables(c, t + dt2))) return rc;
  set_ef(a, c->EF);
  a.src = c->d_Pa;
  a.dst = c->d_Pb;
  a.op = OP_RK_MID;
  a.c1 = dt3;
  a.c2 = dt2;
  if ((rc = rhs(c, a))) return rc;
  a.src = c->d_Pb;
  a.dst = c->d_Pa;
  a.c2 = dt;
  if ((rc = rhs(c, a))) return rc;
  field_at(c->P.p, t + dt, c->EF);
  if (c->vg && (rc = vg_tables(c, t + dt))) return rc;
  set_ef(a, c->EF);
  a.src = c->d_Pa;
  a.dst = c->d_P0;
  a.op = OP_RK_LAST;
  a.c1 = dt6;
  a.hr_out = want_hr(c) ? c->d_hr : nullptr;
  if (c->dyn) {
    CK(cudaMemsetAsync(c->d_maxdp, 0, sizeof(unsigned long long), c->stream));
    a.maxdp = c->d_maxdp;
    a.pcond_plus_ncond = c->P_cond_max + c->n_cond;
  }
  if ((rc = rhs(c, a))) return rc;
  c->e_non0 = field_nonzero(c->EF);
  return 0;
}

// Source_Main/Linear_Multistep_ODE_solvers.cpp:1-93
int step_ab(edus_ctx* c) {
  static const double cf[5][5] = {{1., 0, 0, 0, 0},
                                  {3.0 / 2.0, -1.0 / 2.0, 0, 0, 0},
                                  {23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0, 0, 0},
                                  {55.0 / 24.0, -59.0 / 24.0, 37.0 / 24.0, -9.0 / 24.0, 0},
                                  {1901.0 / 720.0, -2774.0 / 720.0, 2616.0 / 720.0, -1274.0 / 720.0, 251.0 / 720.0}};
  const int p = c->order;
  field_at(c->P.p, c->time_loop, c->EF);
  c->e_non0 = field_nonzero(c->EF);
  int fill = c->ring_idx[p - 1];
  for (int s = p - 1; s > 0; s--) c->ring_idx[s] = c->ring_idx[s - 1];
  c->ring_idx[0] = fill;
  bool startup = c->P.p.ab_rk4_startup && c->it < p - 1;
  if (startup) return step_rk4(c, true);
  StageArgs a = base_args(c);
  set_ef(a, c->EF);
  a.e_non0 = c->e_non0;
  a.src = c->d_P0;
  a.dst = c->d_Pa;
  a.op = OP_AB;
  a.ring = c->d_ring;
  a.dt = c->dt;
  for (int s = 0; s < p; s++) {
    a.ring_idx[s] = c->ring_idx[s];
    a.coef[s] = cf[p - 1][s];
  }
  a.hr_out = want_hr(c) ? c->d_hr : nullptr;
  int rc = rhs(c, a);
  if (rc) return rc;
  std::swap(c->d_P0, c->d_Pa);
  return 0;
}

// Source_Main/Taylor_DE_solver_deriv_Polynom.cpp:1-177
int step_taylor(edus_ctx* c) {
  const int TO = c->order, m = TO - 1;
  field_at(c->P.p, c->time_loop, c->EF);
  c->e_non0 = field_nonzero(c->EF);
  int fill = c->ring_idx[TO - 1];
  for (int s = TO - 1; s > 0; s--) c->ring_idx[s] = c->ring_idx[s - 1];
  c->ring_idx[0] = fill;
  StageArgs a = base_args(c);
  set_ef(a, c->EF);
  a.e_non0 = c->e_non0;
  a.src = c->d_P0;
  a.dst = c->d_Pa;
  a.op = OP_TAYLOR;
  a.ring = c->d_ring;
  a.dt = c->dt;
  for (int s = 0; s < TO; s++) a.ring_idx[s] = c->ring_idx[s];
  double ti[kMaxOrder], tau[kMaxOrder * kMaxOrder], tinv[kMaxOrder * kMaxOrder];
  ti[0] = c->dt_prev[0];
  for (int i = 1; i < m; i++) ti[i] = ti[i - 1] + c->dt_prev[i - 1];
  const double scale = std::pow(10, 7);
  for (int i = 0; i < m; i++)
    for (int q = 0; q < m; q++) tau[i * m + q] = scale * std::pow(ti[i], (q + 1));
  if (inv_gj(m, tau, tinv)) return fail(EDUS_EINVAL, "Taylor tau matrix is singular");
  for (int i = 0; i < m * m; i++) a.tinv[i] = tinv[i] * scale;
  for (int i = 0; i < TO; i++) a.tpow[i] = std::pow(c->dt, i + 1);
  a.hr_out = want_hr(c) ? c->d_hr : nullptr;
  if (c->dyn) {
    CK(cudaMemsetAsync(c->d_maxdp, 0, sizeof(unsigned long long), c->stream));
    a.maxdp = c->d_maxdp;
    a.pcond_plus_ncond = c->P_cond_max + c->n_cond;
  }
  int rc = rhs(c, a);
  if (rc) return rc;
  std::swap(c->d_P0, c->d_Pa);
  return 0;
}

int do_step(edus_ctx* c) {
  if (c->solver == EDUS_SOLVER_TAYLOR) return step_taylor(c);
  if (c->solver == EDUS_SOLVER_AB && !c->dyn) return step_ab(c);
  return step_rk4(c, false);
}

// Source_Main/dyn_dt_evolution.cpp:64-133
int adapt_dt(edus_ctx* c) {
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->d_maxdp, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double mx;
  memcpy(&mx, &bits, sizeof(mx));
  const double eps = c->P.p.eps_step_abs;
  if ((mx > eps) && (c->dt > 0.01))
    c->dt *= eps / mx;
  else if (c->dt < c->dt0)
    c->dt *= 1.02;
  if (c->solver == EDUS_SOLVER_TAYLOR) {
    for (int i = c->order - 1; i > 0; i--) c->dt_prev[i] = c->dt_prev[i - 1];
    c->dt_prev[0] = c->dt;
  }
  return 0;
}

int sync_scalars(edus_ctx* c) {
  double v[2];
  CK(cudaMemcpyAsync(&v[0], c->d_pcmax, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&v[1], c->d_ncond, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->P_cond_max = v[0];
  c->n_cond = v[1];
  return 0;
}

// Snapshot switch of an output step (Source_Main/if_resolution.cpp:18-33):
// a snapshot is due when t > start + icont * step and t < end (icont counted
// from -1); then icont advances and, with PrintPopulation, the state's
// eigenbasis elements go to slot icont (Source_Main/if_resolution.cpp:231-270).
int snapshot(edus_ctx* c) {
  const edus_params& p = c->P.p;
  if (!(c->time_loop > p.print_start + c->icont * p.print_step && c->time_loop < p.print_end)) return 0;
  c->icont++;
  c->snap_t.push_back(c->time_loop * kTimeAuFs);
  if (!c->d_snap && !c->d_edia) return 0;
  if (c->icont >= c->snap_cap) return fail(EDUS_EINVAL, "snapshot %d exceeds the %d slots", c->icont, c->snap_cap);
  if (c->d_snap) {
    CK(launch_snapshot(c->tb, c->d_P0, c->snap_ic, c->snap_jc, c->d_snap + (size_t)c->icont * 3 * c->nk, c->stream));
    c->launches++;
  }
  if (c->d_edia) {
    // the renormalised H of the last RHS evaluation, as the populations use it
    // (headers/Observables_MPI.h:282-303, 440-478)
    CK(launch_band_energies(c->tb, c->d_hr, c->d_edia + (size_t)c->icont * c->n * c->nk, c->stream));
    c->launches++;
  }
  return 0;
}

int run_steps(edus_ctx* c, int nsteps, bool all) {
  int done = 0;
  if (!c->dyn) {
    while (c->it <= c->itfi && (all || done < nsteps)) {
      if (c->it % c->res == 0) {
        int rc = observe(c);
        if (!rc && c->snap_on) rc = snapshot(c);
        if (rc) return rc;
      }
      int rc = do_step(c);
      if (rc) return rc;
      c->time_loop += c->dt;
      c->it++;
      done++;
    }
  } else {
    while (c->time_loop < c->P.p.t_fin && (all || done < nsteps)) {
      if (c->it % c->res == 0) {
        int rc = observe(c);
        if (rc) return rc;
        if ((rc = sync_scalars(c))) return rc;
        if (c->snap_on && (rc = snapshot(c))) return rc;
      }
      int rc = do_step(c);
      if (rc) return rc;
      if ((rc = adapt_dt(c))) return rc;
      c->time_loop += c->dt;
      c->it++;
      done++;
    }
  }
  return 0;
}

// ------------------------------------------------ adaptive step on the device
// A whole adaptive run (Source_Main/dyn_dt_evolution.cpp:1-183) as chunks of K
// captured steps: k_dyn_begin, the output instant where one can fall, the
// stages reading their scalars from the DynStep, k_dyn_end, and at the end of
// the chunk a copy of the active flag into pinned memory. K is a multiple of
// the Taylor ring's period (lcm(2, order): the ring slots rotate and the state
// buffers swap every step), so every chunk starts from the captured host
// state; with K also a multiple of it_resolution the instants sit at fixed
// steps of the chunk, else every step carries a (device-gated) instant.

bool dyn_on_device(const edus_ctx* c) {
  if (!c->dyn || !c->d_dyn || c->vg || c->profiling) return false;
  const char* e = std::getenv("EDUS_DYN_HOST");
  return !(e && std::string(e) == "1");
}

long long lcm_ll(long long a, long long b) {
  long long x = a, y = b;
  while (y) {
    const long long t = x % y;
    x = y;
    y = t;
  }
  return a / x * b;
}

int dyn_period(const edus_ctx* c) { return c->solver == EDUS_SOLVER_TAYLOR ? (int)lcm_ll(2, c->order) : 1; }

// chunk length; *every: an instant launch at every step of the chunk
int dyn_chunk_len(const edus_ctx* c, bool* every) {
  const long long P = dyn_period(c);
  const long long L = lcm_ll(c->res, P);
  if (L <= 512) {
    *every = false;
    return (int)(L * ((16 + L - 1) / L));
  }
  *every = true;
  return (int)(P * ((16 + P - 1) / P));
}

// One Taylor step's rotation of the ring slots (as step_taylor makes it).
void taylor_ring_rotate(edus_ctx* c) {
  const int TO = c->order;
  const int fill = c->ring_idx[TO - 1];
  for (int s = TO - 1; s > 0; s--) c->ring_idx[s] = c->ring_idx[s - 1];
  c->ring_idx[0] = fill;
}

int dyn_enqueue_chunk(edus_ctx* c, int K, bool every) {
  DynStep* d = c->d_dyn;
  const bool taylor = c->solver == EDUS_SOLVER_TAYLOR;
  double2* hr_out = c->coul ? c->d_hr : nullptr;  // every step: an instant reads the last one
  for (int j = 0; j < K; j++) {
    CK(launch_dyn_begin(d, c->stream));
    c->launches++;
    if (every || (c->it + j) % c->res == 0) {
      const double scaleJ = c->P.dk[0] * c->P.dk[1] * c->P.dk[2] / c->P.det_a;
      const double scaleTA = std::fabs(c->P.jac) * c->P.dk[0] * c->P.dk[1] * c->P.dk[2];
      edus_obs rec;
      memset(&rec, 0, sizeof(rec));
      CK(launch_observables(c->tb, c->d_cst, c->d_P0, c->coul ? c->d_hr : nullptr, c->P.p.current, c->P.p.tabs, c->d_part,
                            c->d_done, scaleJ, scaleTA, rec, c->d_log, c->d_ncond, c->d_pcmax, c->stream, d));
      c->launches++;
      if (c->snap_on && c->d_snap) {
        CK(launch_snapshot(c->tb, c->d_P0, c->snap_ic, c->snap_jc, c->d_snap, c->stream, d));
        c->launches++;
      }
      if (c->snap_on && c->d_edia) {
        CK(launch_band_energies(c->tb, c->d_hr, c->d_edia, c->stream, d));
        c->launches++;
      }
    }
    StageArgs a = base_args(c);
    a.dyn = d;
    a.hr_out = nullptr;
    int rc = 0;
    if (taylor) {
      taylor_ring_rotate(c);
      a.src = c->d_P0;
      a.dst = c->d_Pa;
      a.op = OP_TAYLOR;
      a.ring = c->d_ring;
      for (int q = 0; q < c->order; q++) a.ring_idx[q] = c->ring_idx[q];
      a.dyn_stage = 0;
      a.dyn_field = 0;
      a.hr_out = hr_out;
      a.maxdp = &d->maxdp;
      if ((rc = rhs(c, a))) return rc;
      std::swap(c->d_P0, c->d_Pa);
    } else {
      a.src = c->d_P0;
      a.base = c->d_P0;
      a.acc = c->d_P1;
      a.dst = c->d_Pa;
      a.op = OP_RK_FIRST;
      a.dyn_stage = 0;
      a.dyn_field = 0;
      if ((rc = rhs(c, a))) return rc;
      a.src = c->d_Pa;
      a.dst = c->d_Pb;
      a.op = OP_RK_MID;
      a.dyn_stage = 1;
      a.dyn_field = 1;
      if ((rc = rhs(c, a))) return rc;
      a.src = c->d_Pb;
      a.dst = c->d_Pa;
      a.dyn_stage = 2;
      if ((rc = rhs(c, a))) return rc;
      a.src = c->d_Pa;
      a.dst = c->d_P0;
      a.op = OP_RK_LAST;
      a.dyn_stage = 3;
      a.dyn_field = 2;
      a.hr_out = hr_out;
      a.maxdp = &d->maxdp;
      if ((rc = rhs(c, a))) return rc;
    }
    CK(launch_dyn_end(d, c->stream));
    c->launches++;
  }
  CK(cudaMemcpyAsync(c->h_active, &d->active, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  return 0;
}

int run_dyn_device(edus_ctx* c) {
  const edus_params& p = c->P.p;
  DynStep h;
  memset(&h, 0, sizeof(h));
  for (int i = 0; i < EDUS_MAX_PUMPS; i++) h.pump[i] = p.pump[i];
  h.probe = p.probe;
  h.n_pumps = p.n_pumps;
  h.taylor = c->solver == EDUS_SOLVER_TAYLOR;
  h.order = c->order;
  h.res = c->res;
  h.log_cap = c->log_cap;
  h.snap_on = c->snap_on;
  h.snap_cap = (c->d_snap || c->d_edia) ? c->snap_cap : 0;
  h.snap_tcap = c->snapt_cap;
  h.print_start = p.print_start;
  h.print_end = p.print_end;
  h.print_step = p.print_step;
  h.t_fin = p.t_fin;
  h.eps = p.eps_step_abs;
  h.dt0 = c->dt0;
  h.pcmax = c->d_pcmax;
  h.ncond = c->d_ncond;
  h.snap_t = c->d_snapt;
  h.t = c->time_loop;
  h.dt = c->dt;
  h.it = c->it;
  h.nlog = c->nlog;
  h.icont = c->icont;
  h.active = 1;
  h.e_non0 = c->e_non0;
  memcpy(h.EF_last, c->EF, sizeof(h.EF_last));
  memcpy(h.dt_prev, c->dt_prev, sizeof(h.dt_prev));
  h.snap_slot = -1;
  CK(cudaMemcpyAsync(c->d_dyn, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *c->h_active = 1;

  bool every = false;
  const int K = dyn_chunk_len(c, &every);
  const int phase = every ? 0 : c->it % c->res;
  const bool graphs = c->use_graphs;
  if (graphs && c->dyn_exec &&
      (c->dyn_K != K || c->dyn_phase != phase || c->dyn_P0 != c->d_P0 ||
       memcmp(c->dyn_ring, c->ring_idx, sizeof(c->dyn_ring)) != 0)) {
    cudaGraphExecDestroy(c->dyn_exec);
    cudaGraphDestroy(c->dyn_graph);
    c->dyn_exec = nullptr;
    c->dyn_graph = nullptr;
  }
  if (graphs && !c->dyn_exec) {
    c->dyn_K = K;
    c->dyn_phase = phase;
    c->dyn_P0 = c->d_P0;
    memcpy(c->dyn_ring, c->ring_idx, sizeof(c->dyn_ring));
    const long long l0 = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = dyn_enqueue_chunk(c, K, every);
    cudaGraph_t g = nullptr;
    cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    // the capture counted one chunk's kernels; they run at each replay
    c->dyn_chunk_launches = c->launches - l0;
    c->launches = l0;
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return fail(EDUS_ECUDA, "stream capture: %s", cudaGetErrorString(ec));
    c->dyn_graph = g;
    CK(cudaGraphInstantiate(&c->dyn_exec, g, 0));
  }
  for (int i = 0; i < 2; i++)
    if (!c->dyn_ev[i]) CK(cudaEventCreateWithFlags(&c->dyn_ev[i], cudaEventDisableTiming));

  // keep two chunks queued; stop once a finished chunk reports the run over
  const int it0 = c->it;
  const long long kMaxChunks = (1ll << 28) / K;
  long long chunks = 0;
  auto launch = [&]() -> int {
    if (graphs) {
      CK(cudaGraphLaunch(c->dyn_exec, c->stream));
      c->launches += c->dyn_chunk_launches;
    } else {
      int rc = dyn_enqueue_chunk(c, K, every);
      if (rc) return rc;
    }
    CK(cudaEventRecord(c->dyn_ev[chunks & 1], c->stream));
    chunks++;
    return 0;
  };
  int rc = launch();
  if (rc) return rc;
  for (;;) {
    if ((rc = launch())) return rc;
    CK(cudaEventSynchronize(c->dyn_ev[(chunks - 2) & 1]));
    if (!*(volatile int*)c->h_active) break;
    if (chunks > kMaxChunks) return fail(EDUS_EINVAL, "adaptive run: more than 2^28 steps");
  }
  CK(cudaMemcpyAsync(&h, c->d_dyn, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));

  // the host mirror after the run
  const int icont0 = c->icont;
  c->time_loop = h.t;
  c->dt = h.dt;
  c->it = h.it;
  c->nlog = h.nlog;
  c->icont = h.icont;
  c->e_non0 = h.e_non0 != 0;
  memcpy(c->EF, h.EF_last, sizeof(c->EF));
  memcpy(c->dt_prev, h.dt_prev, sizeof(c->dt_prev));
  if (c->solver == EDUS_SOLVER_TAYLOR)
    for (int s = 0; s < (c->it - it0) % dyn_period(c); s++) {
      taylor_ring_rotate(c);
      std::swap(c->d_P0, c->d_Pa);
    }
  if (h.icont > icont0 && c->d_snapt) {
    const int first = icont0 + 1, last = std::min(h.icont, c->snapt_cap - 1);
    if (last >= first) {
      std::vector<double> ts((size_t)(last - first + 1));
      CK(cudaMemcpy(ts.data(), c->d_snapt + first, sizeof(double) * ts.size(), cudaMemcpyDeviceToHost));
      for (double t : ts) c->snap_t.push_back(t);
    }
  }
  if ((rc = sync_scalars(c))) return rc;
  if (h.fault == kDynFaultSnapshots) return fail(EDUS_EINVAL, "snapshot %d exceeds the %d slots", h.icont, c->snap_cap);
  if (h.fault == kDynFaultTaylor) return fail(EDUS_EINVAL, "Taylor tau matrix is singular");
  return 0;
}

// Enqueue nsteps (or the whole run) between the context's two timing events;
// *l0 receives the launch count before them. timed_finish waits for the end
// event and checks the device error word.
int timed_start(edus_ctx* c, int nsteps, bool all, long long* l0_out) {
  CK(cudaSetDevice(c->device));
  long long l0 = c->launches;
  *l0_out = l0;
  if (all && dyn_on_device(c)) {
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = run_dyn_device(c);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    return 0;
  }
  const bool graph = all && !c->dyn && c->use_graphs && c->it == 0;
  if (graph && !c->gexec) {
    // capture the whole loop once; the captured kernels run at cudaGraphLaunch below
    c->P0_start = c->d_P0;
    c->Pa_start = c->d_Pa;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = run_steps(c, nsteps, all);
    cudaGraph_t g = nullptr;
    cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return fail(EDUS_ECUDA, "stream capture: %s", cudaGetErrorString(ec));
    c->graph = g;
    CK(cudaGraphInstantiate(&c->gexec, g, 0));
    c->graph_launches = c->launches - l0;
    auto& h = c->after_graph;
    h.it = c->it;
    h.nlog = c->nlog;
    h.time_loop = c->time_loop;
    h.dt = c->dt;
    memcpy(h.EF, c->EF, sizeof(h.EF));
    h.e_non0 = c->e_non0;
    memcpy(h.ring_idx, c->ring_idx, sizeof(h.ring_idx));
    h.P0 = c->d_P0;
    h.Pa = c->d_Pa;
    h.icont = c->icont;
    h.snap_t = c->snap_t;
    h.vg_t = c->vg_t;
    memcpy(h.vg_A, c->vg_A, sizeof(h.vg_A));
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(cudaGraphLaunch(c->gexec, c->stream));
  } else if (graph) {
    // replay from the state edus_reset restored; advance the host clock as the capture did
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(cudaGraphLaunch(c->gexec, c->stream));
    c->launches += c->graph_launches;
    const auto& h = c->after_graph;
    c->it = h.it;
    c->nlog = h.nlog;
    c->time_loop = h.time_loop;
    c->dt = h.dt;
    memcpy(c->EF, h.EF, sizeof(h.EF));
    c->e_non0 = h.e_non0;
    memcpy(c->ring_idx, h.ring_idx, sizeof(h.ring_idx));
    c->d_P0 = h.P0;
    c->d_Pa = h.Pa;
    c->icont = h.icont;
    c->snap_t = h.snap_t;
    c->vg_t = h.vg_t;
    memcpy(c->vg_A, h.vg_A, sizeof(c->vg_A));
  } else {
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = run_steps(c, nsteps, all);
    if (rc) return rc;
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  return 0;
}

int timed_finish(edus_ctx* c, long long l0) {
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  c->last_launches = c->launches - l0;
  int derr = 0;
  CK(cudaMemcpy(&derr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (derr) return fail(EDUS_ETIMEOUT, "a bounded device wait ran out (error word %d)", derr);
  CK(cudaGetLastError());
  return 0;
}

int timed(edus_ctx* c, int nsteps, bool all) {
  long long l0 = 0;
  int rc = timed_start(c, nsteps, all, &l0);
  if (rc) return rc;
  return timed_finish(c, l0);
}

}  // namespace

// ------------------------------------------------------------ bounded-wait self-test
namespace edus {
namespace selftest {

// One thread initialises an mbarrier expecting one arrival that nothing makes
// (no bulk copy is issued) and waits on it with the kernels' bounded wait, cut
// to `iters` polls: the wait runs out, records the timeout in *err and the
// kernel returns.
__global__ void k_wait_selftest(int* err, int iters) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  mbar_wait(&bar, 0, err, iters);
}

}  // namespace selftest
}  // namespace edus

extern "C" int edus_selftest_bounded_wait(int32_t device, int32_t iters) {
  if (iters < 1 || iters > (1 << 20)) return fail(EDUS_EINVAL, "iters must be in [1, 2^20]");
  CK(cudaSetDevice(device));
  int* err = nullptr;
  CK(cudaMalloc(&err, sizeof(int)));
  int h = 0;
  cudaError_t e = cudaMemset(err, 0, sizeof(int));
  if (e == cudaSuccess) {
    edus::selftest::k_wait_selftest<<<1, 32>>>(err, iters);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(err);
  if (e != cudaSuccess) return fail(EDUS_ECUDA, "bounded-wait self-test: %s", cudaGetErrorString(e));
  if (h == kErrTimeout) return fail(EDUS_ETIMEOUT, "a bounded device wait ran out after %d polls (self-test)", iters);
  return 0;
}

// ------------------------------------------------------------ batch hooks
// A batch runs an instance with the Coulomb mean field as a context of its
// own: the whole loop, captured in one CUDA graph as edus_run replays it, is
// launched on the context's stream and runs beside the batch's chunk graphs.
namespace edus {

int ctx_start_async(edus_ctx* c) {
  if (!c) return fail(EDUS_EINVAL, "null argument");
  if (c->dyn || !c->use_graphs || c->it != 0)
    return fail(EDUS_EUNSUPPORTED, "an asynchronous whole run needs a fresh context at constant dt with graphs");
  return timed_start(c, 0, true, &c->async_l0);
}

int ctx_poll(edus_ctx* c, bool* done) {
  if (!c || !done) return fail(EDUS_EINVAL, "null argument");
  CK(cudaSetDevice(c->device));
  cudaError_t e = cudaEventQuery(c->ev1);
  if (e == cudaErrorNotReady) {
    *done = false;
    return 0;
  }
  if (e != cudaSuccess) return fail(EDUS_ECUDA, "context run: %s", cudaGetErrorString(e));
  *done = true;
  return timed_finish(c, c->async_l0);
}

int ctx_wait(edus_ctx* c) {
  if (!c) return fail(EDUS_EINVAL, "null argument");
  CK(cudaSetDevice(c->device));
  return timed_finish(c, c->async_l0);
}

size_t ctx_device_bytes(const edus_ctx* c) { return c ? c->dev_bytes : 0; }

double ctx_last_ms(const edus_ctx* c) { return c ? c->last_ms : 0.0; }

// Upper bound of the device memory edus_create takes for a problem: the
// state, table and ring planes, the observable log, the Coulomb scratch and
// the snapshot slots, with a margin.
int64_t ctx_footprint_estimate(const Problem& P) {
  const double n = P.ncv, nk = P.nk, nt = n * (n + 1) / 2, plane = 16.0 * nt * nk;
  const int order = P.p.solver == EDUS_SOLVER_RK4 ? 0 : P.p.order;
  double b = plane * (1 + 3 + 3 + 4 + 1 + order) + 16.0 * n * n * nk + 4.0 * P.nnb * nk;
  b += (double)(P.nprint + 2) * sizeof(edus_obs) + (double)obs_parts(P.nk) * obs_part_bytes();
  if (P.p.coulomb) {
    const double nc = P.ncut, side = std::max(P.n1, P.n2);
    b += plane * 2 + 16.0 * 4 * nc * nc * n * n * 3 + 16.0 * 4 * nc * side * nt * 2 + 8.0 * 4 * nc * side;
  }
  return (int64_t)(1.25 * b) + (1 << 20);
}

}  // namespace edus

// =================================================================== C ABI

extern "C" {

const char* edus_strerror(int code) {
  switch (code) {
    case EDUS_OK: return "ok";
    case EDUS_EINVAL: return "invalid argument";
    case EDUS_ENOMEM: return "out of memory (host, HBM or HBM budget)";
    case EDUS_ECUDA: return "CUDA error";
    case EDUS_ENONFINITE: return "non-finite density matrix";
    case EDUS_ETRACE: return "trace drift above tolerance";
    case EDUS_ETIMEOUT: return "device wait timed out";
    case EDUS_ECANCELLED: return "cancelled";
    case EDUS_EIO: return "file could not be read or written";
    case EDUS_EPARSE: return "input.txt grammar error";
    case EDUS_EUNSUPPORTED: return "option not built";
    case EDUS_ENOTREADY: return "result not ready";
  }
  return "unknown error";
}

int edus_abi_version(void) { return EDUS_ABI_VERSION; }

int edus_options_default(edus_options* o) {
  if (!o) return EDUS_EINVAL;
  memset(o, 0, sizeof(*o));
  o->device = 0;
  o->precision = -1;
  o->use_graphs = 1;
  o->health_checks = 0;
  o->trace_tol = 1e-6;
  o->hbm_budget_bytes = 0;
  return 0;
}

int edus_problem_create(const edus_params* p, const char* workdir, edus_problem** out) {
  clear_error();
  if (!p || !out) return fail(EDUS_EINVAL, "null argument");
  edus_problem* pb = new (std::nothrow) edus_problem();
  if (!pb) return fail(EDUS_ENOMEM, "host allocation");
  int rc = build_problem(*p, workdir, pb->P);
  if (rc) {
    delete pb;
    return rc;
  }
  *out = pb;
  return 0;
}

int edus_problem_create_deferred(const edus_params* p, const char* workdir, edus_problem** out) {
  clear_error();
  if (!p || !out) return fail(EDUS_EINVAL, "null argument");
  edus_problem* pb = new (std::nothrow) edus_problem();
  if (!pb) return fail(EDUS_ENOMEM, "host allocation");
  int rc = build_problem(*p, workdir, pb->P, true);
  if (rc) {
    delete pb;
    return rc;
  }
  *out = pb;
  return 0;
}

int edus_problem_drop_decoupled_core(edus_problem* pb) {
  if (!pb) return fail(EDUS_EINVAL, "null argument");
  return drop_decoupled_core(pb->P);
}

int edus_problem_info_get(const edus_problem* pb, edus_problem_info* o) {
  if (!pb || !o) return fail(EDUS_EINVAL, "null argument");
  const Problem& P = pb->P;
  memset(o, 0, sizeof(*o));
  o->ncv = P.ncv;
  o->nch = P.nch;
  o->nv = P.nv;
  o->nc = P.nc;
  o->nk = P.nk;
  o->n1 = P.n1;
  o->n2 = P.n2;
  o->nshell = P.nshell;
  o->nnb = P.nnb;
  o->nrpts = P.nrpts;
  o->n_diss = (int)P.diss_i.size();
  o->nsteps = P.nsteps;
  o->nprint = P.nprint;
  o->t_start = P.t_start;
  o->det_a = P.det_a;
  o->jacobian = P.jac;
  for (int i = 0; i < 3; i++) o->dk[i] = P.dk[i];
  return 0;
}

int edus_problem_get(const edus_problem* pb, const char* name, void* dst, size_t nbytes) {
  if (!pb || !name || !dst) return fail(EDUS_EINVAL, "null argument");
  const Problem& P = pb->P;
  const void* src = nullptr;
  size_t nb = 0;
  std::vector<double> wtmp;
  std::string s = name;
  if (s == "kpt") {
    src = P.kpt.data();
    nb = P.kpt.size() * sizeof(double);
  } else if (s == "H") {
    src = P.H.data();
    nb = P.H.size() * sizeof(cd);
  } else if (s == "U") {
    src = P.U.data();
    nb = P.U.size() * sizeof(cd);
  } else if (s == "D") {
    src = P.D.data();
    nb = P.D.size() * sizeof(cd);
  } else if (s == "GE") {
    src = P.GE.data();
    nb = P.GE.size() * sizeof(cd);
  } else if (s == "P0") {
    src = P.P0.data();
    nb = P.P0.size() * sizeof(cd);
  } else if (s == "nbr") {
    src = P.nbr.data();
    nb = P.nbr.size() * sizeof(int);
  } else if (s == "bvec") {
    src = P.bvec.data();
    nb = P.bvec.size() * sizeof(double);
  } else if (s == "weights") {
    for (int b = 0; b < P.nnb; b++) wtmp.push_back(P.shell_w[P.bshell[b]]);
    src = wtmp.data();
    nb = wtmp.size() * sizeof(double);
  } else if (s == "T") {
    src = P.T;
    nb = sizeof(P.T);
  } else if (s == "HR") {
    src = P.HR.data();
    nb = P.HR.size() * sizeof(cd);
  } else if (s == "rR") {
    src = P.rR.data();
    nb = P.rR.size() * sizeof(cd);
  } else if (s == "Rvec") {
    src = P.Rvec.data();
    nb = P.Rvec.size() * sizeof(double);
  } else {
    return fail(EDUS_EINVAL, "unknown array %s", name);
  }
  if (nb != nbytes) return fail(EDUS_EINVAL, "%s has %zu bytes, caller asked for %zu", name, nb, nbytes);
  memcpy(dst, src, nb);
  return 0;
}

void edus_problem_free(edus_problem* pb) { delete pb; }

}  // extern "C"

namespace {

// Output/k_grid.txt: the crystal coordinates of every k point in grid order,
// one "k0 k1 k2" line each with the default stream format, as the reference
// writes it at its first output step (headers/Observables_MPI.h:492-550,
// called from Source_Main/if_resolution.cpp:100-102).
int write_kgrid(const Problem& P, const char* outdir) {
  mkdir(outdir, 0755);
  std::ofstream f(std::string(outdir) + "/k_grid.txt");
  if (!f) return fail(EDUS_EIO, "cannot write into %s", outdir);
  const std::vector<double>& k = P.kpt;
  for (size_t ik = 0; ik + 2 < k.size(); ik += 3) f << k[ik] << " " << k[ik + 1] << " " << k[ik + 2] << std::endl;
  return f ? 0 : fail(EDUS_EIO, "write error in %s/k_grid.txt", outdir);
}

// Print order of the per-k files: the rows of the grid (nk_x consecutive k
// points) sorted by their first k point's coordinate along the row axis, the
// first of equal values first (Create_sorted_indices_k_MPI and find_index_min,
// headers/Observables_MPI.h:600-660; the reordering of Print_vec3x_MPI,
// :44-62). Returns the source k of every printed line.
std::vector<int> print_order(const Problem& P) {
  const int* Nk = P.p.nk;
  const int nk = P.nk;
  int pol = 1, nk_x = Nk[1] * Nk[0];
  if (Nk[1] > Nk[2]) {
    pol = 0;
    nk_x = Nk[1] * Nk[2];
  }
  const int nk_y = nk / nk_x;
  std::vector<double> kt(nk_y, 0.0);
  for (int ik = 0; ik < nk; ik++)
    if (ik % nk_x == 0 && ik / nk_x < nk_y) kt[ik / nk_x] = P.kpt[(size_t)ik * 3 + pol];
  std::vector<int> idx(nk_y);
  for (int r = 0; r < nk_y; r++) {
    int m = 0;
    double mv = 1e15;
    for (int q = 0; q < nk_y; q++)
      if (kt[q] < mv) {
        mv = kt[q];
        m = q;
      }
    kt[m] = 1e15;
    idx[r] = m;
  }
  std::vector<int> order(nk);
  for (int ik = 0; ik < nk; ik++) {
    const int ikx = ik / nk_x, iky = ik % nk_x;
    order[ik] = ikx < nk_y ? idx[ikx] * nk_x + iky : ik;
  }
  return order;
}

// Output/t_Ek.txt (time of every snapshot, fs), with the Coulomb mean field
// Edia_<m>.txt, and with PrintPopulation the
// three per-k files of every snapshot m: P_val_cond_in_Eigenstate_<v><c>_<m>,
// P_val_in_Eigenstate_<v><v>_<m>, P_cond_in_Eigenstate_<c><c>_<m>, one "re im"
// line per k (Source_Main/if_resolution.cpp:18-33, 231-270, Source_Main/
// open_files.cpp:57-63, headers/Observables_MPI.h:3-130).
int write_snapshots(edus_ctx* c, const std::string& d) {
  std::ofstream ft(d + "/t_Ek.txt");
  if (!ft) return fail(EDUS_EIO, "cannot write into %s", d.c_str());
  for (double t : c->snap_t) ft << t << std::endl;
  const int nk = c->nk, nsnap = std::min(c->icont + 1, c->snap_cap);
  if (c->d_edia) {
    // Output/Edia_<m>.txt: the band energies of every k in grid order, 20 digits
    std::vector<double> e((size_t)c->n * nk);
    for (int m = 0; m < nsnap; m++) {
      CK(cudaMemcpy(e.data(), c->d_edia + (size_t)m * c->n * nk, sizeof(double) * e.size(), cudaMemcpyDeviceToHost));
      std::ostringstream name;
      name << d << "/Edia_" << m << ".txt";
      std::ofstream f(name.str());
      if (!f) return fail(EDUS_EIO, "cannot write %s", name.str().c_str());
      for (int ik = 0; ik < nk; ik++) {
        for (int i = 0; i < c->n; i++) f << std::setprecision(20) << e[(size_t)i * nk + ik] << " ";
        f << std::endl;
      }
    }
  }
  if (!c->d_snap) return 0;
  const std::vector<int> order = print_order(c->P);
  std::vector<double2> buf((size_t)3 * nk);
  const char* label[3] = {"P_val_cond_in_Eigenstate", "P_val_in_Eigenstate", "P_cond_in_Eigenstate"};
  const int ii[3] = {c->snap_ic, c->snap_ic, c->snap_jc}, jj[3] = {c->snap_jc, c->snap_ic, c->snap_jc};
  for (int m = 0; m < nsnap; m++) {
    CK(cudaMemcpy(buf.data(), c->d_snap + (size_t)m * 3 * nk, sizeof(double2) * buf.size(), cudaMemcpyDeviceToHost));
    for (int q = 0; q < 3; q++) {
      std::ostringstream name;
      name << d << "/" << label[q] << "_" << ii[q] << jj[q] << "_" << m << ".txt";
      std::ofstream f(name.str());
      if (!f) return fail(EDUS_EIO, "cannot write %s", name.str().c_str());
      for (int ik = 0; ik < nk; ik++) {
        const double2 v = buf[(size_t)q * nk + order[ik]];
        f << v.x << " ";
        f << v.y << std::endl;
      }
    }
  }
  return 0;
}

// The files the reference writes once, at its first output step
// (Print_initial_H_P, Source_Main/if_resolution.cpp:275-328), one "re im" line
// per k in print order, v / c the top valence and bottom conduction band:
// H_Eigen_{cond,val,val_cond} (eigenvalues of the model H on the diagonal,
// zero elsewhere: Diagonalize_unitary_vec3x, headers/InitialPopulation.h:45-96),
// H_Wannier_cond (model H), P_initial_Wannier_ (the initial state) and Uk_
// (elements cc and cv of U), named <label>_<i><j>_0.txt.
int write_initial(edus_ctx* c, const std::string& d) {
  const int n = c->n, nk = c->nk, v = c->P.nbands - 1, cb = c->P.nbands;
  if (v < 0 || cb >= n) return 0;
  auto tri = [n](int i, int j) { return i * n - (i * (i - 1)) / 2 + (j - i); };
  std::vector<double> eps((size_t)n * nk);
  {
    double* d_eps = nullptr;
    CK(cudaMalloc(&d_eps, sizeof(double) * eps.size()));
    cudaError_t e = launch_band_energies(c->tb, c->tb.H, d_eps, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(eps.data(), d_eps, sizeof(double) * eps.size(), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_eps);
    CK(e);
  }
  auto plane = [&](const double2* src, std::vector<double2>& out) -> int {
    out.resize(nk);
    CK(cudaMemcpy(out.data(), src, sizeof(double2) * nk, cudaMemcpyDeviceToHost));
    return 0;
  };
  std::vector<double2> hcc, pcc, ucc, ucv;
  int rc;
  if ((rc = plane(c->tb.H + (size_t)tri(cb, cb) * nk, hcc)) || (rc = plane(c->d_Pinit + (size_t)tri(cb, cb) * nk, pcc)) ||
      (rc = plane(c->tb.U + (size_t)(cb * n + cb) * nk, ucc)) || (rc = plane(c->tb.U + (size_t)(cb * n + v) * nk, ucv)))
    return rc;
  const std::vector<int> order = print_order(c->P);
  struct Out {
    const char* label;
    int i, j;
    std::function<double2(int)> at;
  };
  const Out files[] = {
      {"H_Eigen_cond", cb, cb, [&](int k) { return make_double2(eps[(size_t)cb * nk + k], 0.0); }},
      {"H_Eigen_val", v, v, [&](int k) { return make_double2(eps[(size_t)v * nk + k], 0.0); }},
      {"H_Eigen_val_cond", v, cb, [&](int) { return make_double2(0.0, 0.0); }},
      {"H_Wannier_cond", cb, cb, [&](int k) { return hcc[k]; }},
      {"P_initial_Wannier_", cb, cb, [&](int k) { return pcc[k]; }},
      {"Uk_", cb, cb, [&](int k) { return ucc[k]; }},
      {"Uk_", cb, v, [&](int k) { return ucv[k]; }},
  };
  for (const Out& o : files) {
    std::ostringstream name;
    name << d << "/" << o.label << "_" << o.i << o.j << "_0.txt";
    std::ofstream f(name.str());
    if (!f) return fail(EDUS_EIO, "cannot write %s", name.str().c_str());
    for (int ik = 0; ik < nk; ik++) {
      const double2 x = o.at(order[ik]);
      f << x.x << " ";
      f << x.y << std::endl;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int edus_problem_write_kgrid(const edus_problem* pb, const char* outdir) {
  if (!pb || !outdir) return fail(EDUS_EINVAL, "null argument");
  return write_kgrid(pb->P, outdir);
}

// <workdir>/Test_matrices.txt: H, U, U H U^dagger, U U^dagger and the dipoles
// of the model at crystal k = (0, 0.3, 0.1), printed as the reference's
// set-up prints them (Source_Main/test_matrix_k.cpp:1-105).
int edus_problem_write_test_matrices(const edus_problem* pb, const char* workdir) {
  if (!pb || !workdir) return fail(EDUS_EINVAL, "null argument");
  const Problem& P = pb->P;
  const int n = P.ncv;
  const double k[3] = {0, 0.3, 0.1};
  std::vector<cd> H((size_t)n * n), U((size_t)n * n), D((size_t)n * n * 3);
  int rc = model_hud(P, k, H.data(), U.data(), D.data());
  if (rc) return rc;
  std::ofstream t(std::string(workdir) + "/Test_matrices.txt");
  if (!t) return fail(EDUS_EIO, "cannot write into %s", workdir);
  auto h = [&](int i, int j) { return H[(size_t)i * n + j]; };
  auto u = [&](int i, int j) { return U[(size_t)i * n + j]; };
  t << "k = " << k[0] << " " << k[1] << " " << k[2] << std::endl;
  t << "Energy: \n";
  for (int ic = 0; ic < n; ic++) {
    for (int jc = 0; jc < n; jc++) t << h(ic, jc) << " ";
    t << "\n";
  }
  t << "\n";
  t << "Unitary: \n";
  for (int ic = 0; ic < n; ic++) {
    for (int jc = 0; jc < n; jc++) t << u(ic, jc) << " ";
    t << "\n";
  }
  t << "\n";
  t << "U E_W U_dagger (to compare with eq. 104 in notes).\n";
  for (int ic = 0; ic < n; ic++) {
    for (int jc = 0; jc < n; jc++) {
      cd e2 = 0.;
      for (int mc = 0; mc < n; mc++)
        for (int nc = 0; nc < n; nc++) e2 += u(ic, mc) * h(mc, nc) * std::conj(u(jc, nc));
      t << e2 << " ";
    }
    t << "\n";
  }
  t << "U  U_dagger (should be 1).\n";
  for (int ic = 0; ic < n; ic++) {
    for (int jc = 0; jc < n; jc++) {
      cd e2 = 0.;
      for (int mc = 0; mc < n; mc++) e2 += u(ic, mc) * std::conj(u(jc, mc));
      t << e2 << " ";
      if (std::abs(e2) > 1e-10 && ic != jc) t << "ERROR" << " ";
      if (std::abs(e2 - 1.) > 1e-10 && ic == jc) t << "ERROR" << " ";
    }
    t << "\n";
  }
  t << "\n";
  const char* lab[3] = {"dx: \n", "dy: \n", "dz: \n"};
  for (int x = 0; x < 3; x++) {
    t << lab[x];
    for (int ic = 0; ic < n; ic++) {
      for (int jc = 0; jc < n; jc++) t << D[((size_t)ic * n + jc) * 3 + x] << " ";
      t << "\n";
    }
    t << "\n";
  }
  return t ? 0 : fail(EDUS_EIO, "write error in %s/Test_matrices.txt", workdir);
}

// <workdir>/kpt.txt: "ik i0 i1 i2 k0 k1 k2" per k point of the Monkhorst-Pack
// grid, default stream format, as BZ_parameters writes it while it builds the
// grid (headers/InitParameters.h:17-39).
int edus_problem_write_kpt(const edus_problem* pb, const char* workdir) {
  if (!pb || !workdir) return fail(EDUS_EINVAL, "null argument");
  const Problem& P = pb->P;
  if (P.p.kpt_read) return 0;  // the reference writes it only for its own grid
  std::ofstream f(std::string(workdir) + "/kpt.txt");
  if (!f) return fail(EDUS_EIO, "cannot write into %s", workdir);
  const int* Nk = P.p.nk;
  for (int ik = 0; ik < P.nk; ik++) {
    const int iik[3] = {(ik / (Nk[2] * Nk[1])) % Nk[0], (ik / Nk[2]) % Nk[1], ik % Nk[2]};
    f << ik << " " << iik[0] << " " << iik[1] << " " << iik[2];
    for (int c = 0; c < 3; c++) f << " " << P.kpt[(size_t)ik * 3 + c];
    f << std::endl;
  }
  return f ? 0 : fail(EDUS_EIO, "write error in %s/kpt.txt", workdir);
}

int edus_model_hud(const edus_problem* pb, const double kcrys[3], double* H, double* U, double* D) {
  if (!pb || !kcrys || !H || !U || !D) return fail(EDUS_EINVAL, "null argument");
  return model_hud(pb->P, kcrys, (cd*)H, (cd*)U, (cd*)D);
}

int edus_struct_sizes(int64_t out[4]) {
  if (!out) return fail(EDUS_EINVAL, "null argument");
  out[0] = sizeof(edus_params);
  out[1] = sizeof(edus_obs);
  out[2] = sizeof(edus_problem_info);
  out[3] = sizeof(edus_options);
  return 0;
}

void edus_destroy(edus_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void* p : c->allocs) cudaFree(p);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  if (c->dyn_exec) cudaGraphExecDestroy(c->dyn_exec);
  if (c->dyn_graph) cudaGraphDestroy(c->dyn_graph);
  for (cudaEvent_t e : c->dyn_ev)
    if (e) cudaEventDestroy(e);
  if (c->h_active) cudaFreeHost(c->h_active);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int edus_create(const edus_problem* pb, const edus_options* opt, edus_ctx** out) {
  clear_error();
  if (!pb || !out) return fail(EDUS_EINVAL, "null argument");
  if (pb->P.model_deferred)
    return fail(EDUS_EUNSUPPORTED, "the problem's model is tabulated on the device only in batches (edus_problem_create)");
  edus_options o;
  edus_options_default(&o);
  if (opt) o = *opt;
  edus_ctx* c = new (std::nothrow) edus_ctx();
  if (!c) return fail(EDUS_ENOMEM, "host allocation");
  c->P = pb->P;
  const Problem& P = c->P;
  c->device = o.device;
  int rc = 0;
  auto bail = [&](int code) {
    edus_destroy(c);
    return code;
  };
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bail(fail(EDUS_ECUDA, "no CUDA device"));
  if (cudaSetDevice(c->device) != cudaSuccess) return bail(fail(EDUS_ECUDA, "cannot select device %d", c->device));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(EDUS_ECUDA, "stream"));
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  const int n = P.ncv, nk = P.nk, nt = n * (n + 1) / 2;
  c->n = n;
  c->ntri = nt;
  c->nk = nk;
  c->plane = (size_t)nt * nk;
  if (n != 1 && n != 2 && n != 3 && n != 4 && n != 5 && n != 8 && n != 16)
    return bail(fail(EDUS_EUNSUPPORTED, "band count %d has no FP64 kernel instance (1-5, 8, 16)", n));
  if (P.nnb > kMaxNb) return bail(fail(EDUS_EUNSUPPORTED, "stencil with %d neighbours (max %d)", P.nnb, kMaxNb));
  c->solver = P.p.solver;
  c->order = P.p.solver == EDUS_SOLVER_RK4 ? 0 : P.p.order;
  if (c->order > kMaxOrder) return bail(fail(EDUS_EINVAL, "order %d > %d", c->order, kMaxOrder));
  if (P.p.ab_rk4_startup && P.p.solver == EDUS_SOLVER_AB && c->order < 1) return bail(fail(EDUS_EINVAL, "AB order"));
  c->dyn = P.p.dynamical_dt != 0;
  c->coul = P.p.coulomb != 0;
  c->res = P.p.it_resolution > 0 ? P.p.it_resolution : 1;
  // dipoles are stored as upper triangles: symmetric ones (Wannier and
  // tight-binding models) or Hermitian ones (the Crystal interface)
  const bool herm = P.p.mode == EDUS_MODE_CRYSTAL;
  for (int k = 0; k < nk; k++)
    for (int i = 0; i < n; i++)
      for (int j = i + (herm ? 0 : 1); j < n; j++)
        for (int x = 0; x < 3; x++) {
          const cd u = P.D[(((size_t)k * n + i) * n + j) * 3 + x], l = P.D[(((size_t)k * n + j) * n + i) * 3 + x];
          if (herm ? (l != std::conj(u)) : (l != u))
            return bail(fail(EDUS_EUNSUPPORTED, "dipole matrix is not %s at k=%d (%d,%d)", herm ? "Hermitian" : "symmetric", k, i, j));
        }
  // ---- device tables
  std::vector<double2> pl;
  double2 *dH, *dD, *dU = nullptr, *dGE = nullptr;
  int* dnbr;
  if ((rc = dalloc(c, &dH, c->plane)) || (rc = dalloc(c, &dD, 3 * c->plane)) || (rc = dalloc(c, &dnbr, (size_t)P.nnb * nk)))
    return bail(rc);
  to_planes(P.H.data(), nk, n, 1, pl);
  if ((rc = upload(c, dH, pl))) return bail(rc);
  to_planes(P.D.data(), nk, n, 3, pl);
  if ((rc = upload(c, dD, pl))) return bail(rc);
  {
    std::vector<double2> u((size_t)n * n * nk);
    for (int k = 0; k < nk; k++)
      for (int e = 0; e < n * n; e++) {
        cd v = P.U[(size_t)k * n * n + e];
        u[(size_t)e * nk + k] = make_double2(v.real(), v.imag());
      }
    if ((rc = dalloc(c, &dU, u.size())) || (rc = upload(c, dU, u))) return bail(rc);
  }
  if (P.p.current && !c->coul) {
    to_planes(P.GE.data(), nk, n, 3, pl);
    if ((rc = dalloc(c, &dGE, pl.size())) || (rc = upload(c, dGE, pl))) return bail(rc);
  }
  {
    std::vector<int> nb((size_t)P.nnb * nk);
    for (int k = 0; k < nk; k++)
      for (int b = 0; b < P.nnb; b++) nb[(size_t)b * nk + k] = P.nbr[(size_t)k * P.nnb + b];
    if (cudaMemcpyAsync(dnbr, nb.data(), sizeof(int) * nb.size(), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
      return bail(fail(EDUS_ECUDA, "upload nbr"));
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "sync"));
  }
  // ---- constants
  DevConsts& h = c->hc;
  memset(&h, 0, sizeof(h));
  for (int b = 0; b < P.nnb; b++) {
    h.wb[b] = P.shell_w[P.bshell[b]];
    for (int x = 0; x < 3; x++) h.bvec[b][x] = P.bvec[b * 3 + x];
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) h.T[i * n + j] = P.T[i][j];
  for (size_t t = 0; t < P.diss_i.size(); t++) {
    h.diss_i[t] = P.diss_i[t];
    h.diss_j[t] = P.diss_j[t];
  }
  // ---- state
  if ((rc = dalloc(c, &c->d_P0, c->plane)) || (rc = dalloc(c, &c->d_P1, c->plane)) || (rc = dalloc(c, &c->d_Pa, c->plane)) ||
      (rc = dalloc(c, &c->d_Pb, c->plane)))
    return bail(rc);
  if (c->order > 0 && (rc = dalloc(c, &c->d_ring, (size_t)c->order * c->plane))) return bail(rc);
  if (c->d_ring && cudaMemsetAsync(c->d_ring, 0, sizeof(double2) * c->order * c->plane, c->stream) != cudaSuccess)
    return bail(fail(EDUS_ECUDA, "memset ring"));
  for (int i = 0; i < kMaxOrder; i++) c->ring_idx[i] = i;
  if ((rc = state_to_dev(c, (const double*)P.P0.data(), c->d_P0))) return bail(rc);
  if ((rc = dalloc(c, &c->d_Pinit, c->plane))) return bail(rc);
  if (cudaMemcpyAsync(c->d_Pinit, c->d_P0, sizeof(double2) * c->plane, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
    return bail(fail(EDUS_ECUDA, "copy initial state"));
  c->use_graphs = o.use_graphs != 0;
  // ---- observables
  if ((rc = dalloc(c, (char**)&c->d_part, obs_parts(nk) * obs_part_bytes())) || (rc = dalloc(c, &c->d_done, 1)) ||
      (rc = dalloc(c, &c->d_ncond, 1)) || (rc = dalloc(c, &c->d_pcmax, 1)) || (rc = dalloc(c, &c->d_maxdp, 1)) ||
      (rc = dalloc(c, &c->d_err, 1)))
    return bail(rc);
  cudaMemsetAsync(c->d_ncond, 0, sizeof(double), c->stream);
  cudaMemsetAsync(c->d_done, 0, sizeof(unsigned int), c->stream);
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->d_pcmax, 0, sizeof(double), c->stream);
  c->log_cap = P.p.dynamical_dt ? 1 << 16 : P.nprint + 2;
  if ((rc = dalloc(c, &c->d_log, c->log_cap))) return bail(rc);
  if (c->dyn) {
    // adaptive step on the device: its scalars, the pinned flag, snapshot times
    if ((rc = dalloc(c, &c->d_dyn, 1))) return bail(rc);
    if (cudaHostAlloc(&c->h_active, sizeof(int), cudaHostAllocDefault) != cudaSuccess)
      return bail(fail(EDUS_ENOMEM, "pinned flag"));
    if (P.p.print_population || P.p.print_band_dispersion) {
      c->snapt_cap = c->log_cap;
      if ((rc = dalloc(c, &c->d_snapt, (size_t)c->snapt_cap))) return bail(rc);
    }
  }
  // ---- per-k snapshots: slots for every snapshot the run can take
  c->snap_on = P.p.print_population || P.p.print_band_dispersion;
  if (c->snap_on && (P.p.print_population || c->coul)) {
    c->snap_ic = P.nbands - 1;  // top valence and bottom conduction band (Nb[0] + Nb[1] - 1, Nb[0] + Nb[1])
    c->snap_jc = P.nbands;
    if (P.p.print_population && (c->snap_ic < 0 || c->snap_jc >= n))
      return bail(fail(EDUS_EUNSUPPORTED, "PrintPopulation needs a valence and a conduction band"));
    int cap = 0;
    if (!c->dyn) {
      // the snapshot switch along the constant-dt clock of the run loop
      double t = P.t_start;
      int ic = -1;
      for (int it = 0; it <= P.itfi; it++) {
        if (it % c->res == 0 && t > P.p.print_start + ic * P.p.print_step && t < P.p.print_end) ic++;
        t += P.p.dt;
      }
      cap = ic + 1;
    } else if (P.p.print_step > 0) {
      cap = (int)std::min<double>(c->log_cap, std::floor((P.p.print_end - P.p.print_start) / P.p.print_step) + 2);
    } else {
      return bail(fail(EDUS_EUNSUPPORTED, "PrintPopulation with step <= 0 under a dynamical dt"));
    }
    if ((double)cap * (3 * sizeof(double2) + n * sizeof(double)) * nk > 16e9)
      return bail(fail(EDUS_EUNSUPPORTED, "%d snapshots exceed 16 GB", cap));
    c->snap_cap = cap;
    if (cap > 0 && P.p.print_population && (rc = dalloc(c, &c->d_snap, (size_t)cap * 3 * nk))) return bail(rc);
    if (cap > 0 && c->coul && (rc = dalloc(c, &c->d_edia, (size_t)cap * n * nk))) return bail(rc);
  }
  // ---- tables struct
  DevTables& tb = c->tb;
  memset(&tb, 0, sizeof(tb));
  tb.n = n;
  tb.ntri = nt;
  tb.nk = nk;
  tb.nnb = P.nnb;
  tb.n1 = P.p.sample_110 ? P.p.nk[0] : P.p.nk[1];
  tb.n2 = P.p.sample_110 ? P.p.nk[1] : P.p.nk[2];
  tb.nch = P.nch;
  tb.nbands = P.nbands;
  tb.H = dH;
  tb.D = dD;
  tb.U = dU;
  tb.GE = dGE;
  tb.nbr = dnbr;
  tb.err = c->d_err;
  tb.n_diss = (int)P.diss_i.size();
  tb.herm_dip = herm ? 1 : 0;
  // ---- velocity gauge (tdse{ velocity_gauge }): Fourier coefficients of the
  // model; the tables tb.H, tb.D are rebuilt at k + A for every stage
  c->vg = P.p.velocity_gauge != 0;
  if (c->vg) {
    if (P.p.mode != EDUS_MODE_WANNIER || P.HR.empty())
      return bail(fail(EDUS_EUNSUPPORTED, "velocity gauge: Wannier models only (H(R), r(R) tables)"));
    if (c->solver != EDUS_SOLVER_RK4 || c->dyn || P.p.coulomb || P.p.conduction_shift > 1e-16 || !P.diss_i.empty())
      return bail(fail(EDUS_EUNSUPPORTED,
                       "velocity gauge: RK4 at constant dt, without the Coulomb mean field, scissor shift or dissipation"));
    const int nr = P.nrpts;
    std::vector<double2> coef((size_t)4 * nt * nr);
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++) {
        const int e = i * n - (i * (i - 1)) / 2 + (j - i);
        for (int r = 0; r < nr; r++) {
          const cd h = P.HR[((size_t)i * n + j) * nr + r];
          coef[(size_t)e * nr + r] = make_double2(h.real(), h.imag());
          for (int x = 0; x < 3; x++) {
            const cd d = 0.5 * (P.rR[(((size_t)x * n + i) * n + j) * nr + r] + P.rR[(((size_t)x * n + j) * n + i) * nr + r]);
            coef[((size_t)(1 + x) * nt + e) * nr + r] = make_double2(d.real(), d.imag());
          }
        }
      }
    double2* dcoef = nullptr;
    double *dk = nullptr, *dR = nullptr;
    if ((rc = dalloc(c, &dcoef, coef.size())) || (rc = upload(c, dcoef, coef)) || (rc = dalloc(c, &dk, (size_t)3 * nk)) ||
        (rc = dalloc(c, &dR, (size_t)3 * nr)))
      return bail(rc);
    if (cudaMemcpyAsync(dk, P.kpt.data(), sizeof(double) * 3 * nk, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
        cudaMemcpyAsync(dR, P.Rvec.data(), sizeof(double) * 3 * nr, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
      return bail(fail(EDUS_ECUDA, "velocity gauge: upload"));
    VgArgs& v = c->vga;
    v.n = n;
    v.ntri = nt;
    v.nk = nk;
    v.nr = nr;
    v.kpt = dk;
    v.Rvec = dR;
    v.coef = dcoef;
    v.H = dH;
    v.D = dD;
    const int prec = o.precision >= 0 ? o.precision : P.p.precision;
    c->vg_tc = prec == EDUS_PREC_MIXED && batch::tc_seg_k(nr) <= 1024;
    if (c->vg_tc) {
      // power-of-two scale of each GEMM column from max_R |c(R)| (bounds |Re|, |Im| of
      // e^{2 pi i A.R} c(R) for every A): every sliced value lies in [-1/2, 1/2]
      const int ncols = 8 * nt, kpad = batch::tc_pad_k(nr);
      std::vector<double> cs(ncols);
      for (int ce = 0; ce < 4 * nt; ce++) {
        double amax = 0.;
        for (int r = 0; r < nr; r++) amax = std::max(amax, std::hypot(coef[(size_t)ce * nr + r].x, coef[(size_t)ce * nr + r].y));
        cs[2 * ce] = cs[2 * ce + 1] = amax > 0. ? std::ldexp(1.0, std::ilogb(amax) + 2) : 1.0;
      }
      double* dcs = nullptr;
      uint16_t *dA = nullptr, *dB = nullptr;
      double* dC = nullptr;
      if ((rc = dalloc(c, &dcs, (size_t)ncols)) || (rc = dalloc(c, &dA, (size_t)nk * kpad)) ||
          (rc = dalloc(c, &dB, (size_t)ncols * kpad)) || (rc = dalloc(c, &dC, (size_t)nk * ncols)))
        return bail(rc);
      if (cudaMemcpyAsync(dcs, cs.data(), sizeof(double) * ncols, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        return bail(fail(EDUS_ECUDA, "velocity gauge: upload"));
      batch::TcVgArgs& g = c->vgt;
      g.n = n;
      g.ntri = nt;
      g.nk = nk;
      g.nr = nr;
      g.kpt = dk;
      g.Rvec = dR;
      g.coef = dcoef;
      g.colscale = dcs;
      g.Aw = dA;
      g.Bw = dB;
      g.Cw = dC;
      g.H = dH;
      g.D = dD;
      g.err = c->d_err;
      if (batch::tc_vg_prepare(g, c->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "velocity gauge: phase slices"));
      // the TMA tensor maps, unless EDUS_TC_GEMM=cpasync selects the cp.async form
      if (batch::tc_gemm_tma_wanted()) batch::tc_vg_maps(g);
    }
    c->vg_t = P.t_start;
    if ((rc = vg_tables(c, P.t_start))) return bail(rc);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "velocity gauge: initial tables"));
  }
  // ---- Coulomb
  if (c->coul) {
    const int nc = P.ncut, n1 = tb.n1, n2 = tb.n2;
    if (n1 * n2 != nk) return bail(fail(EDUS_EINVAL, "Coulomb needs a 2D grid"));
    const int a1 = P.p.sample_110 ? 0 : 1, a2 = P.p.sample_110 ? 1 : 2;
    std::vector<double> t1c((size_t)nc * n1), t1s((size_t)nc * n1), t2c((size_t)nc * n2), t2s((size_t)nc * n2);
    for (int m = 0; m < nc; m++) {
      for (int i1 = 0; i1 < n1; i1++) {
        double x = 2 * M_PI * m * (P.kpt[(size_t)(i1 * n2) * 3 + a1]);
        t1c[(size_t)m * n1 + i1] = std::cos(x);
        t1s[(size_t)m * n1 + i1] = std::sin(x);
      }
      for (int i2 = 0; i2 < n2; i2++) {
        double x = 2 * M_PI * m * (P.kpt[(size_t)i2 * 3 + a2]);
        t2c[(size_t)m * n2 + i2] = std::cos(x);
        t2s[(size_t)m * n2 + i2] = std::sin(x);
      }
    }
    double *d1c, *d1s, *d2c, *d2s;
    if ((rc = dalloc(c, &d1c, t1c.size())) || (rc = dalloc(c, &d1s, t1s.size())) || (rc = dalloc(c, &d2c, t2c.size())) ||
        (rc = dalloc(c, &d2s, t2s.size())))
      return bail(rc);
    cudaMemcpyAsync(d1c, t1c.data(), sizeof(double) * t1c.size(), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d1s, t1s.data(), sizeof(double) * t1s.size(), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d2c, t2c.data(), sizeof(double) * t2c.size(), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d2s, t2s.data(), sizeof(double) * t2s.size(), cudaMemcpyHostToDevice, c->stream);
    // bulk-copy layouts: t2T [n2][2 ncut] and t1P [2][ncut][n1|1], both padded to 16 bytes
    std::vector<double> t2T(coulomb_t2T_count(n2, nc), 0.0), t1P(coulomb_t1P_count(n1, nc), 0.0);
    for (int i2 = 0; i2 < n2; i2++)
      for (int m = 0; m < nc; m++) {
        t2T[(size_t)i2 * 2 * nc + m] = t2c[(size_t)m * n2 + i2];
        t2T[(size_t)i2 * 2 * nc + nc + m] = t2s[(size_t)m * n2 + i2];
      }
    const int ld = n1 | 1;
    for (int m = 0; m < nc; m++)
      for (int i1 = 0; i1 < n1; i1++) {
        t1P[(size_t)m * ld + i1] = t1c[(size_t)m * n1 + i1];
        t1P[(size_t)(nc + m) * ld + i1] = t1s[(size_t)m * n1 + i1];
      }
    double *d2T, *d1P;
    if ((rc = dalloc(c, &d2T, t2T.size())) || (rc = dalloc(c, &d1P, t1P.size()))) return bail(rc);
    cudaMemcpyAsync(d2T, t2T.data(), sizeof(double) * t2T.size(), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d1P, t1P.data(), sizeof(double) * t1P.size(), cudaMemcpyHostToDevice, c->stream);
    c->cd.t2T = d2T;
    c->cd.t1P = d1P;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "upload trig tables"));
    std::vector<double2> cf[4];
    const std::vector<cd>* src[4] = {&P.cA, &P.cB, &P.cC, &P.cD};
    std::vector<unsigned char> isd(nt);
    std::vector<int> diag_of(nt, 0);
    for (int q = 0; q < 4; q++) {
      cf[q].assign((size_t)nc * nc * nt, make_double2(0, 0));
      for (int mm = 0; mm < nc * nc; mm++)
        for (int i = 0; i < n; i++)
          for (int j = i; j < n; j++) {
            int lin = (i == j) ? 0 : i * n + j;
            cd v = (*src[q])[(size_t)mm * n * n + lin];
            cf[q][(size_t)mm * nt + tri_index(i, j, n)] = make_double2(v.real(), v.imag());
          }
    }
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++) {
        int e = tri_index(i, j, n);
        isd[e] = (i == j);
        diag_of[e] = i;
        int lin = (i == j) ? 0 : i * n + j;
        cd s = std::conj(P.screen[lin]);
        h.screen[e] = make_double2(s.real(), s.imag());
      }
    // diagonal basis (headers/RungeKutta.h:96-108): Screen_const[0][0] on the
    // diagonal, conj(Screen_const[0][1]) on every off-diagonal element
    h.screen_d00 = make_double2(P.screen[0].real(), P.screen[0].imag());
    if (n > 1) h.screen_d01c = make_double2(P.screen[1].real(), -P.screen[1].imag());
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) h.VH[i * n + j] = P.VH[(size_t)i * n + j];
    double2* dcf[4];
    for (int q = 0; q < 4; q++) {
      if ((rc = dalloc(c, &dcf[q], cf[q].size())) || (rc = upload(c, dcf[q], cf[q]))) return bail(rc);
    }
    unsigned char* disd;
    int* ddo;
    if ((rc = dalloc(c, &disd, nt)) || (rc = dalloc(c, &ddo, nt))) return bail(rc);
    cudaMemcpyAsync(disd, isd.data(), nt, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(ddo, diag_of.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, c->stream);
    double2 *dg, *dfd, *dPW0;
    if ((rc = dalloc(c, &dg, (size_t)n1 * 2 * nc * nt)) || (rc = dalloc(c, &c->d_h, (size_t)n1 * 2 * nc * nt)) ||
        (rc = dalloc(c, &c->d_X0, (size_t)4 * nc * nc * nt)) || (rc = dalloc(c, &dfd, n)) || (rc = dalloc(c, &dPW0, c->plane)) ||
        (rc = dalloc(c, &c->d_hr, c->plane)))
      return bail(rc);
    c->cd.g = dg;
    c->cd.t1c = d1c;
    c->cd.t1s = d1s;
    c->cd.t2c = d2c;
    c->cd.t2s = d2s;
    c->cd.A = dcf[0];
    c->cd.B = dcf[1];
    c->cd.C = dcf[2];
    c->cd.D = dcf[3];
    c->cd.is_diag = disd;
    c->cd.diag_of = ddo;
    c->cd.fdiag = dfd;
    tb.ncut = nc;
    tb.t2c = d2c;
    tb.t2s = d2s;
    tb.fdiag = dfd;
    tb.PW0 = dPW0;
    tb.ncond = c->d_ncond;
    // equilibrium coefficients (main_MPI.cpp:276-337): X0 = X(P0), E_H0 from f_cc(0,0)
    if (cudaMemcpyAsync(dPW0, c->d_P0, sizeof(double2) * c->plane, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
      return bail(fail(EDUS_ECUDA, "copy PW0"));
    if (cudaMemcpyAsync(c->d_hr, dH, sizeof(double2) * c->plane, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
      return bail(fail(EDUS_ECUDA, "copy Hr"));
    if (coulomb_prepare(tb) != cudaSuccess) return bail(fail(EDUS_EUNSUPPORTED, "Coulomb tables exceed shared memory"));
    const double2* eq = c->d_P0;
    if (P.p.diag_basis) {
      // the equilibrium state in the eigenbasis: 1 on the filled bands (main_MPI.cpp:291-304)
      if (n > 4) return bail(fail(EDUS_EUNSUPPORTED, "Coulomb_diag_basis: up to 4 bands"));
      c->diagb = true;
      if ((rc = dalloc(c, &c->d_pdiag, c->plane)) || (rc = dalloc(c, &c->d_xw, c->plane))) return bail(rc);
      std::vector<double2> pe(c->plane, make_double2(0, 0));
      for (int i = 0; i < P.nbands && i < n; i++)
        for (int k = 0; k < nk; k++) pe[(size_t)tri_index(i, i, n) * nk + k] = make_double2(1.0, 0.0);
      if ((rc = upload(c, c->d_pdiag, pe))) return bail(rc);
      eq = c->d_pdiag;
    }
    if (launch_coulomb(tb, c->cd, eq, nullptr, c->d_X0, nullptr, c->stream) != cudaSuccess)
      return bail(fail(EDUS_ECUDA, "equilibrium Coulomb pass"));
    std::vector<double2> fd(n);
    cudaMemcpyAsync(fd.data(), dfd, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "sync"));
    for (int i = 0; i < n; i++) {
      double eh = 0;
      for (int j = 0; j < n; j++) eh += fd[j].x * P.VH[(size_t)i * n + j];
      h.EH0[i] = eh;
    }
    tb.h = c->d_h;
  }
  if ((rc = dalloc(c, &c->d_cst, 1))) return bail(rc);
  if (cudaMemcpyAsync(c->d_cst, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    return bail(fail(EDUS_ECUDA, "upload constants"));
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "sync"));
  // ---- loop state (Source_Main/const_dt_evolution.cpp:1-9, main_MPI.cpp:269-274)
  c->it = 0;
  c->itfi = P.itfi;
  c->time_loop = P.t_start;
  c->dt = P.p.dt;
  c->dt0 = P.p.dt;
  for (int i = 0; i < kMaxOrder; i++) c->dt_prev[i] = P.p.dt;
  c->e_non0 = true;
  c->n_cond = c->dyn ? std::pow(10, -16) : 0;
  c->P_cond_max = 0;
  *out = c;
  return 0;
}

int edus_reset(edus_ctx* c) {
  if (!c) return fail(EDUS_EINVAL, "null argument");
  CK(cudaSetDevice(c->device));
  if (c->P0_start) {
    c->d_P0 = c->P0_start;
    c->d_Pa = c->Pa_start;
  }
  CK(cudaMemcpyAsync(c->d_P0, c->d_Pinit, sizeof(double2) * c->plane, cudaMemcpyDeviceToDevice, c->stream));
  if (c->d_ring) CK(cudaMemsetAsync(c->d_ring, 0, sizeof(double2) * c->order * c->plane, c->stream));
  CK(cudaMemsetAsync(c->d_ncond, 0, sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_pcmax, 0, sizeof(double), c->stream));
  if (c->coul) CK(cudaMemcpyAsync(c->d_hr, c->tb.H, sizeof(double2) * c->plane, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->it = 0;
  c->time_loop = c->P.t_start;
  c->dt = c->P.p.dt;
  for (int i = 0; i < kMaxOrder; i++) {
    c->ring_idx[i] = i;
    c->dt_prev[i] = c->P.p.dt;
  }
  memset(c->EF, 0, sizeof(c->EF));
  c->e_non0 = true;
  c->n_cond = c->dyn ? std::pow(10, -16) : 0;
  c->P_cond_max = 0;
  c->nlog = 0;
  c->icont = -1;
  c->snap_t.clear();
  if (c->vg) {
    // the tables at k + A(t0) = k
    c->vg_t = c->P.t_start;
    c->vg_A[0] = c->vg_A[1] = c->vg_A[2] = 0.;
    int rc = vg_tables(c, c->P.t_start);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
  }
  return 0;
}

int edus_set_state(edus_ctx* c, const double* rho) {
  if (!c || !rho) return fail(EDUS_EINVAL, "null argument");
  return state_to_dev(c, rho, c->d_P0);
}
int edus_get_state(edus_ctx* c, double* rho) {
  if (!c || !rho) return fail(EDUS_EINVAL, "null argument");
  return state_from_dev(c, c->d_P0, rho);
}
int edus_slot_set(edus_ctx* c, int32_t slot, const double* rho) {
  double2* d = c ? slot_ptr(c, slot) : nullptr;
  if (!d || !rho) return fail(EDUS_EINVAL, "bad slot %d", slot);
  return state_to_dev(c, rho, d);
}
int edus_slot_get(edus_ctx* c, int32_t slot, double* rho) {
  double2* d = c ? slot_ptr(c, slot) : nullptr;
  if (!d || !rho) return fail(EDUS_EINVAL, "bad slot %d", slot);
  return state_from_dev(c, d, rho);
}
int edus_slot_copy(edus_ctx* c, int32_t src, int32_t dst) {
  double2 *s = c ? slot_ptr(c, src) : nullptr, *d = c ? slot_ptr(c, dst) : nullptr;
  if (!s || !d) return fail(EDUS_EINVAL, "bad slot");
  CK(cudaMemcpyAsync(d, s, sizeof(double2) * c->plane, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int edus_get_derivative(edus_ctx* c, int32_t p_slot, const double EF[6], double wx2, int32_t e_non0) {
  double2* s = c ? slot_ptr(c, p_slot) : nullptr;
  if (!s || !EF) return fail(EDUS_EINVAL, "bad slot %d", p_slot);
  if (p_slot == EDUS_SLOT_PV) return fail(EDUS_EINVAL, "derivative of the Pv slot would overwrite its input");
  StageArgs a = base_args(c);
  for (int i = 0; i < 3; i++) {
    a.EF[0][i] = EF[i];
    a.EF[1][i] = EF[3 + i];
  }
  a.wx2 = wx2;
  a.e_non0 = e_non0;
  a.src = s;
  a.dst = c->d_Pb;
  a.op = OP_PV;
  a.hr_out = c->coul ? c->d_hr : nullptr;
  int rc = rhs(c, a);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int edus_runge_kutta_ad(edus_ctx* c, int32_t src, int32_t dst, double dt) {
  // P_dst = P_src + dt * Pv as an element-wise device update
  double2 *s = c ? slot_ptr(c, src) : nullptr, *d = c ? slot_ptr(c, dst) : nullptr;
  if (!s || !d || src == EDUS_SLOT_PV || dst == EDUS_SLOT_PV) return fail(EDUS_EINVAL, "bad slot");
  CK(cudaSetDevice(c->device));
  CK(launch_axpy(s, c->d_Pb, dt, d, c->plane, c->stream));
  c->launches++;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int edus_runge_kutta_ac(edus_ctx* c, int32_t dst, double dt) { return edus_runge_kutta_ad(c, dst, dst, dt); }

int edus_coulomb_hk(edus_ctx* c, int32_t p_slot, double* hk_out) {
  if (!c || !hk_out) return fail(EDUS_EINVAL, "null argument");
  if (!c->coul) return fail(EDUS_EINVAL, "Coulomb is off in this problem");
  double EF[6] = {0, 0, 0, 0, 0, 0};
  // evaluates the RHS on the slot, which also stores Hk_renorm
  int rc = edus_get_derivative(c, p_slot, EF, 0.0, 0);
  if (rc) return rc;
  return state_from_dev(c, c->d_hr, hk_out);
}

int edus_step(edus_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return fail(EDUS_EINVAL, "bad argument");
  return timed(c, nsteps, false);
}

int edus_run(edus_ctx* c) {
  if (!c) return fail(EDUS_EINVAL, "null argument");
  return timed(c, 0, true);
}

int edus_clock(edus_ctx* c, int32_t* it, double* t, double* dt) {
  if (!c) return fail(EDUS_EINVAL, "null argument");
  if (it) *it = c->it;
  if (t) *t = c->time_loop;
  if (dt) *dt = c->dt;
  return 0;
}

int edus_obs_count(edus_ctx* c, int32_t* n) {
  if (!c || !n) return fail(EDUS_EINVAL, "null argument");
  *n = c->nlog < c->log_cap ? c->nlog : c->log_cap;
  return 0;
}

int edus_obs_get(edus_ctx* c, int32_t first, int32_t count, edus_obs* out) {
  if (!c || !out || first < 0 || count < 0) return fail(EDUS_EINVAL, "bad argument");
  int avail = c->nlog < c->log_cap ? c->nlog : c->log_cap;
  if (first + count > avail) return fail(EDUS_EINVAL, "only %d records", avail);
  if (count == 0) return 0;
  CK(cudaMemcpyAsync(out, c->d_log + first, sizeof(edus_obs) * count, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int edus_observables(edus_ctx* c, edus_obs* out) {
  if (!c || !out) return fail(EDUS_EINVAL, "null argument");
  edus_obs rec;
  memset(&rec, 0, sizeof(rec));
  rec.t = c->time_loop;
  rec.dt = c->dt;
  if (!c->d_obs_one) {
    int rc = dalloc(c, &c->d_obs_one, 1);
    if (rc) return rc;
  }
  edus_obs* tmp = c->d_obs_one;
  double scaleJ = c->P.dk[0] * c->P.dk[1] * c->P.dk[2] / c->P.det_a;
  double scaleTA = std::fabs(c->P.jac) * c->P.dk[0] * c->P.dk[1] * c->P.dk[2];
  CK(launch_observables(c->tb, c->d_cst, c->d_P0, c->vg ? c->vga.H : (c->coul ? c->d_hr : nullptr), c->P.p.current, c->P.p.tabs, c->d_part,
                        c->d_done, scaleJ, scaleTA, rec, tmp, nullptr, nullptr, c->stream));
  CK(cudaMemcpyAsync(out, tmp, sizeof(edus_obs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int edus_profile(edus_ctx* c, int32_t nsteps, double* rhs_ms, int64_t* rhs_launches, double* coul_ms,
                 int64_t* coul_launches) {
  return edus_profile_ex(c, nsteps, 1, rhs_ms, rhs_launches, coul_ms, coul_launches);
}

int edus_profile_ex(edus_ctx* c, int32_t nsteps, int32_t reps, double* rhs_ms, int64_t* rhs_launches, double* coul_ms,
                    int64_t* coul_launches) {
  if (!c || nsteps < 0 || reps < 1) return fail(EDUS_EINVAL, "bad argument");
  CK(cudaSetDevice(c->device));
  c->profiling = true;
  c->prof_reps = reps;
  c->prof_pairs.clear();
  int rc = run_steps(c, nsteps, false);
  c->profiling = false;
  c->prof_reps = 1;
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  double t[2] = {0, 0};
  int64_t n[2] = {0, 0};
  for (auto& p : c->prof_pairs) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, p.a, p.b));
    t[p.kind] += ms;
    n[p.kind] += p.reps;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  c->prof_pairs.clear();
  if (rhs_ms) *rhs_ms = t[0];
  if (rhs_launches) *rhs_launches = n[0];
  if (coul_ms) *coul_ms = t[1];
  if (coul_launches) *coul_launches = n[1];
  return 0;
}

int edus_last_timing(edus_ctx* c, double* ms, int64_t* launches) {
  if (!c) return fail(EDUS_EINVAL, "null argument");
  if (ms) *ms = c->last_ms;
  if (launches) *launches = c->last_launches;
  return 0;
}

// Output/{EF,J1,J2,Losses,TransientAbs,k_grid}.txt with the reference's stream
// formats (headers/Observables_MPI.h:134-140, 398-406, 492-550, 586-595,
// 707-712, 766-771).
int edus_write_outputs(edus_ctx* c, const char* outdir) {
  if (!c || !outdir) return fail(EDUS_EINVAL, "null argument");
  int32_t n = 0;
  edus_obs_count(c, &n);
  std::vector<edus_obs> log(n);
  int rc = edus_obs_get(c, 0, n, log.data());
  if (rc) return rc;
  if ((rc = write_kgrid(c->P, outdir))) return rc;
  std::string d = outdir;
  if (c->snap_on && (rc = write_snapshots(c, d))) return rc;
  if ((rc = write_initial(c, d))) return rc;
  std::ofstream fe(d + "/EF.txt"), fl(d + "/Losses.txt");
  // Exciton.txt receives one empty line per output instant, J3.txt and
  // Jintra.txt are opened with the currents and left empty, as in the
  // reference (Source_Main/open_files.cpp:22-36, headers/Observables_MPI.h:407)
  std::ofstream fx(d + "/Exciton.txt");
  std::ofstream f1, f2, ft;
  if (c->P.p.current) {
    f1.open(d + "/J1.txt");
    f2.open(d + "/J2.txt");
    std::ofstream(d + "/J3.txt");
    std::ofstream(d + "/Jintra.txt");
  }
  if (c->P.p.tabs) ft.open(d + "/TransientAbs.txt");
  // extension (no reference counterpart): polarisation per cell (1/Nk) sum_k Tr(D_x rho),
  // complex x, y, z, in J1.txt's column format
  std::ofstream fp(d + "/Polarization.txt");
  // k-resolved transient absorption: one file per TAbsK point, opened and left
  // empty as the reference leaves it (Source_Main/open_files.cpp:43-55)
  for (int i = 0; c->P.p.tabs_k && i < c->P.p.n_tabs_k; i++) {
    std::ostringstream name;
    name << d << "/TAbsK_" << c->P.p.tabs_k_pts[i][0] << "_" << c->P.p.tabs_k_pts[i][1] << "_" << c->P.p.tabs_k_pts[i][2] << ".txt";
    std::ofstream fk(name.str());
    if (!fk) return fail(EDUS_EIO, "cannot write %s", name.str().c_str());
  }
  if (!fe || !fl || !fp) return fail(EDUS_EIO, "cannot write into %s", outdir);
  const int ncv = c->n;
  for (const edus_obs& o : log) {
    const double tfs = o.t * kTimeAuFs;
    fe << std::setw(15) << std::setprecision(8) << tfs;
    for (int i = 0; i < 3; i++) fe << std::setw(15) << std::setprecision(8) << o.EF_pump[i];
    fe << std::endl;
    fl << std::setprecision(16) << tfs << "   ";
    for (int i = 0; i < ncv; i++) fl << std::setprecision(16) << o.pop[i] << "   ";
    fl << std::endl;
    fx << std::endl;
    fp << std::setw(15) << std::setprecision(8) << tfs;
    for (int x = 0; x < 3; x++) {
      fp << std::setw(25) << std::setprecision(15) << std::scientific << o.pol[2 * x];
      fp << std::setw(25) << std::setprecision(15) << std::scientific << o.pol[2 * x + 1];
    }
    fp << std::defaultfloat << std::endl;
    if (c->P.p.current) {
      f1 << std::setw(15) << std::setprecision(8) << tfs;
      for (int x = 0; x < 3; x++) {
        f1 << std::setw(25) << std::setprecision(15) << std::scientific << o.J1[2 * x];
        f1 << std::setw(25) << std::setprecision(15) << std::scientific << o.J1[2 * x + 1];
      }
      f1 << std::endl;
      f2 << std::setw(15) << std::setprecision(8) << tfs;
      for (int x = 0; x < 3; x++) f2 << std::setw(25) << std::setprecision(15) << std::scientific << o.J2[x];
      f2 << std::endl;
    }
    if (c->P.p.tabs) {
      ft << std::setw(15) << std::setprecision(8) << tfs;
      for (int i = 0; i < 3; i++) ft << std::setw(15) << std::setprecision(8) << o.EF_probe[i];
      for (int x = 0; x < 3; x++) {
        ft << std::setw(15) << std::setprecision(8) << o.tabs[2 * x];
        ft << std::setw(15) << std::setprecision(8) << o.tabs[2 * x + 1];
      }
      ft << std::endl;
    }
  }
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// edus_observables_static — observables of the current state with the
// reduction scratch (per-block partial sums, the arrival counter of the
// last-block reduction, the output record) in a file-scope device array
// instead of device memory the call or the context allocates.
namespace {

// Up to 4096 per-block partials of the observable reduction, i.e. up to
// 4096 * 128 = 524 288 k points; 384 bytes per partial (the partial is 336).
constexpr int kStaticObsParts = 4096;
constexpr size_t kStaticPartBytes = 384;
constexpr size_t kStaticDoneOff = (size_t)kStaticObsParts * kStaticPartBytes;  // 256-aligned
constexpr size_t kStaticRecOff = kStaticDoneOff + 256;
constexpr size_t kStaticScratchBytes = kStaticRecOff + 512;
static_assert(sizeof(edus_obs) <= 512, "observable record exceeds its static slot");
static_assert(kStaticDoneOff % 256 == 0, "counter offset must stay aligned");

static __device__ __align__(256) unsigned char g_obs_scratch[kStaticScratchBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
unsigned char* g_static_base[kStaticMaxDevices] = {};

// Once per device, with that device current: the address of the scratch
// array in this device's memory. The address is kept for the life of the
// process; it belongs to the device's primary context, so it must not be used
// after that context is destroyed (cudaDeviceReset): a caller that resets a
// device must not call edus_observables_static on it again.
int static_scratch(int device, unsigned char** base) {
  if (device < 0 || device >= kStaticMaxDevices) return fail(EDUS_EINVAL, "device %d out of range", device);
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_base[device]) {
    unsigned char* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_obs_scratch);
    if (e != cudaSuccess) return fail(EDUS_ECUDA, "cudaGetSymbolAddress(static observable scratch): %s", cudaGetErrorString(e));
    g_static_base[device] = p;
  }
  *base = g_static_base[device];
  return 0;
}

}  // namespace

extern "C" int edus_observables_static(edus_ctx* c, edus_obs* out) {
  if (!c || !out) return fail(EDUS_EINVAL, "null argument");
  const int parts = obs_parts(c->P.nk);
  if (parts > kStaticObsParts)
    return fail(EDUS_EINVAL, "%d k points exceed the static observable scratch (at most %d k points)", c->P.nk,
                kStaticObsParts * 128);
  if (obs_part_bytes() > kStaticPartBytes) return fail(EDUS_EUNSUPPORTED, "observable partial larger than its static slot");
  CK(cudaSetDevice(c->device));
  unsigned char* base = nullptr;
  int rc = static_scratch(c->device, &base);
  if (rc) return rc;
  unsigned int* done = (unsigned int*)(base + kStaticDoneOff);
  edus_obs* rec_dev = (edus_obs*)(base + kStaticRecOff);
  // the last-block reduction counts arriving blocks from zero
  CK(cudaMemsetAsync(done, 0, sizeof(unsigned int), c->stream));
  edus_obs rec;
  memset(&rec, 0, sizeof(rec));
  rec.t = c->time_loop;
  rec.dt = c->dt;
  double scaleJ = c->P.dk[0] * c->P.dk[1] * c->P.dk[2] / c->P.det_a;
  double scaleTA = std::fabs(c->P.jac) * c->P.dk[0] * c->P.dk[1] * c->P.dk[2];
  CK(launch_observables(c->tb, c->d_cst, c->d_P0, c->vg ? c->vga.H : (c->coul ? c->d_hr : nullptr), c->P.p.current, c->P.p.tabs, base, done,
                        scaleJ, scaleTA, rec, rec_dev, nullptr, nullptr, c->stream));
  CK(cudaMemcpyAsync(out, rec_dev, sizeof(edus_obs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}
