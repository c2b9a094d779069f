// fp64.cu — Coulomb transform and observable kernels (FP64, sm_100a).
//
// k_coul_rows    first pass of the separable truncated Fourier transform of rho
//                over the k grid (headers/Coulomb.h:300-350 restated as two 1-D
//                passes): g[i1][cs][n][e] = sum_i2 rho_e(i1,i2) {cos,sin}(2 pi n k2).
//                One block per k-grid row; the row and the trig table sit in
//                shared memory and every thread owns whole dot products.
// k_coul_modes   second pass + combination with A,B,C,D (Coulomb.h:424-466) and
//                the first pass of the inverse transform (Coulomb.h:510-541).
// k_obs          populations (Observables_MPI.h:217-484), J1/J2 (:668-775) and the
//                transient absorption (:559-598) per k; the last block to finish
//                reduces the per-block partials in a fixed order and writes the
//                output record (no second launch, no host round trip).
#include <cstdio>

#include "dev.cuh"
#include <algorithm>

#include "eig.cuh"
#include "dyn.cuh"
#include "kernels.hpp"

namespace edus {

template <int N>
struct Tri {
  static constexpr int NT = N * (N + 1) / 2;
  static __device__ __forceinline__ int idx(int i, int j) { return i * N - (i * (i - 1)) / 2 + (j - i); }
};

// ----------------------------------------------------------------------- Coulomb

constexpr int kRowThreads = 256;

// grid (n1), block kRowThreads: g[i1][cs][n][e] = sum_i2 rho_e(i1,i2) t_n(i2).
// The row of rho (all elements) and the k2 trig table (transposed to [i2][cs*ncut+n])
// are staged in shared memory; each thread owns whole dot products.
__global__ void __launch_bounds__(kRowThreads) k_coul_rows(const double2* __restrict__ rho, int nk, int n1, int n2, int ntri,
                                                           int ncut, const double* __restrict__ t2T, double2* __restrict__ g,
                                                           int* __restrict__ err) {
  extern __shared__ double2 srow[];  // [ntri][n2] then trig [n2][2 ncut] doubles
  __shared__ unsigned long long bar;
  const int i1 = blockIdx.x;
  const int nq = 2 * ncut;
  double* st = reinterpret_cast<double*>(srow + (size_t)ntri * n2);
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const uint32_t row_bytes = (uint32_t)n2 * sizeof(double2);
  if (threadIdx.x == 0) {
    // the trig table does not depend on the previous kernel: in flight before the wait
    const uint32_t trig_bytes = ((uint32_t)(n2 * nq * sizeof(double)) + 15u) & ~15u;
    mbar_expect_tx(&bar, (uint32_t)ntri * row_bytes + trig_bytes);
    bulk_g2s(st, t2T, trig_bytes, &bar);
  }
  pdl_wait();
  if (threadIdx.x == 0)
    for (int e = 0; e < ntri; e++) bulk_g2s(srow + (size_t)e * n2, rho + (size_t)e * nk + (size_t)i1 * n2, row_bytes, &bar);
  mbar_wait(&bar, 0, err);
  for (int o = threadIdx.x; o < ntri * nq; o += kRowThreads) {
    const int e = o / nq, q = o - e * nq;
    const double2* r = srow + (size_t)e * n2;
    double ax = 0, ay = 0, bx = 0, by = 0;
    int i2 = 0;
    for (; i2 + 1 < n2; i2 += 2) {
      const double2 v0 = r[i2], v1 = r[i2 + 1];
      const double t0 = st[i2 * nq + q], t1 = st[(i2 + 1) * nq + q];
      ax += v0.x * t0;
      ay += v0.y * t0;
      bx += v1.x * t1;
      by += v1.y * t1;
    }
    if (i2 < n2) {
      const double2 v0 = r[i2];
      const double t0 = st[i2 * nq + q];
      ax += v0.x * t0;
      ay += v0.y * t0;
    }
    g[((size_t)q * ntri + e) * n1 + i1] = cmk(ax + bx, ay + by);  // column-contiguous for k_coul_modes
  }
}

constexpr int kModeThreads = 128;

// One block per (n, e): f_xy(m,n,e) over m, X_xy = combine(A,B,C,D) - X0,
// h(i1, {c,s}, n, e) = sum_m X t_m(i1). The k1 trig tables and the g column
// are staged in shared memory.
__global__ void __launch_bounds__(kModeThreads) k_coul_modes(const double2* __restrict__ g, int n1, int ntri, int ncut,
                                                             double invN, const double* __restrict__ t1P, int* __restrict__ err,
                                                             const double2* __restrict__ cA,
                                                             const double2* __restrict__ cB, const double2* __restrict__ cC,
                                                             const double2* __restrict__ cD, const double2* __restrict__ X0,
                                                             const unsigned char* __restrict__ is_diag, double2* __restrict__ h,
                                                             double2* __restrict__ Xout, double2* __restrict__ fdiag,
                                                             const int* __restrict__ diag_of) {
  const int n = blockIdx.x, e = blockIdx.y;
  extern __shared__ double2 sm[];
  double2* gc = sm;           // [2][n1] column of g for this (n, e)
  double2* f = gc + 2 * n1;   // [4][ncut]: cc, cs, sc, ss
  double2* X = f + 4 * ncut;  // [4][ncut]
  const int ld = n1 | 1;  // odd row stride: per-m reads across threads hit distinct banks
  double* tc = reinterpret_cast<double*>(X + 4 * ncut);  // [ncut][ld] (host-padded copy of cos)
  double* ts = tc + (size_t)ncut * ld;                     // [ncut][ld] (sin)
  const double PI = 3.14159265358979323846;
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const uint32_t col_bytes = (uint32_t)n1 * sizeof(double2);
  if (threadIdx.x == 0) {
    // the trig table does not depend on the previous kernel: in flight before the wait
    const uint32_t trig_bytes = ((uint32_t)(2 * ncut * ld * sizeof(double)) + 15u) & ~15u;
    mbar_expect_tx(&bar, 2 * col_bytes + trig_bytes);
    bulk_g2s(tc, t1P, trig_bytes, &bar);
  }
  pdl_wait();
  if (threadIdx.x == 0) {
    bulk_g2s(gc, g + ((size_t)n * ntri + e) * n1, col_bytes, &bar);
    bulk_g2s(gc + n1, g + ((size_t)(ncut + n) * ntri + e) * n1, col_bytes, &bar);
  }
  mbar_wait(&bar, 0, err);
  for (int o = threadIdx.x; o < 4 * ncut; o += kModeThreads) {
    const int xy = o / ncut, m = o - xy * ncut;
    const double* t = (xy < 2 ? tc : ts) + (size_t)m * ld;
    const double2* gv = gc + (xy & 1) * n1;
    double ax = 0, ay = 0, bx = 0, by = 0;
    int i1 = 0;
    for (; i1 + 1 < n1; i1 += 2) {
      const double2 v0 = gv[i1], v1 = gv[i1 + 1];
      ax += v0.x * t[i1];
      ay += v0.y * t[i1];
      bx += v1.x * t[i1 + 1];
      by += v1.y * t[i1 + 1];
    }
    if (i1 < n1) {
      ax += gv[i1].x * t[i1];
      ay += gv[i1].y * t[i1];
    }
    const double corr = -4 * PI * PI * (double)(m * m + n * n) * invN / 27.0;
    const double sc = invN * (1. + corr);
    f[o] = cmk((ax + bx) * sc, (ay + by) * sc);
  }
  __syncthreads();
  const bool dg = is_diag[e];
  for (int m = threadIdx.x; m < ncut; m += kModeThreads) {
    const size_t mm = (size_t)m * ncut + n;
    const double2 A = cA[mm * ntri + e], D = cD[mm * ntri + e];
    const double2 fcc = f[0 * ncut + m], fcs = f[1 * ncut + m], fsc = f[2 * ncut + m], fss = f[3 * ncut + m];
    double2 xcc = cadd(cmul(A, fcc), cmul(D, fss));
    double2 xcs = csub(cmul(A, fcs), cmul(D, fsc));
    double2 xsc = csub(cmul(A, fsc), cmul(D, fcs));
    double2 xss = cadd(cmul(A, fss), cmul(D, fcc));
    if (X0) {
      xcc = csub(xcc, X0[(0 * ncut * ncut + mm) * ntri + e]);
      xcs = csub(xcs, X0[(1 * ncut * ncut + mm) * ntri + e]);
      xsc = csub(xsc, X0[(2 * ncut * ncut + mm) * ntri + e]);
      xss = csub(xss, X0[(3 * ncut * ncut + mm) * ntri + e]);
    }
    if (!dg) {
      const double2 B = cB[mm * ntri + e], C = cC[mm * ntri + e];
      xcc = cadd(xcc, cadd(cmul(B, fcs), cmul(C, fsc)));
      xcs = cadd(xcs, csub(cmul(C, fss), cmul(B, fcc)));
      xsc = cadd(xsc, csub(cmul(B, fss), cmul(C, fcc)));
      xss = csub(xss, cadd(cmul(B, fsc), cmul(C, fcs)));
    }
    X[0 * ncut + m] = xcc;
    X[1 * ncut + m] = xcs;
    X[2 * ncut + m] = xsc;
    X[3 * ncut + m] = xss;
    if (Xout) {
      Xout[(0 * ncut * ncut + mm) * ntri + e] = xcc;
      Xout[(1 * ncut * ncut + mm) * ntri + e] = xcs;
      Xout[(2 * ncut * ncut + mm) * ntri + e] = xsc;
      Xout[(3 * ncut * ncut + mm) * ntri + e] = xss;
    }
  }
  if (n == 0 && dg && threadIdx.x == 0 && fdiag) fdiag[diag_of[e]] = f[0];
  __syncthreads();
  if (!h) return;
  for (int o = threadIdx.x; o < 2 * n1; o += kModeThreads) {
    const int cs = o / n1, i1 = o - cs * n1;
    double ax = 0, ay = 0;
    // cs = 0: sum_m X_cc c_m + X_sc s_m ; cs = 1: sum_m X_cs c_m + X_ss s_m
    const double2* Xc = X + (cs == 0 ? 0 : 1) * ncut;
    const double2* Xs = X + (cs == 0 ? 2 : 3) * ncut;
    for (int m = 0; m < ncut; m++) {
      const double c = tc[(size_t)m * ld + i1], s = ts[(size_t)m * ld + i1];
      ax += Xc[m].x * c + Xs[m].x * s;
      ay += Xc[m].y * c + Xs[m].y * s;
    }
    h[((size_t)i1 * 2 * ncut + cs * ncut + n) * ntri + e] = cmk(ax, ay);
  }
}

// ----------------------------------------------------------------------- observables

struct ObsPart {
  double pop[kMaxBands];
  double2 J1[3], J2[3], TA[3], PL[3];
  double pmax, pmin;
};

__device__ __forceinline__ void obs_zero(ObsPart& p) {
  for (int i = 0; i < kMaxBands; i++) p.pop[i] = 0;
  for (int x = 0; x < 3; x++) p.J1[x] = p.J2[x] = p.TA[x] = p.PL[x] = cz();
  p.pmax = 0;
  p.pmin = 1.0;
}
__device__ __forceinline__ void obs_add(ObsPart& d, const ObsPart& o, int n) {
  for (int i = 0; i < n; i++) d.pop[i] += o.pop[i];
  for (int x = 0; x < 3; x++) {
    d.J1[x] = cadd(d.J1[x], o.J1[x]);
    d.J2[x] = cadd(d.J2[x], o.J2[x]);
    d.TA[x] = cadd(d.TA[x], o.TA[x]);
    d.PL[x] = cadd(d.PL[x], o.PL[x]);
  }
  d.pmax = fmax(d.pmax, o.pmax);
  d.pmin = fmin(d.pmin, o.pmin);
}

struct ObsArgs {
  const double2* rho;
  const double2* hr;
  int want_current, want_tabs;
  ObsPart* part;
  unsigned int* done;
  double scaleJ, scaleTA;
  ObsRecord rec;
  ObsRecord* log;
  double* ncond_dev;
  double* pcmax_dev;
  // adaptive step on the device: the instant is taken only when dyn->obs_now,
  // with the clock, field and step of *dyn, into record dyn->nlog of log
  const DynStep* dyn;
};

constexpr int kObsThreads = 128;

template <int N>
__global__ void __launch_bounds__(kObsThreads) k_obs(DevTables tb, const DevConsts* __restrict__ cst, ObsArgs a) {
  constexpr int NT = Tri<N>::NT;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = tb.nk;
  __shared__ ObsPart sp[kObsThreads];
  __shared__ bool last;
  ObsPart my;
  obs_zero(my);
  const double2* rho = a.rho;
  const double2* hr = a.hr;
  pdl_wait();
  if (a.dyn && !a.dyn->obs_now) return;  // uniform: no instant at this step
  if (k < nk) {
    double2 P[NT];
#pragma unroll
    for (int e = 0; e < NT; e++) P[e] = rho[(size_t)e * nk + k];
    auto Pf = [&](int i, int j) -> double2 { return (i <= j) ? P[Tri<N>::idx(i, j)] : cconj(P[Tri<N>::idx(j, i)]); };
    double2 Ue[N * N];
    if (hr) {
      double2 A[N * N], Z[N * N];
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
          const double2 v = hr[(size_t)Tri<N>::idx(i, j) * nk + k];
          A[i * N + j] = v;
          A[j * N + i] = cconj(v);
        }
      eig_herm_dev<N>(A, Z);
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) Ue[i * N + j] = cconj(Z[j * N + i]);
    } else {
#pragma unroll
      for (int e = 0; e < N * N; e++) Ue[e] = tb.U[(size_t)e * nk + k];
    }
#pragma unroll
    for (int c = 0; c < N; c++) {
      double2 acc = cz();
#pragma unroll
      for (int ii = 0; ii < N; ii++) {
        double2 m = cz();
#pragma unroll
        for (int jj = 0; jj < N; jj++) m = cadd(m, cmul(Pf(ii, jj), Ue[c * N + jj]));
        acc = cadd(acc, cmul(cconj(Ue[c * N + ii]), m));
      }
      const double Pik = acc.x;
      my.pop[c] = Pik;
      if (c < tb.nbands) {
        my.pmax = fmax(my.pmax, fabs(1. - Pik));
        my.pmin = fmin(my.pmin, 1. - Pik);
      } else {
        my.pmax = fmax(my.pmax, fabs(Pik));
        my.pmin = fmin(my.pmin, Pik);
      }
    }
    if (a.want_current) {
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
          const int e = Tri<N>::idx(i, j);
          double2 ge[3];
          if (hr) {
            ge[0] = ge[1] = ge[2] = cz();
            const double2 h0 = hr[(size_t)e * nk + k];
            for (int b = 0; b < tb.nnb; b++) {
              const int kb = tb.nbr[(size_t)b * nk + k];
              const double2 d = csub(hr[(size_t)e * nk + kb], h0);
#pragma unroll
              for (int x = 0; x < 3; x++) ge[x] = cadd(ge[x], cscale(d, cst->wb[b] * cst->bvec[b][x]));
            }
          } else {
#pragma unroll
            for (int x = 0; x < 3; x++) ge[x] = tb.GE[(size_t)(x * NT + e) * nk + k];
          }
#pragma unroll
          for (int x = 0; x < 3; x++) {
            my.J1[x] = cadd(my.J1[x], cmul(P[e], ge[x]));
            if (i != j) my.J1[x] = cadd(my.J1[x], cmul(cconj(P[e]), cconj(ge[x])));
          }
        }
      const double2* Hs = hr ? hr : tb.H;
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          const double2 pij = Pf(i, j);
#pragma unroll
          for (int l = 0; l < N; l++) {
            const double2 hil = (i <= l) ? Hs[(size_t)Tri<N>::idx(i, l) * nk + k] : cconj(Hs[(size_t)Tri<N>::idx(l, i) * nk + k]);
            const double2 ph = cmul(pij, hil);
            const int lo = j < l ? j : l, hi = j < l ? l : j;
            // D_jl: the stored upper entry, conjugated below the diagonal for Hermitian dipoles
            const bool cj = tb.herm_dip && j > l;
#pragma unroll
            for (int x = 0; x < 3; x++) {
              const double2 ds = tb.D[(size_t)(x * NT + Tri<N>::idx(lo, hi)) * nk + k];
              const double2 d = cj ? cconj(ds) : ds;
              my.J2[x] = cadd(my.J2[x], cmulc(ph, d));
            }
          }
        }
    }
    // polarisation: Tr(D_x rho) = sum_ij D_x,ij P_ij in the reference's P[k][i][j] = rho_ji
    // convention (lower D entries: D_ji = D_ij, or conj(D_ij) for Hermitian dipoles)
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const bool cj = tb.herm_dip && i > j;
        const double2 pij = Pf(i, j);
#pragma unroll
        for (int x = 0; x < 3; x++) {
          const double2 ds = tb.D[(size_t)(x * NT + Tri<N>::idx(lo, hi)) * nk + k];
          my.PL[x] = cadd(my.PL[x], cmul(cj ? cconj(ds) : ds, pij));
        }
      }
    if (a.want_tabs)
      for (int i = 0; i < tb.nch; i++)
        for (int j = tb.nch; j < N; j++) {
          const int e = Tri<N>::idx(i, j);
          for (int x = 0; x < 3; x++)
            my.TA[x] = csub(my.TA[x], cmul(cscale(tb.D[(size_t)(x * NT + e) * nk + k], 2.), P[e]));
        }
  }
  sp[threadIdx.x] = my;
  __syncthreads();
  for (int s = kObsThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) obs_add(sp[threadIdx.x], sp[threadIdx.x + s], N);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.part[blockIdx.x] = sp[0];
    __threadfence();
    const unsigned int prev = atomicAdd(a.done, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  // last block: fixed-order reduction of all block partials
  __threadfence();
  ObsPart t;
  obs_zero(t);
  for (int b = threadIdx.x; b < gridDim.x; b += kObsThreads) obs_add(t, a.part[b], N);
  sp[threadIdx.x] = t;
  __syncthreads();
  for (int s = kObsThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) obs_add(sp[threadIdx.x], sp[threadIdx.x + s], N);
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const ObsPart& T = sp[0];
  ObsRecord rec = a.rec;
  ObsRecord* slot = a.log;
  if (a.dyn) {
    const DynStep* d = a.dyn;
    rec.t = d->t;
    rec.dt = d->dt;
    for (int x = 0; x < 3; x++) {
      rec.EF_pump[x] = d->EF_last[0][x];
      rec.EF_probe[x] = d->EF_last[1][x];
    }
    slot = (a.log && d->nlog < d->log_cap) ? a.log + d->nlog : nullptr;
  }
  const double inv = 1. / nk;
  double trace = -(double)tb.nbands;
  double nc = 0;
  for (int i = 0; i < N; i++) {
    double v = T.pop[i] * inv;
    trace += v;
    if (i < tb.nbands) v = 1.0 - v;
    rec.pop[i] = v;
    if (v > nc) nc = v;
  }
  for (int x = 0; x < 3; x++) {
    rec.J1[2 * x] = T.J1[x].x * a.scaleJ;
    rec.J1[2 * x + 1] = T.J1[x].y * a.scaleJ;
    rec.J2[x] = -2. * (T.J2[x].y * a.scaleJ);
    rec.tabs[2 * x] = T.TA[x].x * a.scaleTA * inv;
    rec.tabs[2 * x + 1] = T.TA[x].y * a.scaleTA * inv;
    rec.pol[2 * x] = T.PL[x].x * inv;
    rec.pol[2 * x + 1] = T.PL[x].y * inv;
  }
  rec.trace_dev = trace;
  rec.p_cond_max = T.pmax;
  rec.p_min = T.pmin;
  rec.n_cond = nc;
  if (slot) *slot = rec;
  if (a.ncond_dev) *a.ncond_dev = nc;
  if (a.pcmax_dev) *a.pcmax_dev = T.pmax;
  *a.done = 0u;
}

// ----------------------------------------------------------------------- launchers

static size_t pad16(size_t b) { return (b + 15) & ~(size_t)15; }
size_t coulomb_rows_smem(const DevTables& tb) {
  return sizeof(double2) * (size_t)tb.ntri * tb.n2 + pad16(sizeof(double) * 2 * (size_t)tb.ncut * tb.n2);
}
size_t coulomb_modes_smem(const DevTables& tb) {
  return sizeof(double2) * (2 * (size_t)tb.n1 + 8 * (size_t)tb.ncut) + pad16(sizeof(double) * 2 * (size_t)tb.ncut * (tb.n1 | 1));
}
// element counts (doubles, padded to 16 bytes) of the host-prepared trig layouts
size_t coulomb_t2T_count(int n2, int ncut) { return pad16(sizeof(double) * 2 * (size_t)ncut * n2) / sizeof(double); }
size_t coulomb_t1P_count(int n1, int ncut) { return pad16(sizeof(double) * 2 * (size_t)ncut * (n1 | 1)) / sizeof(double); }

cudaError_t coulomb_prepare(const DevTables& tb) {
  // opt in to more than 48 KB of dynamic shared memory where needed (227 KB max per block)
  cudaError_t e = cudaFuncSetAttribute(k_coul_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coulomb_rows_smem(tb));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_coul_modes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coulomb_modes_smem(tb));
}

cudaError_t launch_coulomb(const DevTables& tb, const CoulDev& c, const double2* rho, double2* h, double2* Xout,
                           const double2* X0, cudaStream_t s) {
  cudaError_t e = launch_pdl(k_coul_rows, dim3(tb.n1), dim3(kRowThreads), coulomb_rows_smem(tb), s, rho, tb.nk, tb.n1, tb.n2,
                             tb.ntri, tb.ncut, (const double*)c.t2T, c.g, tb.err);
  if (e != cudaSuccess) return e;
  dim3 grid(tb.ncut, tb.ntri);
  return launch_pdl(k_coul_modes, grid, dim3(kModeThreads), coulomb_modes_smem(tb), s, (const double2*)c.g, tb.n1, tb.ntri,
                    tb.ncut, 1.0 / tb.nk, (const double*)c.t1P, tb.err, (const double2*)c.A, (const double2*)c.B,
                    (const double2*)c.C, (const double2*)c.D, X0, (const unsigned char*)c.is_diag, h, Xout, c.fdiag,
                    (const int*)c.diag_of);
}

// Per-k snapshot: elements (ic, jc), (ic, ic) and (jc, jc) of the state in
// the model's eigenbasis, P_dia_rc = sum_ii sum_jj conj(U_r,ii) P_ii,jj U_c,jj
// in the reference's summation order (headers/InitParameters.h:232-255), for
// the snapshots of Source_Main/if_resolution.cpp:231-270. One thread per k.
__global__ void k_snapshot(DevTables tb, const double2* __restrict__ rho, int ic, int jc, double2* __restrict__ out,
                           const DynStep* __restrict__ dyn) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = tb.nk, n = tb.n;
  if (dyn) {
    // adaptive step on the device: slot of this instant's snapshot, if one is due
    const int slot = dyn->snap_slot;
    if (slot < 0) return;
    out += (size_t)slot * 3 * nk;
  }
  if (k >= nk) return;
  auto tri = [n](int i, int j) { return i * n - (i * (i - 1)) / 2 + (j - i); };
  const int rows[3] = {ic, ic, jc}, cols[3] = {jc, ic, jc};
  for (int q = 0; q < 3; q++) {
    const int r = rows[q], c = cols[q];
    double2 acc = cz();
    for (int ii = 0; ii < n; ii++) {
      const double2 ur = cconj(tb.U[(size_t)(r * n + ii) * nk + k]);
      for (int jj = 0; jj < n; jj++) {
        const double2 p = ii <= jj ? rho[(size_t)tri(ii, jj) * nk + k] : cconj(rho[(size_t)tri(jj, ii) * nk + k]);
        acc = cadd(acc, cmul(cmul(ur, p), tb.U[(size_t)(c * n + jj) * nk + k]));
      }
    }
    out[(size_t)q * nk + k] = acc;
  }
}

cudaError_t launch_snapshot(const DevTables& tb, const double2* rho, int ic, int jc, double2* out, cudaStream_t s,
                            const DynStep* dyn) {
  if (!tb.U || ic < 0 || jc < 0 || ic >= tb.n || jc >= tb.n) return cudaErrorInvalidValue;
  k_snapshot<<<(tb.nk + 127) / 128, 128, 0, s>>>(tb, rho, ic, jc, out, dyn);
  return cudaGetLastError();
}

// Band energies of the renormalised Hamiltonian at every k (ascending, as
// eig_sym returns them; headers/Observables_MPI.h:282-303), for the Edia
// snapshot files. One thread per k.
template <int N>
__global__ void k_band_energies(int nk, const double2* __restrict__ hr, double* __restrict__ out, const DynStep* __restrict__ dyn) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (dyn) {
    const int slot = dyn->snap_slot;
    if (slot < 0) return;
    out += (size_t)slot * N * nk;
  }
  if (k >= nk) return;
  double2 A[N * N], Z[N * N];
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i; j < N; j++) {
      const double2 v = hr[(size_t)Tri<N>::idx(i, j) * nk + k];
      A[i * N + j] = v;
      A[j * N + i] = cconj(v);
    }
  eig_herm_dev<N>(A, Z);
#pragma unroll
  for (int i = 0; i < N; i++) out[(size_t)i * nk + k] = A[i * N + i].x;
}

cudaError_t launch_band_energies(const DevTables& tb, const double2* hr, double* out, cudaStream_t s, const DynStep* dyn) {
  const dim3 g((tb.nk + 63) / 64), b(64);
  switch (tb.n) {
    case 1: k_band_energies<1><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    case 2: k_band_energies<2><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    case 3: k_band_energies<3><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    case 4: k_band_energies<4><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    case 5: k_band_energies<5><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    case 8: k_band_energies<8><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    case 16: k_band_energies<16><<<g, b, 0, s>>>(tb.nk, hr, out, dyn); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Coulomb in the diagonal basis (headers/RungeKutta.h:35-55, 96-123).
// The state in the model's eigenbasis, P_d = sum_ii,jj conj(U_c,ii) P_ii,jj U_c',jj
// with a real diagonal (get_P_in_dia_vect, headers/InitParameters.h:264-333),
// as upper planes for the forward transform. One thread per k.
template <int N>
__global__ void k_pdiag(DevTables tb, const double2* __restrict__ rho, double2* __restrict__ pd) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = tb.nk;
  if (k >= nk) return;
  double2 P[N * N], M[N * N];
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i; j < N; j++) {
      const double2 v = rho[(size_t)Tri<N>::idx(i, j) * nk + k];
      P[i * N + j] = v;
      P[j * N + i] = cconj(v);
    }
  // M[jc][ii] = sum_jj P[ii][jj] U[jc][jj]
#pragma unroll
  for (int ii = 0; ii < N; ii++)
#pragma unroll
    for (int jc = 0; jc < N; jc++) {
      double2 m = cz();
#pragma unroll
      for (int jj = 0; jj < N; jj++) m = cadd(m, cmul(P[ii * N + jj], tb.U[(size_t)(jc * N + jj) * nk + k]));
      M[jc * N + ii] = m;
    }
#pragma unroll
  for (int ic = 0; ic < N; ic++)
#pragma unroll
    for (int jc = ic; jc < N; jc++) {
      double2 v = cz();
#pragma unroll
      for (int ii = 0; ii < N; ii++) v = cadd(v, cmul(cconj(tb.U[(size_t)(ic * N + ii) * nk + k]), M[jc * N + ii]));
      if (ic == jc) v.y = 0.;
      pd[(size_t)Tri<N>::idx(ic, jc) * nk + k] = v;
    }
}

// The mean-field term for the diagonal basis: X_d from the inverse-transform
// rows of the P_d coefficients, the screening correction of that basis
// (X_d,ii -= S00 (P_d,ii - [i < Nch + Nv]), X_d,ij -= conj(S01) conj(P_d,ij)),
// then X_W = U^dagger X_d U (get_Xd_in_Wannier_vect, headers/InitParameters.h:
// 339-373), written as upper planes. One thread per k.
template <int N>
__global__ void k_coulomb_xw(DevTables tb, const DevConsts* __restrict__ cst, const double2* __restrict__ pd,
                             double2* __restrict__ xw) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = tb.nk;
  if (k >= nk) return;
  constexpr int NT = Tri<N>::NT;
  const int n2 = tb.n2, nc = tb.ncut;
  const int i1 = k / n2, i2 = k - i1 * n2;
  double2 X[N * N];
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i; j < N; j++) {
      const int e = Tri<N>::idx(i, j);
      const double2* hrow = tb.h + (size_t)i1 * 2 * nc * NT + e;
      double yx = 0., yy = 0.;
      for (int m = 0; m < nc; m++) {
        const double cn = tb.t2c[m * n2 + i2], sn = tb.t2s[m * n2 + i2];
        const double2 c = hrow[(size_t)m * NT], s = hrow[(size_t)(nc + m) * NT];
        yx += c.x * cn + s.x * sn;
        yy += c.y * cn + s.y * sn;
      }
      double2 x = cmk(-yx, yy);
      const double2 p = pd[(size_t)e * nk + k];
      if (i == j) {
        const double pb = i < tb.nbands ? 1.0 : 0.0;
        x = csub(x, cscale(cst->screen_d00, p.x - pb));
      } else {
        x = csub(x, cmul(cst->screen_d01c, cconj(p)));
      }
      X[i * N + j] = x;
      if (i != j) X[j * N + i] = cconj(x);
    }
  // M[ii][jc] = sum_jj X[ii][jj] U[jj][jc]; X_W[ic][jc] = sum_ii conj(U[ii][ic]) M[ii][jc]
  double2 M[N * N];
#pragma unroll
  for (int ii = 0; ii < N; ii++)
#pragma unroll
    for (int jc = 0; jc < N; jc++) {
      double2 m = cz();
#pragma unroll
      for (int jj = 0; jj < N; jj++) m = cadd(m, cmul(X[ii * N + jj], tb.U[(size_t)(jj * N + jc) * nk + k]));
      M[ii * N + jc] = m;
    }
#pragma unroll
  for (int ic = 0; ic < N; ic++)
#pragma unroll
    for (int jc = ic; jc < N; jc++) {
      double2 v = cz();
#pragma unroll
      for (int ii = 0; ii < N; ii++) v = cadd(v, cmul(cconj(tb.U[(size_t)(ii * N + ic) * nk + k]), M[ii * N + jc]));
      xw[(size_t)Tri<N>::idx(ic, jc) * nk + k] = v;
    }
}

cudaError_t launch_pdiag(const DevTables& tb, const double2* rho, double2* pd, cudaStream_t s) {
  const dim3 g((tb.nk + 127) / 128), b(128);
  switch (tb.n) {
    case 1: k_pdiag<1><<<g, b, 0, s>>>(tb, rho, pd); break;
    case 2: k_pdiag<2><<<g, b, 0, s>>>(tb, rho, pd); break;
    case 3: k_pdiag<3><<<g, b, 0, s>>>(tb, rho, pd); break;
    case 4: k_pdiag<4><<<g, b, 0, s>>>(tb, rho, pd); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_coulomb_xw(const DevTables& tb, const DevConsts* cst, const double2* pd, double2* xw, cudaStream_t s) {
  const dim3 g((tb.nk + 127) / 128), b(128);
  switch (tb.n) {
    case 1: k_coulomb_xw<1><<<g, b, 0, s>>>(tb, cst, pd, xw); break;
    case 2: k_coulomb_xw<2><<<g, b, 0, s>>>(tb, cst, pd, xw); break;
    case 3: k_coulomb_xw<3><<<g, b, 0, s>>>(tb, cst, pd, xw); break;
    case 4: k_coulomb_xw<4><<<g, b, 0, s>>>(tb, cst, pd, xw); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// d = a + dt * v over n complex entries, multiply then add without
// contraction, as Runge_Kutta_Ad / Runge_Kutta_Ac (headers/RungeKutta.h:301-355).
__global__ void k_axpy(const double2* a, const double2* __restrict__ v, double dt, double2* d,
                       size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 x = a[i], y = v[i];
    d[i] = make_double2(__dadd_rn(x.x, __dmul_rn(y.x, dt)), __dadd_rn(x.y, __dmul_rn(y.y, dt)));
  }
}

cudaError_t launch_axpy(const double2* a, const double2* v, double dt, double2* d, size_t n, cudaStream_t s) {
  const size_t blocks = std::min<size_t>((n + 255) / 256, 148 * 8);
  k_axpy<<<(unsigned)(blocks ? blocks : 1), 256, 0, s>>>(a, v, dt, d, n);
  return cudaGetLastError();
}

int obs_parts(int nk) { return (nk + kObsThreads - 1) / kObsThreads; }
size_t obs_part_bytes() { return sizeof(ObsPart); }

template <int N>
static cudaError_t launch_obs_n(const DevTables& tb, const DevConsts* cst, const ObsArgs& a, cudaStream_t s) {
  return launch_pdl(k_obs<N>, dim3(obs_parts(tb.nk)), dim3(kObsThreads), 0, s, tb, cst, a);
}

cudaError_t launch_observables(const DevTables& tb, const DevConsts* cst, const double2* rho, const double2* hr,
                               int want_current, int want_tabs, void* part, unsigned int* done, double scaleJ,
                               double scaleTA, const ObsRecord& rec, ObsRecord* log, double* ncond_dev,
                               double* pcmax_dev, cudaStream_t s, const DynStep* dyn) {
  ObsArgs a;
  a.dyn = dyn;
  a.rho = rho;
  a.hr = hr;
  a.want_current = want_current;
  a.want_tabs = want_tabs && tb.nch > 0;
  a.part = (ObsPart*)part;
  a.done = done;
  a.scaleJ = scaleJ;
  a.scaleTA = scaleTA;
  a.rec = rec;
  a.log = log;
  a.ncond_dev = ncond_dev;
  a.pcmax_dev = pcmax_dev;
  switch (tb.n) {
    case 1: return launch_obs_n<1>(tb, cst, a, s);
    case 2: return launch_obs_n<2>(tb, cst, a, s);
    case 3: return launch_obs_n<3>(tb, cst, a, s);
    case 4: return launch_obs_n<4>(tb, cst, a, s);
    case 5: return launch_obs_n<5>(tb, cst, a, s);
    case 8: return launch_obs_n<8>(tb, cst, a, s);
    case 16: return launch_obs_n<16>(tb, cst, a, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace edus
