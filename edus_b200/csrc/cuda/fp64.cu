// fp64.cu — FP64 kernels of the k-space density-matrix propagation (sm_100a).
//
// k_rhs<N>       one thread per k point: builds H~ = H + E.D (+ Coulomb X + Hartree),
//                evaluates -i[H~, rho] (headers/RungeKutta.h:158-212), the RWA term
//                (:209), dissipation (:219-254), the k-gradient stencil (:258-276),
//                hermitizes (:283-294) and applies the stage update of the integrator
//                in the same pass (RK4 headers/RungeKutta.h:301-355 +
//                Source_Main/RungeKutta.cpp; Adams–Bashforth
//                Source_Main/Linear_Multistep_ODE_solvers.cpp:57-94; Taylor
//                Source_Main/Taylor_DE_solver_deriv_Polynom.cpp:100-177). Pv never
//                touches HBM.
// k_coul_rows    first half of the separable truncated Fourier transform of rho over
//                the k grid (headers/Coulomb.h:300-350 restated as two 1-D passes).
// k_coul_modes   second pass + combination with A,B,C,D (Coulomb.h:424-466) + first
//                pass of the inverse transform (Coulomb.h:510-541).
// k_obs / k_obs_final  populations (Observables_MPI.h:217-484), J1/J2 (:668-775),
//                transient absorption (:559-598), reduced in a fixed block order.
#include <cstdio>

#include "dev.cuh"
#include "kernels.hpp"

namespace edus {

// ----------------------------------------------------------------------- helpers

template <int N>
struct Tri {
  static constexpr int NT = N * (N + 1) / 2;
  static __device__ __forceinline__ int idx(int i, int j) { return i * N - (i * (i - 1)) / 2 + (j - i); }
};

__device__ __forceinline__ void atomic_max_pos(unsigned long long* p, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// Hermitian eigenvectors by cyclic Jacobi (device copy of the host routine);
// Z columns are eigenvectors, eigenvalues ascending.
template <int N>
__device__ void eig_herm_dev(double2* A, double2* Z) {
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) Z[i * N + j] = (i == j) ? cmk(1., 0.) : cz();
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = 0, diag = 0;
    for (int i = 0; i < N; i++) {
      diag += A[i * N + i].x * A[i * N + i].x;
      for (int j = i + 1; j < N; j++) off += A[i * N + j].x * A[i * N + j].x + A[i * N + j].y * A[i * N + j].y;
    }
    if (off <= 1e-34 * (diag + 1e-300)) break;
    for (int p = 0; p < N; p++)
      for (int q = p + 1; q < N; q++) {
        double2 apq = A[p * N + q];
        double mag = hypot(apq.x, apq.y);
        if (mag < 1e-300) continue;
        double app = A[p * N + p].x, aqq = A[q * N + q].x;
        double2 ph = cmk(apq.x / mag, apq.y / mag);
        double theta = 0.5 * atan2(2.0 * mag, aqq - app);
        double s, c;
        sincos(theta, &s, &c);
        double2 sp = cscale(ph, s), sc = cscale(cconj(ph), s);
        for (int k = 0; k < N; k++) {
          double2 akp = A[k * N + p], akq = A[k * N + q];
          A[k * N + p] = csub(cscale(akp, c), cmul(sc, akq));
          A[k * N + q] = cadd(cmul(sp, akp), cscale(akq, c));
        }
        for (int k = 0; k < N; k++) {
          double2 apk = A[p * N + k], aqk = A[q * N + k];
          A[p * N + k] = csub(cscale(apk, c), cmul(sp, aqk));
          A[q * N + k] = cadd(cmul(sc, apk), cscale(aqk, c));
        }
        A[p * N + q] = cz();
        A[q * N + p] = cz();
        A[p * N + p].y = 0;
        A[q * N + q].y = 0;
        for (int k = 0; k < N; k++) {
          double2 zkp = Z[k * N + p], zkq = Z[k * N + q];
          Z[k * N + p] = csub(cscale(zkp, c), cmul(sc, zkq));
          Z[k * N + q] = cadd(cmul(sp, zkp), cscale(zkq, c));
        }
      }
  }
  // insertion sort of columns by eigenvalue
  for (int i = 1; i < N; i++) {
    int j = i;
    while (j > 0 && A[(j - 1) * N + (j - 1)].x > A[j * N + j].x) {
      double2 t = A[(j - 1) * N + (j - 1)];
      A[(j - 1) * N + (j - 1)] = A[j * N + j];
      A[j * N + j] = t;
      for (int r = 0; r < N; r++) {
        double2 z = Z[r * N + j - 1];
        Z[r * N + j - 1] = Z[r * N + j];
        Z[r * N + j] = z;
      }
      j--;
    }
  }
}

// ----------------------------------------------------------------------- RHS + update

template <int N>
__global__ void __launch_bounds__(128) k_rhs(DevTables tb, const DevConsts* __restrict__ cst, StageArgs a) {
  constexpr int NT = Tri<N>::NT;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = tb.nk;
  if (k >= nk) return;
  const int nch = tb.nch;

  double2 P[NT];
#pragma unroll
  for (int e = 0; e < NT; e++) P[e] = a.src[(size_t)e * nk + k];

  // H~ (Hermitian, upper) = H + Coulomb X + Hartree
  double2 Hu[NT];
#pragma unroll
  for (int e = 0; e < NT; e++) Hu[e] = tb.H[(size_t)e * nk + k];
  if (tb.h) {
    const int i1 = k / tb.n2, i2 = k - (k / tb.n2) * tb.n2;
    const int nc = tb.ncut;
    const double2* hrow = tb.h + (size_t)i1 * 2 * nc * NT;
    double2 Y[NT];
#pragma unroll
    for (int e = 0; e < NT; e++) Y[e] = cz();
    for (int m = 0; m < nc; m++) {
      const double cn = tb.t2c[m * tb.n2 + i2], sn = tb.t2s[m * tb.n2 + i2];
      const double2* hc = hrow + (size_t)m * NT;
      const double2* hs = hrow + (size_t)(nc + m) * NT;
#pragma unroll
      for (int e = 0; e < NT; e++) {
        double2 c = hc[e], s = hs[e];
        Y[e].x += c.x * cn + s.x * sn;
        Y[e].y += c.y * cn + s.y * sn;
      }
    }
    const bool screen = *tb.ncond > 1e-20;
    // Hartree shift E_H[a] = sum_j Re f_cc(0,0)_jj VH[a][j] - E_H0[a]
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = i; j < N; j++) {
        const int e = Tri<N>::idx(i, j);
        double2 X = cmk(-Y[e].x, Y[e].y);  // conj(-Y)
        if (screen) {
          double2 dP = csub(P[e], tb.PW0[(size_t)e * nk + k]);
          X = csub(X, cmul(cst->screen[e], cconj(dP)));
        }
        if (i == j) {
          X.y = 0.;
          double eh = 0.;
#pragma unroll
          for (int jj = 0; jj < N; jj++) eh += tb.fdiag[jj].x * cst->VH[i * N + jj];
          eh -= cst->EH0[i];
          Hu[e] = cadd(Hu[e], X);
          Hu[e].x += eh;
        } else {
          Hu[e] = cadd(Hu[e], X);
        }
      }
    if (a.hr_out) {
#pragma unroll
      for (int e = 0; e < NT; e++) a.hr_out[(size_t)e * nk + k] = Hu[e];
    }
  }

  // field-dressed H~F[i][j] = H~[i][j] + EF[w] . D[i][j], w = probe iff exactly one index is core
  double2 HF[N * N];
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      const int lo = i < j ? i : j, hi = i < j ? j : i;
      const int e = Tri<N>::idx(lo, hi);
      double2 h = (i <= j) ? Hu[e] : cconj(Hu[e]);
      const int w = (i >= nch && j < nch) || (i < nch && j >= nch);
      const double2 d0 = tb.D[(size_t)(0 * NT + e) * nk + k];
      const double2 d1 = tb.D[(size_t)(1 * NT + e) * nk + k];
      const double2 d2 = tb.D[(size_t)(2 * NT + e) * nk + k];
      h = cadd(h, cscale(d0, a.EF[w][0]));
      h = cadd(h, cscale(d1, a.EF[w][1]));
      h = cadd(h, cscale(d2, a.EF[w][2]));
      HF[i * N + j] = h;
    }
  auto Pf = [&](int i, int j) -> double2 { return (i <= j) ? P[Tri<N>::idx(i, j)] : cconj(P[Tri<N>::idx(j, i)]); };

  double2 Pv[NT];
  // populations: Pv_ii = 2 Im sum_j H~F[i][j] P[i][j]
#pragma unroll
  for (int i = 0; i < N; i++) {
    double2 beta = cz();
#pragma unroll
    for (int j = 0; j < N; j++) beta = cadd(beta, cmul(HF[i * N + j], Pf(i, j)));
    Pv[Tri<N>::idx(i, i)] = cmk(2. * beta.y, 0.);
  }
  // coherences: Pv_ij = -i sum_l (H~F[j][l] P[i][l] - conj(H~F[i][l] P[j][l]))
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i + 1; j < N; j++) {
      double2 beta = cz();
#pragma unroll
      for (int l = 0; l < N; l++) {
        double2 x = cmul(HF[j * N + l], Pf(i, l));
        double2 y = cmul(HF[i * N + l], Pf(j, l));
        beta = cadd(beta, csub(x, cconj(y)));
      }
      double2 v = cmi(beta);
      if (i < nch && j >= nch) v = cadd(v, cmi(cscale(P[Tri<N>::idx(i, j)], -a.wx2)));
      Pv[Tri<N>::idx(i, j)] = v;
    }
  // dissipation (Wannier gauge)
  if (tb.n_diss > 0) {
    double2 Uk[N * N];
#pragma unroll
    for (int e = 0; e < N * N; e++) Uk[e] = tb.U[(size_t)e * nk + k];
    double2 Mk[N * N];
#pragma unroll
    for (int e = 0; e < N * N; e++) Mk[e] = cz();
    for (int t = 0; t < tb.n_diss; t++) {
      const int ii = cst->diss_i[t], jj = cst->diss_j[t];
      double2 m = cz();
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) m = cadd(m, cmul(cmulc(Uk[jj * N + j], Uk[ii * N + i]), Pf(i, j)));
      Mk[ii * N + jj] = m;
    }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = i; j < N; j++) {
        double2 v = Pv[Tri<N>::idx(i, j)];
        for (int t = 0; t < tb.n_diss; t++) {
          const int ii = cst->diss_i[t], jj = cst->diss_j[t];
          // hU[j][jj] = conj(U[jj][j])
          double2 hu = cconj(Uk[jj * N + j]);
          double2 f = cscale(cmulc(hu, Uk[i * N + ii]), cst->T[ii * N + jj]);
          v = csub(v, cmul(f, Mk[ii * N + jj]));
        }
        double2 tii = cz();
        for (int q = 0; q < tb.nbands; q++) {
          // hU[j][q] * conj(hU[i][q]) = conj(U[q][j]) * U[q][i]
          double2 f = cmulc(Uk[q * N + i], Uk[q * N + j]);
          tii = cadd(tii, cscale(f, cst->T[q * N + q]));
        }
        Pv[Tri<N>::idx(i, j)] = cadd(v, tii);
      }
  }
  // k-gradient: sum_b (w_b E_pump . b) rho(k+b)
  if (a.e_non0) {
    double2 G[NT];
#pragma unroll
    for (int e = 0; e < NT; e++) G[e] = cz();
    for (int b = 0; b < tb.nnb; b++) {
      const int kb = tb.nbr[(size_t)b * nk + k];
      const double c0 = cst->wb[b] * a.EF[0][0] * cst->bvec[b][0];
      const double c1 = cst->wb[b] * a.EF[0][1] * cst->bvec[b][1];
      const double c2 = cst->wb[b] * a.EF[0][2] * cst->bvec[b][2];
#pragma unroll
      for (int e = 0; e < NT; e++) {
        const double2 pn = a.src[(size_t)e * nk + kb];
        G[e] = cadd(G[e], cscale(pn, c0));
        G[e] = cadd(G[e], cscale(pn, c1));
        G[e] = cadd(G[e], cscale(pn, c2));
      }
    }
#pragma unroll
    for (int e = 0; e < NT; e++) Pv[e] = cadd(Pv[e], G[e]);
  }
  // hermitize: diagonal real
#pragma unroll
  for (int i = 0; i < N; i++) Pv[Tri<N>::idx(i, i)].y = 0.;

  // ---- stage update
  double dpmax = 0.;
  switch (a.op) {
    case OP_PV:
#pragma unroll
      for (int e = 0; e < NT; e++) a.dst[(size_t)e * nk + k] = Pv[e];
      break;
    case OP_RK_FIRST:
#pragma unroll
      for (int e = 0; e < NT; e++) {
        if (a.ring) a.ring[((size_t)a.ring_idx[0] * NT + e) * nk + k] = Pv[e];  // RK4 start-up of AB
        const double2 b0 = a.base[(size_t)e * nk + k];
        a.acc[(size_t)e * nk + k] = cadd(b0, cscale(Pv[e], a.c1));
        a.dst[(size_t)e * nk + k] = cadd(b0, cscale(Pv[e], a.c2));
      }
      break;
    case OP_RK_MID:
#pragma unroll
      for (int e = 0; e < NT; e++) {
        const double2 b0 = a.base[(size_t)e * nk + k];
        a.acc[(size_t)e * nk + k] = cadd(a.acc[(size_t)e * nk + k], cscale(Pv[e], a.c1));
        a.dst[(size_t)e * nk + k] = cadd(b0, cscale(Pv[e], a.c2));
      }
      break;
    case OP_RK_LAST:
#pragma unroll
      for (int e = 0; e < NT; e++) {
        const double2 nv = cadd(a.acc[(size_t)e * nk + k], cscale(Pv[e], a.c1));
        if (a.maxdp) {
#pragma unroll
          for (int i = 0; i < N; i++)
            if (e == Tri<N>::idx(i, i)) {
              const double2 old = a.dst[(size_t)e * nk + k];
              double v = 2 * hypot(old.x - nv.x, old.y - nv.y) / (a.pcond_plus_ncond + hypot(nv.x, nv.y) + 1.0e-7);
              dpmax = fmax(dpmax, v);
            }
        }
        a.dst[(size_t)e * nk + k] = nv;
      }
      break;
    case OP_AB:
#pragma unroll
      for (int e = 0; e < NT; e++) {
        a.ring[((size_t)a.ring_idx[0] * NT + e) * nk + k] = Pv[e];
        double2 d = cz();
        for (int s = 0; s < a.order; s++) {
          const double2 f = (s == 0) ? Pv[e] : a.ring[((size_t)a.ring_idx[s] * NT + e) * nk + k];
          d = cadd(d, cscale(f, a.coef[s]));
        }
        a.dst[(size_t)e * nk + k] = cadd(a.src[(size_t)e * nk + k], cscale(d, a.dt));
      }
      break;
    case OP_TAYLOR: {
      const int TO = a.order, m = TO - 1;
#pragma unroll
      for (int e = 0; e < NT; e++) {
        a.ring[((size_t)a.ring_idx[0] * NT + e) * nk + k] = Pv[e];
        const double2 f0 = Pv[e];
        double2 dP[kMaxOrder];
        for (int i = 0; i < m; i++) dP[i] = csub(f0, a.ring[((size_t)a.ring_idx[i + 1] * NT + e) * nk + k]);
        double2 d = cscale(f0, a.dt);
        for (int i = 1; i < TO; i++) {
          double2 al = cz();
          for (int q = 0; q < m; q++) al = cadd(al, cscale(dP[q], a.tinv[(i - 1) * m + q]));
          const double2 inc = cscale(cscale(al, a.tpow[i]), 1.0 / (double)(i + 1));
          d = cadd(d, inc);
        }
        const double2 old = a.src[(size_t)e * nk + k];
        const double2 nv = cadd(old, d);
        if (a.maxdp) {
#pragma unroll
          for (int i = 0; i < N; i++)
            if (e == Tri<N>::idx(i, i)) {
              double v = 2 * hypot(old.x - nv.x, old.y - nv.y) / (a.pcond_plus_ncond + hypot(nv.x, nv.y) + 1.0e-7);
              dpmax = fmax(dpmax, v);
            }
        }
        a.dst[(size_t)e * nk + k] = nv;
      }
    } break;
  }
  if (a.maxdp) {
    for (int o = 16; o > 0; o >>= 1) dpmax = fmax(dpmax, __shfl_xor_sync(0xffffffffu, dpmax, o));
    if ((threadIdx.x & 31) == 0) atomic_max_pos(a.maxdp, dpmax);
  }
}

// ----------------------------------------------------------------------- Coulomb

// g[i1][cs][n][e] = sum_i2 rho_e(i1,i2) {cos,sin}(2 pi n k2(i2))
__global__ void k_coul_rows(const double2* __restrict__ rho, int nk, int n1, int n2, int ntri, int ncut,
                            const double* __restrict__ t2c, const double* __restrict__ t2s, double2* __restrict__ g) {
  const int i1 = blockIdx.x;
  const int nout = 2 * ncut * ntri;
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int e = o % ntri;
    const int cn = o / ntri;  // cs * ncut + n
    const int cs = cn / ncut, n = cn - cs * ncut;
    const double* t = (cs == 0 ? t2c : t2s) + (size_t)n * n2;
    const double2* r = rho + (size_t)e * nk + (size_t)i1 * n2;
    double sx = 0, sy = 0;
    for (int i2 = 0; i2 < n2; i2++) {
      const double2 v = r[i2];
      const double tv = t[i2];
      sx += v.x * tv;
      sy += v.y * tv;
    }
    g[((size_t)i1 * 2 * ncut + cn) * ntri + e] = cmk(sx, sy);
  }
}

// One block per (n, e): f_xy(m,n,e) over m, X_xy = combine(A,B,C,D) - X0,
// h(i1, {c,s}, n, e) = sum_m X t_m(i1).
__global__ void k_coul_modes(const double2* __restrict__ g, int n1, int ntri, int ncut, double invN,
                             const double* __restrict__ t1c, const double* __restrict__ t1s,
                             const double2* __restrict__ cA, const double2* __restrict__ cB,
                             const double2* __restrict__ cC, const double2* __restrict__ cD,
                             const double2* __restrict__ X0, const unsigned char* __restrict__ is_diag,
                             double2* __restrict__ h, double2* __restrict__ Xout, double2* __restrict__ fdiag,
                             const int* __restrict__ diag_of) {
  const int n = blockIdx.x, e = blockIdx.y;
  extern __shared__ double2 sm[];
  double2* f = sm;               // [4][ncut]: cc, cs, sc, ss
  double2* X = sm + 4 * ncut;    // [4][ncut]
  const double PI = 3.14159265358979323846;
  for (int o = threadIdx.x; o < 4 * ncut; o += blockDim.x) {
    const int xy = o / ncut, m = o - xy * ncut;
    const double* t = (xy < 2 ? t1c : t1s) + (size_t)m * n1;
    const int ycs = xy & 1;  // second letter: 0 = c (g cos), 1 = s (g sin)
    double sx = 0, sy = 0;
    for (int i1 = 0; i1 < n1; i1++) {
      const double2 v = g[((size_t)i1 * 2 * ncut + ycs * ncut + n) * ntri + e];
      sx += v.x * t[i1];
      sy += v.y * t[i1];
    }
    const double corr = -4 * PI * PI * (double)(m * m + n * n) * invN / 27.0;
    const double sc = invN * (1. + corr);
    f[o] = cmk(sx * sc, sy * sc);
  }
  __syncthreads();
  const bool dg = is_diag[e];
  for (int m = threadIdx.x; m < ncut; m += blockDim.x) {
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
  for (int o = threadIdx.x; o < 2 * n1; o += blockDim.x) {
    const int cs = o / n1, i1 = o - cs * n1;
    double2 acc = cz();
    // cs = 0: sum_m X_cc c_m + X_sc s_m ; cs = 1: sum_m X_cs c_m + X_ss s_m
    const double2* Xc = X + (cs == 0 ? 0 : 1) * ncut;
    const double2* Xs = X + (cs == 0 ? 2 : 3) * ncut;
    for (int m = 0; m < ncut; m++) {
      const double c = t1c[(size_t)m * n1 + i1], s = t1s[(size_t)m * n1 + i1];
      acc.x += Xc[m].x * c + Xs[m].x * s;
      acc.y += Xc[m].y * c + Xs[m].y * s;
    }
    h[((size_t)i1 * 2 * ncut + cs * ncut + n) * ntri + e] = acc;
  }
}

// ----------------------------------------------------------------------- observables

struct ObsPart {
  double pop[kMaxBands];
  double2 J1[3], J2[3];
  double pmax, pmin;
};

template <int N>
__global__ void __launch_bounds__(128) k_obs(DevTables tb, const DevConsts* __restrict__ cst, const double2* __restrict__ rho,
                                             const double2* __restrict__ hr, int want_current, ObsPart* __restrict__ part) {
  constexpr int NT = Tri<N>::NT;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = tb.nk;
  __shared__ ObsPart sp[128];
  ObsPart my;
  for (int i = 0; i < kMaxBands; i++) my.pop[i] = 0;
  for (int x = 0; x < 3; x++) my.J1[x] = my.J2[x] = cz();
  my.pmax = 0;
  my.pmin = 1.0;
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
    // populations in the eigenbasis: Re sum_ii conj(U[c][ii]) sum_jj P[ii][jj] U[c][jj]
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
    if (want_current) {
      // J1 = sum_ij P_ij GE_ij ; GE from the renormalised H when Coulomb is on
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
      // J2 = sum_{i,j,l} P[i][j] Hs[i][l] conj(D[j][l])
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
#pragma unroll
            for (int x = 0; x < 3; x++) {
              const double2 d = tb.D[(size_t)(x * NT + Tri<N>::idx(lo, hi)) * nk + k];
              my.J2[x] = cadd(my.J2[x], cmulc(ph, d));
            }
          }
        }
    }
  }
  sp[threadIdx.x] = my;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      ObsPart& d = sp[threadIdx.x];
      const ObsPart& o = sp[threadIdx.x + s];
      for (int i = 0; i < N; i++) d.pop[i] += o.pop[i];
      for (int x = 0; x < 3; x++) {
        d.J1[x] = cadd(d.J1[x], o.J1[x]);
        d.J2[x] = cadd(d.J2[x], o.J2[x]);
      }
      d.pmax = fmax(d.pmax, o.pmax);
      d.pmin = fmin(d.pmin, o.pmin);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sp[0];
}

// transient absorption: -2 sum_{i<nch<=j} D_ij P_ij (one block; tiny for nch=0 or 1)
__global__ void k_tabs(DevTables tb, const double2* __restrict__ rho, double2* __restrict__ out3) {
  __shared__ double2 s[3][256];
  double2 acc[3] = {cz(), cz(), cz()};
  const int n = tb.n, nk = tb.nk, ntri = tb.ntri;
  for (int k = threadIdx.x; k < nk; k += blockDim.x)
    for (int i = 0; i < tb.nch; i++)
      for (int j = tb.nch; j < n; j++) {
        const int e = tri_index(i, j, n);
        const double2 p = rho[(size_t)e * nk + k];
        for (int x = 0; x < 3; x++) acc[x] = csub(acc[x], cmul(cscale(tb.D[(size_t)(x * ntri + e) * nk + k], 2.), p));
      }
  for (int x = 0; x < 3; x++) s[x][threadIdx.x] = acc[x];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int x = 0; x < 3; x++) s[x][threadIdx.x] = cadd(s[x][threadIdx.x], s[x][threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int x = 0; x < 3; x++) out3[x] = s[x][0];
}

__global__ void k_obs_final(const ObsPart* __restrict__ part, int nparts, int n, int nbands, int nk, double scaleJ,
                            double scaleTA, const double2* __restrict__ tabs3, ObsRecord rec, ObsRecord* __restrict__ log,
                            double* __restrict__ ncond_dev, double* __restrict__ pcmax_dev) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  ObsPart t;
  for (int i = 0; i < kMaxBands; i++) t.pop[i] = 0;
  for (int x = 0; x < 3; x++) t.J1[x] = t.J2[x] = cz();
  t.pmax = 0;
  t.pmin = 1.0;
  for (int b = 0; b < nparts; b++) {
    const ObsPart& p = part[b];
    for (int i = 0; i < n; i++) t.pop[i] += p.pop[i];
    for (int x = 0; x < 3; x++) {
      t.J1[x] = cadd(t.J1[x], p.J1[x]);
      t.J2[x] = cadd(t.J2[x], p.J2[x]);
    }
    t.pmax = fmax(t.pmax, p.pmax);
    t.pmin = fmin(t.pmin, p.pmin);
  }
  const double inv = 1. / nk;
  double trace = -(double)nbands;
  double nc = 0;
  for (int i = 0; i < n; i++) {
    double v = t.pop[i] * inv;
    trace += v;
    if (i < nbands) v = 1.0 - v;
    rec.pop[i] = v;
    if (v > nc) nc = v;
  }
  for (int x = 0; x < 3; x++) {
    rec.J1[2 * x] = t.J1[x].x * scaleJ;
    rec.J1[2 * x + 1] = t.J1[x].y * scaleJ;
    rec.J2[x] = -2. * (t.J2[x].y * scaleJ);
    if (tabs3) {
      rec.tabs[2 * x] = tabs3[x].x * scaleTA * inv;
      rec.tabs[2 * x + 1] = tabs3[x].y * scaleTA * inv;
    }
  }
  rec.trace_dev = trace;
  rec.p_cond_max = t.pmax;
  rec.p_min = t.pmin;
  rec.n_cond = nc;
  if (log) *log = rec;
  if (ncond_dev) *ncond_dev = nc;
  if (pcmax_dev) *pcmax_dev = t.pmax;
}

// ----------------------------------------------------------------------- launchers

template <int N>
static cudaError_t launch_rhs_n(const DevTables& tb, const DevConsts* cst, const StageArgs& a, cudaStream_t s) {
  const int bs = 128;
  k_rhs<N><<<(tb.nk + bs - 1) / bs, bs, 0, s>>>(tb, cst, a);
  return cudaGetLastError();
}

cudaError_t launch_rhs(const DevTables& tb, const DevConsts* cst, const StageArgs& a, cudaStream_t s) {
  switch (tb.n) {
    case 1: return launch_rhs_n<1>(tb, cst, a, s);
    case 2: return launch_rhs_n<2>(tb, cst, a, s);
    case 3: return launch_rhs_n<3>(tb, cst, a, s);
    case 4: return launch_rhs_n<4>(tb, cst, a, s);
    case 5: return launch_rhs_n<5>(tb, cst, a, s);
    case 6: return launch_rhs_n<6>(tb, cst, a, s);
    case 8: return launch_rhs_n<8>(tb, cst, a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_coulomb(const DevTables& tb, const CoulDev& c, const double2* rho, double2* h, double2* Xout,
                           const double2* X0, cudaStream_t s) {
  k_coul_rows<<<tb.n1, 256, 0, s>>>(rho, tb.nk, tb.n1, tb.n2, tb.ntri, tb.ncut, c.t2c, c.t2s, c.g);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 grid(tb.ncut, tb.ntri);
  size_t smem = sizeof(double2) * 8 * tb.ncut;
  k_coul_modes<<<grid, 128, smem, s>>>(c.g, tb.n1, tb.ntri, tb.ncut, 1.0 / tb.nk, c.t1c, c.t1s, c.A, c.B, c.C, c.D, X0,
                                       c.is_diag, h, Xout, c.fdiag, c.diag_of);
  return cudaGetLastError();
}

template <int N>
static cudaError_t launch_obs_n(const DevTables& tb, const DevConsts* cst, const double2* rho, const double2* hr,
                                int want_current, ObsPart* part, cudaStream_t s) {
  k_obs<N><<<(tb.nk + 127) / 128, 128, 0, s>>>(tb, cst, rho, hr, want_current, part);
  return cudaGetLastError();
}

int obs_parts(int nk) { return (nk + 127) / 128; }
size_t obs_part_bytes() { return sizeof(ObsPart); }

cudaError_t launch_observables(const DevTables& tb, const DevConsts* cst, const double2* rho, const double2* hr,
                               int want_current, int want_tabs, void* part, double2* tabs3, double scaleJ,
                               double scaleTA, const ObsRecord& rec, ObsRecord* log, double* ncond_dev,
                               double* pcmax_dev, cudaStream_t s) {
  cudaError_t e;
  ObsPart* pp = (ObsPart*)part;
  switch (tb.n) {
    case 1: e = launch_obs_n<1>(tb, cst, rho, hr, want_current, pp, s); break;
    case 2: e = launch_obs_n<2>(tb, cst, rho, hr, want_current, pp, s); break;
    case 3: e = launch_obs_n<3>(tb, cst, rho, hr, want_current, pp, s); break;
    case 4: e = launch_obs_n<4>(tb, cst, rho, hr, want_current, pp, s); break;
    case 5: e = launch_obs_n<5>(tb, cst, rho, hr, want_current, pp, s); break;
    case 6: e = launch_obs_n<6>(tb, cst, rho, hr, want_current, pp, s); break;
    case 8: e = launch_obs_n<8>(tb, cst, rho, hr, want_current, pp, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  if (want_tabs && tb.nch > 0) {
    k_tabs<<<1, 256, 0, s>>>(tb, rho, tabs3);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k_obs_final<<<1, 32, 0, s>>>(pp, obs_parts(tb.nk), tb.n, tb.nbands, tb.nk, scaleJ, scaleTA,
                                (want_tabs && tb.nch > 0) ? tabs3 : nullptr, rec, log, ncond_dev, pcmax_dev);
  return cudaGetLastError();
}

}  // namespace edus
