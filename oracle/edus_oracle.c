/*
 * edus_oracle.c — CPU FP64 oracle: a plain-C restatement of the EDUS
 * k-space density-matrix propagation (anpicon/EDUS, C++14/OpenMP/MPI).
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path, never shipped).
 * Every function names the reference file:line it restates. The reference
 * itself needs MPI, Armadillo, LAPACK and FFTW (Makefile:1-13), so it is not
 * built here; its three LAPACK uses on this path (eig_sym, inv, pinv) are
 * replaced by a cyclic Jacobi eigensolver, Gauss–Jordan inversion and a
 * one-sided Jacobi SVD. The oracle is pinned against the shipped AB5
 * golden run (example/Adams–Bashforth ODE Solver example/AB5_.../Output).
 * Parity unpinned for the parts no shipped file covers: the tight-binding
 * models other than Haldane_CoreBN_Nedge and the Crystal interface (the
 * reference ships no crystal data).
 *
 * Layout: P[k][i][j] complex128 exactly as the reference's vec3x P0
 * (Source_Main/allocate_arr.cpp:39); Dipole[k][i][j][x] as vec4x Dipole.
 * k is parallelised with OpenMP; all arithmetic per k is sequential, and
 * every reduction over k uses a fixed per-thread block order so results do
 * not depend on the thread count.
 */
#define _POSIX_C_SOURCE 200809L
#include "edus_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* headers/Constants.h:14-36 */
static const double PI = 3.14159265358979323846;
static const double C_LIGHT = 137.036;
static const double TIME_AU_FS = 0.02418884326505;
static const double ENERGY_AU_EV = 27.211396;
#define ENERGY_EV_AU (1.0 / 27.211396)
static const double SPACE_AU_A = 0.52917721092;
#define SPACE_A_AU (1.0 / 0.52917721092)

#define MAXSH 32
#define MAXNB 256
/* reductions over k: fixed block partition (the golden run used 7 OpenMP
 * threads, main_MPI.cpp:109-125); block sums are combined in block order */
#define NBLK 7

struct orc {
  edus_params p;
  int ncv, nch, nv, nbands; /* nbands = Nch + Nv (filled bands) */
  int nk, n1, n2;
  double M[3][3], MI[3][3], jac;
  double det_a, dk[3];
  double *kpt;              /* [nk][3] */
  int nshell, shell_n[MAXSH];
  double weights[MAXSH];
  double bvec[MAXNB][3];    /* all b vectors, shell-major */
  int bshell[MAXNB];
  int nnb;
  int *nbr;                 /* [nk][nnb] */
  /* model tables */
  cplx *H, *U, *hU, *D, *GE; /* H,U [nk][n][n]; D,GE [nk][n][n][3] */
  /* Wannier */
  int nrpts;
  double *Rvec;             /* [nrpts][3] */
  cplx *HR, *xR, *yR, *zR;  /* [n][n][nrpts] as Hvv[i][j][iR] */
  /* tb model constants */
  double tb_a, tb_b, tb_g, tb_t2, tb_phi0, tb_core, tb_rchv, tb_rchc;
  double tb_c, tb_d, tb_f;  /* GeS hoppings; DLGraphene interlayer distance (c) and hopping (d) */
  int tb_kind;
  /* Crystal model: H, x and y Berry connections on the nkf x nkf file grid, [i][j][k1][k2], i >= j */
  int cy_nkf;
  cplx *cyH, *cyDx, *cyDy;
  /* dissipation */
  double T[EDUS_MAX_BANDS][EDUS_MAX_BANDS];
  int n_diss, diss_i[EDUS_MAX_BANDS * EDUS_MAX_BANDS], diss_j[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  /* state */
  cplx *P0, *P1, *P2, *Pv, *Pgrad;
  cplx *ring;               /* AB: [order][nk][n][n]; Taylor: [order][nk][n*n] */
  int ring_idx[16];
  double dt_prev[16];
  cplx *Pprev_diag;         /* P_W_prev diagonal [nk][n] */
  cplx *Psave_diag;         /* OMP_private.P0 diagonal [nk][n] */
  /* Coulomb */
  int ncut;
  cplx *cA, *cB, *cC, *cD;  /* [ncut^2][n^2] */
  cplx screen[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  double VH[EDUS_MAX_BANDS][EDUS_MAX_BANDS];
  cplx *Xcc, *Xcs, *Xsc, *Xss, *Xcc0, *Xcs0, *Xsc0, *Xss0; /* [ncut^2][n^2] */
  double EH[EDUS_MAX_BANDS], EH0[EDUS_MAX_BANDS];
  double *cos_m1, *sin_m1, *cos_m2, *sin_m2; /* [ncut][nk] */
  cplx *PW0;                /* P_Wannier_0 */
  cplx *Pd;                 /* diagonal basis: P in the eigenbasis [nk][n][n] */
  cplx *Hr;                 /* Hk_renorm [nk][n][n] */
  double n_cond_coul;       /* Coulomb_set.n_cond */
  /* time loop */
  int it, itfi;
  double time_loop, dt, dt0;
  double EF[2][3];
  int e_non0;
  double n_cond, P_cond_max, P_cond_max_loc, P_min;
  /* velocity gauge (an option the reference does not have): vector potential
   * A(t) = -int_t0^t E_pump, Cartesian, tracked up to time A_t */
  int vg;
  double A_t, A_cart[3];
};

#define IDX3(k, i, j, n) (((size_t)(k) * (n) + (i)) * (n) + (j))
#define IDX4(k, i, j, x, n) ((((size_t)(k) * (n) + (i)) * (n) + (j)) * 3 + (x))

static cplx cmul(cplx a, cplx b) { return a * b; }

/* ------------------------------------------------------------ small linear algebra */

/* 3x3 inverse by Gauss–Jordan with partial pivoting (Armadillo inv in
 * headers/Coordinate.h:68-93). */
static int inv_gj(int n, const double* A, double* Ainv) {
  double a[32 * 64];
  if (n > 32) return -1;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < 2 * n; j++) a[i * 2 * n + j] = (j < n) ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (fabs(a[r * 2 * n + c]) > fabs(a[piv * 2 * n + c])) piv = r;
    if (a[piv * 2 * n + c] == 0.0) return -1;
    if (piv != c)
      for (int j = 0; j < 2 * n; j++) {
        double t = a[c * 2 * n + j];
        a[c * 2 * n + j] = a[piv * 2 * n + j];
        a[piv * 2 * n + j] = t;
      }
    double d = a[c * 2 * n + c];
    for (int j = 0; j < 2 * n; j++) a[c * 2 * n + j] /= d;
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      double f = a[r * 2 * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; j++) a[r * 2 * n + j] -= f * a[c * 2 * n + j];
    }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) Ainv[i * n + j] = a[i * 2 * n + n + j];
  return 0;
}

static double det3(const double m[3][3]) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

/* Moore–Penrose pseudo-inverse times a vector via one-sided Jacobi SVD
 * (Armadillo pinv(A, 1e-16) * q, headers/CalculateWeigths.h:100). A is
 * rows x cols, row-major, cols <= MAXSH. */
static void pinv_solve(int rows, int cols, const double* A, const double* q, double tol, double* w) {
  double U[21 * MAXSH], V[MAXSH * MAXSH];
  memcpy(U, A, sizeof(double) * rows * cols);
  for (int i = 0; i < cols; i++)
    for (int j = 0; j < cols; j++) V[i * cols + j] = (i == j);
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0;
    for (int p = 0; p < cols; p++)
      for (int r = p + 1; r < cols; r++) {
        double alpha = 0, beta = 0, gamma = 0;
        for (int i = 0; i < rows; i++) {
          alpha += U[i * cols + p] * U[i * cols + p];
          beta += U[i * cols + r] * U[i * cols + r];
          gamma += U[i * cols + p] * U[i * cols + r];
        }
        if (gamma == 0.0) continue;
        double rel = fabs(gamma) / sqrt(alpha * beta);
        if (rel > off) off = rel;
        if (rel < 1e-17) continue;
        double zeta = (beta - alpha) / (2.0 * gamma);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < rows; i++) {
          double up = U[i * cols + p], ur = U[i * cols + r];
          U[i * cols + p] = c * up - s * ur;
          U[i * cols + r] = s * up + c * ur;
        }
        for (int i = 0; i < cols; i++) {
          double vp = V[i * cols + p], vr = V[i * cols + r];
          V[i * cols + p] = c * vp - s * vr;
          V[i * cols + r] = s * vp + c * vr;
        }
      }
    if (off < 1e-17) break;
  }
  /* singular values = column norms of U */
  double sv[MAXSH], ut_q[MAXSH];
  for (int j = 0; j < cols; j++) {
    double s2 = 0;
    for (int i = 0; i < rows; i++) s2 += U[i * cols + j] * U[i * cols + j];
    sv[j] = sqrt(s2);
    double d = 0;
    for (int i = 0; i < rows; i++) d += U[i * cols + j] * q[i];
    ut_q[j] = (sv[j] > tol) ? d / (sv[j] * sv[j]) : 0.0; /* (u_j/s_j)^T q / s_j */
  }
  for (int i = 0; i < cols; i++) {
    double acc = 0;
    for (int j = 0; j < cols; j++) acc += V[i * cols + j] * ut_q[j];
    w[i] = acc;
  }
}

/* Hermitian eigen-decomposition by cyclic complex Jacobi; eigenvalues
 * ascending, vectors in columns of Z (Armadillo eig_sym). A is n x n
 * row-major, overwritten. */
static void eig_herm(int n, cplx* A, double* evals, cplx* Z) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) Z[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, diag = 0;
    for (int i = 0; i < n; i++) {
      diag += creal(A[i * n + i]) * creal(A[i * n + i]);
      for (int j = i + 1; j < n; j++) off += creal(A[i * n + j] * conj(A[i * n + j]));
    }
    if (off <= 1e-34 * (diag + 1e-300)) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        cplx apq = A[p * n + q];
        double mag = cabs(apq);
        if (mag < 1e-300) continue;
        double app = creal(A[p * n + p]), aqq = creal(A[q * n + q]);
        cplx ph = apq / mag; /* e^{i phi} */
        double theta = 0.5 * atan2(2.0 * mag, aqq - app);
        double c = cos(theta), s = sin(theta);
        /* rotation R acting on columns p,q: col_p' = c col_p - s conj(ph) col_q? use unitary
           G = [[c, s*ph],[-s*conj(ph), c]] so that (G^H A G)_{pq} = 0 */
        for (int k = 0; k < n; k++) { /* A <- A G */
          cplx akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * conj(ph) * akq;
          A[k * n + q] = s * ph * akp + c * akq;
        }
        for (int k = 0; k < n; k++) { /* A <- G^H A */
          cplx apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * ph * aqk;
          A[q * n + k] = s * conj(ph) * apk + c * aqk;
        }
        A[p * n + q] = 0;
        A[q * n + p] = 0;
        A[p * n + p] = creal(A[p * n + p]);
        A[q * n + q] = creal(A[q * n + q]);
        for (int k = 0; k < n; k++) {
          cplx zkp = Z[k * n + p], zkq = Z[k * n + q];
          Z[k * n + p] = c * zkp - s * conj(ph) * zkq;
          Z[k * n + q] = s * ph * zkp + c * zkq;
        }
      }
  }
  /* sort ascending */
  int ord[EDUS_MAX_BANDS];
  double ev[EDUS_MAX_BANDS];
  for (int i = 0; i < n; i++) {
    ord[i] = i;
    ev[i] = creal(A[i * n + i]);
  }
  for (int i = 1; i < n; i++) {
    int t = ord[i], j = i;
    while (j > 0 && ev[ord[j - 1]] > ev[t]) {
      ord[j] = ord[j - 1];
      j--;
    }
    ord[j] = t;
  }
  cplx Zs[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  for (int j = 0; j < n; j++) {
    evals[j] = ev[ord[j]];
    for (int i = 0; i < n; i++) Zs[i * n + j] = Z[i * n + ord[j]];
  }
  memcpy(Z, Zs, sizeof(cplx) * n * n);
}

/* ------------------------------------------------------------ coordinates */

/* headers/Coordinate.h:68-93 (set_crys_to_cart) */
static int set_crys_to_cart(orc* o) {
  double Mf[9], MIf[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      o->M[i][j] = o->p.b[j][i];
      Mf[i * 3 + j] = o->M[i][j];
    }
  if (inv_gj(3, Mf, MIf)) return EDUS_EINVAL;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o->MI[i][j] = MIf[i * 3 + j];
  o->jac = fabs(det3(o->M));
  return 0;
}

/* headers/Coordinate.h:133-149 (setcrys) */
static void crys_to_cart(const orc* o, const double* c, double* x) {
  for (int i = 0; i < 3; i++) {
    x[i] = 0.0;
    for (int j = 0; j < 3; j++) x[i] += o->M[i][j] * c[j];
  }
}
/* headers/Coordinate.h:120-128 (setcart) */
static void cart_to_crys(const orc* o, const double* x, double* c) {
  for (int i = 0; i < 3; i++) c[i] = o->MI[i][0] * x[0] + o->MI[i][1] * x[1] + o->MI[i][2] * x[2];
}

/* ------------------------------------------------------------ grid & stencil */

/* headers/InitParameters.h:13-40 (BZ_parameters k grid); with nkpt read the
 * listed points (headers/ReadInput.h:429-437) */
static int make_grid(orc* o) {
  const int* Nk = o->p.nk;
  for (int c = 0; c < 3; c++) o->dk[c] = 1.0 / Nk[c];
  if (o->p.kpt_read) {
    FILE* f = fopen(o->p.input_path, "r");
    if (!f) return EDUS_EIO;
    fseek(f, (long)o->p.kpt_offset, SEEK_SET);
    for (int ik = 0; ik < o->nk; ik++)
      if (fscanf(f, "%lf %lf %lf", &o->kpt[ik * 3], &o->kpt[ik * 3 + 1], &o->kpt[ik * 3 + 2]) != 3) {
        fclose(f);
        return EDUS_EPARSE;
      }
    fclose(f);
    return 0;
  }
  for (int ik = 0; ik < o->nk; ik++) {
    int iik[3] = {(ik / (Nk[2] * Nk[1])) % Nk[0], (ik / Nk[2]) % Nk[1], ik % Nk[2]};
    for (int c = 0; c < 3; c++) o->kpt[ik * 3 + c] = (o->dk[c] != 1.0) ? -0.5 + o->dk[c] * iik[c] : 0.0;
  }
  return 0;
}

/* headers/CalculateWeigths.h:1-138 (b-vector shells and weights) */
static int calc_weights(orc* o) {
  int plane = -1;
  for (int i = 0; i < 3; i++)
    if (o->p.nk[i] == 1) plane = i;
  double mins[MAXSH + 2];
  int nmin = 1;
  mins[0] = 1.e-08;
  int enough = 0;
  o->nshell = 0;
  o->nnb = 0;
  while (!enough) {
    mins[nmin++] = 1000.;
    for (int ik = 0; ik < o->nk; ik++) {
      double x[3];
      crys_to_cart(o, &o->kpt[ik * 3], x);
      double nrm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
      int in = 0;
      for (int i = 0; i < nmin - 1; i++) in = in || (nrm <= mins[i] + 1.e-11);
      if (!in && nrm < mins[nmin - 1]) mins[nmin - 1] = nrm;
    }
    int s = o->nshell++;
    o->shell_n[s] = 0;
    for (int ik = 0; ik < o->nk; ik++) {
      double x[3];
      crys_to_cart(o, &o->kpt[ik * 3], x);
      double nrm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
      if (fabs(nrm - mins[nmin - 1]) < 1.e-11) {
        if (o->nnb >= MAXNB) return EDUS_EINVAL;
        memcpy(o->bvec[o->nnb], x, sizeof(x));
        o->bshell[o->nnb] = s;
        o->nnb++;
        o->shell_n[s]++;
      }
    }
    int ns = o->nshell;
    double A[21 * MAXSH];
    memset(A, 0, sizeof(A));
    int base = 0;
    for (int sh = 0; sh < ns; sh++) {
      int row = 0;
      for (int id = 0; id < 3; id++)
        if (id != plane) {
          for (int b = base; b < base + o->shell_n[sh]; b++) A[row * ns + sh] += o->bvec[b][id] * o->bvec[b][id];
          row++;
        }
      for (int id = 0; id < 3; id++)
        for (int jd = id + 1; jd < 3; jd++)
          if (id != plane && jd != plane) {
            for (int b = base; b < base + o->shell_n[sh]; b++) A[row * ns + sh] += o->bvec[b][id] * o->bvec[b][jd];
            row++;
          }
      row = 5;
      for (int id = 0; id < 3; id++)
        for (int jd = id; jd < 3; jd++)
          for (int ld = jd; ld < 3; ld++)
            for (int md = ld; md < 3; md++) {
              for (int b = base; b < base + o->shell_n[sh]; b++)
                A[row * ns + sh] += o->bvec[b][id] * o->bvec[b][jd] * o->bvec[b][ld] * o->bvec[b][md];
              row++;
            }
      base += o->shell_n[sh];
    }
    double q[21];
    memset(q, 0, sizeof(q));
    q[0] = 1;
    q[1] = 1;
    q[2] = !(plane + 1);
    double w[MAXSH];
    pinv_solve(21, ns, A, q, 1.e-16, w);
    double r2 = 0;
    for (int r = 0; r < 21; r++) {
      double acc = 0;
      for (int sh = 0; sh < ns; sh++) acc += A[r * ns + sh] * w[sh];
      r2 += (acc - q[r]) * (acc - q[r]);
    }
    for (int sh = 0; sh < ns; sh++) o->weights[sh] = w[sh];
    enough = sqrt(r2) < 1.e-07;
    if (o->nshell == 32 && !enough) return EDUS_EINVAL;
  }
  return 0;
}

/* headers/CalculateWeigths.h:145-226 (CalculateIndices: k+b lookup) */
static int calc_indices(orc* o) {
  int bad = 0;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++) {
    double kk[3];
    crys_to_cart(o, &o->kpt[ik * 3], kk);
    for (int b = 0; b < o->nnb; b++) {
      double x[3] = {kk[0] + o->bvec[b][0], kk[1] + o->bvec[b][1], kk[2] + o->bvec[b][2]};
      double c[3];
      cart_to_crys(o, x, c);
      for (int i = 0; i < 3; i++) c[i] = fmod(c[i] + 0.5, 1.) - 0.5;
      /* candidate from grid arithmetic, verified with the reference's test */
      int found = -1;
      int cand[3];
      for (int i = 0; i < 3; i++) {
        int N = o->p.nk[i];
        if (N == 1) {
          cand[i] = 0;
          continue;
        }
        long r = lround((c[i] + 0.5) * N);
        cand[i] = (int)(((r % N) + N) % N);
      }
      int ck = (cand[0] * o->p.nk[1] + cand[1]) * o->p.nk[2] + cand[2];
      /* a listed grid: the reference's linear search only (first match in list order) */
      for (int pass = o->p.kpt_read ? 1 : 0; pass < 2 && found < 0; pass++) {
        int lo = pass == 0 ? ck : 0, hi = pass == 0 ? ck + 1 : o->nk;
        for (int k1 = lo; k1 < hi; k1++) {
          int ok = 1;
          for (int i = 0; i < 3 && ok; i++) {
            double d = c[i] - o->kpt[k1 * 3 + i];
            ok = fabs(d) < 1.e-08 || fabs(d - 1.) < 1.e-08 || fabs(d + 1.) < 1.e-08;
          }
          if (ok) {
            found = k1;
            break;
          }
        }
      }
      if (found < 0) {
#pragma omp atomic write
        bad = 1;
        found = ik;
      }
      o->nbr[(size_t)ik * o->nnb + b] = found;
    }
  }
  return bad ? EDUS_EINVAL : 0;
}

/* ------------------------------------------------------------ TB models */

enum {
  TB_HALDANE_N = 1,
  TB_HALDANE_B,
  TB_GEN2D,
  TB_BN,
  TB_COREBN_N,
  TB_COREBN_B,
  TB_GRAPHENE,
  TB_COREGRAPHENE,
  TB_GRAPHENE_COSTD,
  TB_GRAPHENE_SYMD,
  TB_GRAPHENE_ZURRON,
  TB_BN1B,
  TB_VAMPA,
  TB_GES,
  TB_DLGRAPHENE
};

/* headers/TightBinding.h:98-122: Vampa2015 cosine-series coefficients [band][axis][j] */
static const double VAMPA[2][3][6] = {
    {{-0.0928, 0.0705, 0.0200, -0.0012, 0.0029, 0.0006}, {-0.0307, 0.0307, 0, 0, 0, 0}, {-0.0059, 0.0059, 0, 0, 0, 0}},
    {{0.0898, -0.0814, -0.0024, -0.0048, -0.0003, -0.0009}, {0.1147, -0.1147, 0, 0, 0, 0}, {0.0435, -0.0435, 0, 0, 0, 0}}};

/* headers/TightBinding.h:43-173 (init / set_hopping) for the models built here */
static int tb_init(orc* o) {
  const char* nm = o->p.tb_type;
  double eV = ENERGY_EV_AU;
  o->tb_a = 2.5 * SPACE_A_AU;
  o->tb_b = 3.16 * eV;
  o->tb_g = 6.2 * eV;
  o->tb_t2 = 0;
  o->tb_phi0 = 0;
  if (!strcmp(nm, "Haldane_CoreBN_Nedge") || !strcmp(nm, "Haldane_CoreBN_Bedge")) {
    o->tb_kind = !strcmp(nm, "Haldane_CoreBN_Nedge") ? TB_HALDANE_N : TB_HALDANE_B;
    o->tb_g = o->p.hopping[0];
    o->tb_b = o->p.hopping[1];
    o->tb_t2 = o->p.hopping[2];
    o->tb_phi0 = o->p.hopping[3];
  } else if (!strcmp(nm, "gen2d_hexagonal")) {
    o->tb_kind = TB_GEN2D;
    o->tb_a = o->p.hopping[0];
    o->tb_g = o->p.hopping[1];
    o->tb_b = o->p.hopping[2];
    o->tb_t2 = o->p.hopping[3];
    o->tb_phi0 = o->p.hopping[4];
    o->tb_core = o->p.hopping[5];
    o->tb_rchv = o->p.hopping[6];
    o->tb_rchc = o->p.hopping[7];
  } else if (!strcmp(nm, "BoronNitride")) {
    o->tb_kind = TB_BN;
  } else if (!strcmp(nm, "BN1b")) {
    o->tb_kind = TB_BN1B;
  } else if (!strcmp(nm, "Vampa2015")) {
    o->tb_kind = TB_VAMPA;
    o->tb_g = 0.1213;
  } else if (!strcmp(nm, "GeS") || !strcmp(nm, "GeS_HSE06")) {
    /* TightBinding.h:135-154 */
    int hse = !strcmp(nm, "GeS_HSE06");
    o->tb_kind = TB_GES;
    o->tb_g = (hse ? 0.62 : 0.41) * eV;
    o->tb_f = (hse ? 2.91 : -2.33) * eV;
    o->tb_t2 = (hse ? -0.797 : 0.61) * eV;
    o->tb_b = (hse ? -0.05 : 0.13) * eV;
    o->tb_c = (hse ? -0.14 : 0.07) * eV;
    o->tb_d = (hse ? 0.106 : -0.09) * eV;
  } else if (!strcmp(nm, "DLGraphene")) {
    /* TightBinding.h:90-97 */
    o->tb_kind = TB_DLGRAPHENE;
    o->tb_a = 2.46 * SPACE_A_AU;
    o->tb_b = 2.97 * eV;
    o->tb_c = 3.35 * SPACE_A_AU;
    o->tb_d = 0.39 * eV;
    o->tb_g = 0;
  } else if (!strcmp(nm, "CoreBN_Nedge") || !strcmp(nm, "CoreBN_Bedge")) {
    o->tb_kind = !strcmp(nm, "CoreBN_Nedge") ? TB_COREBN_N : TB_COREBN_B;
  } else if (!strcmp(nm, "Graphene") || !strcmp(nm, "CoreGraphene") || !strcmp(nm, "Graphene_costD") ||
             !strcmp(nm, "Graphene_symmetricD") || !strcmp(nm, "GrapheneZurron")) {
    /* TightBinding.h:48-80: a = 2.46 A, b = 2.97 eV, no gap */
    o->tb_kind = !strcmp(nm, "Graphene")         ? TB_GRAPHENE
                 : !strcmp(nm, "CoreGraphene")   ? TB_COREGRAPHENE
                 : !strcmp(nm, "Graphene_costD") ? TB_GRAPHENE_COSTD
                 : !strcmp(nm, "GrapheneZurron") ? TB_GRAPHENE_ZURRON
                                                 : TB_GRAPHENE_SYMD;
    o->tb_a = 2.46 * SPACE_A_AU;
    o->tb_b = 2.97 * eV;
    o->tb_g = 0;
  } else {
    return EDUS_EUNSUPPORTED;
  }
  return 0;
}

static cplx cexpi(double phase) { return cos(phase) + I * sin(phase); }

/* headers/TightBinding.h:271-290 (BoronNitride) and :387-440 (Haldane family) */
static cplx tb_energy(const orc* o, int ic, int jc, const double* k) {
  double g = o->tb_g, b = o->tb_b, t2 = o->tb_t2, phi0 = o->tb_phi0;
  double k1 = k[1], k2 = k[2];
  if (o->tb_kind == TB_COREBN_N || o->tb_kind == TB_COREBN_B) {
    /* TightBinding.h:177-207 */
    cplx f = (1. + cexpi(2. * PI * k1)) + cexpi(2. * PI * k2);
    if (ic == 0) return jc == 0 ? (o->tb_kind == TB_COREBN_N ? -15.06 : -6.91) : 0;
    if (ic == 1) return jc == 1 ? -g / 2. : (jc == 2 ? b * conj(f) : 0);
    if (ic == 2) return jc == 1 ? b * f : (jc == 2 ? g / 2. : 0);
    return 0;
  }
  if (o->tb_kind == TB_BN1B) {
    /* TightBinding.h:307-311 */
    cplx f = (cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2);
    return 0.5 * creal(csqrt(g * g + 4. * b * b * f * conj(f)));
  }
  if (o->tb_kind == TB_DLGRAPHENE) {
    /* TightBinding.h:291-312 */
    if (ic == jc) return 0.;
    cplx f = (cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2);
    if ((ic == 0 && jc == 1) || (ic == 2 && jc == 3)) return conj(f) * b;
    if ((ic == 1 && jc == 0) || (ic == 3 && jc == 2)) return f * b;
    if ((ic == 3 && jc == 0) || (ic == 0 && jc == 3)) return o->tb_d;
    return 0.;
  }
  if (o->tb_kind == TB_VAMPA) {
    /* TightBinding.h:312-326 */
    if (ic != jc) return 0.;
    cplx e = 0.;
    for (int x = 0; x < 3; x++)
      for (int j = 0; j < 6; j++) e += VAMPA[ic][x][j] * cos(j * k[x]);
    if (ic == 1) e += g;
    return e;
  }
  if (o->tb_kind == TB_GES) {
    /* TightBinding.h:441-462 */
    if (ic == jc) {
      double tor = -2. * o->tb_c * (cos(2. * PI * k1) + cos(2. * PI * k2)) - 2. * o->tb_d * (cos(2. * PI * (k1 - k2)));
      return ic == 0 ? g + tor : -g + tor;
    }
    cplx phix = cexpi(2. * PI * k1) + cexpi(2. * PI * k2);
    cplx tor = -o->tb_f - t2 * phix - b * conj(phix);
    return ic == 0 ? conj(tor) : tor;
  }
  if (o->tb_kind == TB_GRAPHENE_COSTD || o->tb_kind == TB_GRAPHENE_SYMD) {
    /* TightBinding.h:225-239 */
    if (ic == jc && ic < 2) return -10.892178;
    if (ic >= 2 && jc >= 2 && ic == jc) {
      double modf = cabs((cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2));
      return ic == 2 ? -b * modf : b * modf;
    }
    return 0.;
  }
  if (o->tb_kind == TB_GRAPHENE_ZURRON) {
    /* TightBinding.h:257-269, with the Cartesian k */
    if (ic == jc) return 0.;
    double kc[3];
    crys_to_cart(o, k, kc);
    double a = o->tb_a;
    cplx f = cexpi(-a * kc[1] / sqrt(3.)) * (1. + 2. * cexpi(sqrt(3.) * a * kc[1] / 2.) * cos(a * kc[2] / 2.));
    return ic == 0 ? f * b : conj(f) * b;
  }
  if (o->tb_kind == TB_GRAPHENE) {
    /* TightBinding.h:209-222 */
    if (ic == jc) return 0.;
    cplx f = (cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2);
    return ic == 0 ? conj(f) * b : f * b;
  }
  if (o->tb_kind == TB_COREGRAPHENE) {
    /* TightBinding.h:241-255 */
    if (ic == jc && ic < 2) return -10.892178;
    if (ic >= 2 && jc >= 2 && ic != jc) {
      cplx f = (cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2);
      return ic == 2 ? conj(f) * b : f * b;
    }
    return 0.;
  }
  if (o->tb_kind == TB_BN) {
    if (ic == jc) return ic == 0 ? -g / 2 : (ic == 1 ? g / 2 : 0);
    cplx f = (cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2);
    return ic == 0 ? conj(f) * b : f * b;
  }
  if (ic == 0) {
    if (jc != 0) return 0;
    if (o->tb_kind == TB_HALDANE_N) return -15.06;
    if (o->tb_kind == TB_HALDANE_B) return -6.91;
    return o->tb_core;
  }
  if (ic == 1) {
    if (jc == 1) {
      cplx f2 = cexpi(2. * PI * k1 - 2. * PI * k2) + cexpi(2. * PI * k2) + cexpi(-2. * PI * k1);
      return -g / 2. + 2. * creal(t2 * cexpi(phi0) * f2);
    }
    if (jc == 2) {
      cplx f = 1. + cexpi(-2. * PI * k1) + cexpi(-2. * PI * k2);
      return b * f;
    }
    return 0;
  }
  if (ic == 2) {
    if (jc == 1) {
      cplx f = 1. + cexpi(-2. * PI * k1) + cexpi(-2. * PI * k2);
      return b * conj(f);
    }
    if (jc == 2) {
      cplx f2 = cexpi(2. * PI * k1 - 2. * PI * k2) + cexpi(2. * PI * k2) + cexpi(-2. * PI * k1);
      return g / 2. + 2. * creal(t2 * cexpi(-phi0) * f2);
    }
  }
  return 0;
}

/* headers/TightBinding.h:920-1003 (unitary) */
static cplx tb_unitary(const orc* o, int ic, int jc, const double* k) {
  double g = o->tb_g, b = o->tb_b, t2 = o->tb_t2, phi0 = o->tb_phi0;
  double k1 = k[1], k2 = k[2];
  if (o->tb_kind == TB_COREBN_N || o->tb_kind == TB_COREBN_B) {
    /* TightBinding.h:894-921 */
    if (ic == 0) return jc == 0 ? 1. : 0.;
    if (jc == 0) return 0.;
    cplx f = (1. + cexpi(2. * PI * k1)) + cexpi(2. * PI * k2);
    double E = creal(csqrt(g * g + 4. * b * b * f * conj(f))) / 2.;
    double a = sqrt((g + 2. * E) / (4. * E));
    double h = sqrt((2. * E - g) / (4. * E));
    if (ic == 1) return jc == 1 ? (cplx)a : -h * conj(f) / cabs(f);
    if (ic == 2) return jc == 1 ? (cplx)h : a * conj(f) / cabs(f);
    return 0.;
  }
  if (o->tb_kind == TB_GRAPHENE_COSTD || o->tb_kind == TB_GRAPHENE_SYMD || o->tb_kind == TB_BN1B || o->tb_kind == TB_VAMPA)
    return ic == jc ? 1. : 0.; /* :1064-1070, 1147-1155 */
  if (o->tb_kind == TB_DLGRAPHENE) {
    /* TightBinding.h:1083-1145: rows 0 and 3 normalised by n1, rows 1 and 2 by n2 */
    double d = o->tb_d;
    cplx f = (cexpi(2. * PI * k1) + 1.) + cexpi(2. * PI * k2);
    cplx s = csqrt(pow(d, 2) + 4 * pow(b, 2) * f * conj(f));
    double n1 = sqrt(8 + pow(cabs((d - s) / (b * conj(f))), 2) + 16 * pow(cabs((b * f) / (d + s)), 2));
    double n2 = sqrt(8 + 16 * pow(cabs((b * f) / (d - s)), 2) + pow(cabs((d + s) / (b * conj(f))), 2));
    double nr = (ic == 0 || ic == 3) ? n1 : n2;
    if (jc == 0) return (ic == 0 || ic == 2) ? -2 / nr : 2 / nr;
    if (jc == 3) return 2 / nr;
    if (jc == 1) {
      if (ic == 0 || ic == 3) return (-d + conj(s)) / (b * f * nr);
      return -((d + conj(s)) / (b * f * nr));
    }
    if (ic == 0) return (-4 * b * f) / (nr * (d + conj(s)));
    if (ic == 1) return (4 * b * f) / (nr * (d - conj(s)));
    if (ic == 2) return (-4 * b * f) / (nr * (d - conj(s)));
    return (4 * b * f) / (nr * (d + conj(s)));
  }
  if (o->tb_kind == TB_GES) {
    /* TightBinding.h:1005-1030 */
    cplx phix = cexpi(2. * PI * k1) + cexpi(2. * PI * k2);
    cplx tor = -o->tb_f - t2 * phix - b * conj(phix);
    double Bx = creal(tor), By = cimag(tor), Bz = g;
    double B = sqrt(Bx * Bx + By * By + Bz * Bz);
    double phi = atan2(By, Bx) / 2.;
    double costh2 = sqrt((B + Bz) / 2. / B), sinth2 = sqrt((B - Bz) / 2. / B);
    if (ic == 0) return jc == 0 ? cexpi(phi) * sinth2 : -cexpi(-phi) * costh2;
    return jc == 0 ? cexpi(phi) * costh2 : cexpi(-phi) * sinth2;
  }
  if (o->tb_kind == TB_GRAPHENE_ZURRON) {
    /* TightBinding.h:1072-1081 */
    if (jc != 1) return 1. / sqrt(2.);
    double kc[3];
    crys_to_cart(o, k, kc);
    double a = o->tb_a;
    cplx f = cexpi(-a * kc[1] / sqrt(3.)) * (1. + 2. * cexpi(sqrt(3.) * a * kc[1] / 2.) * cos(a * kc[2] / 2.));
    return ic == 0 ? -f / (sqrt(2.) * cabs(f)) : f / (sqrt(2.) * cabs(f));
  }
  if (o->tb_kind == TB_GRAPHENE || o->tb_kind == TB_COREGRAPHENE) {
    /* TightBinding.h:1032-1059 */
    int off2 = o->tb_kind == TB_COREGRAPHENE ? 2 : 0;
    if (ic < off2) return ic == jc ? 1. : 0.;
    if (jc == off2 + 1) {
      cplx f = (cexpi(-2. * PI * k1) + 1.) + cexpi(-2. * PI * k2);
      return ic == off2 ? -f / (sqrt(2.) * cabs(f)) : f / (sqrt(2.) * cabs(f));
    }
    if (jc == off2) return 1. / sqrt(2.);
    return 0.;
  }
  int off = 0;
  if (o->tb_kind != TB_BN) {
    if (ic == 0) return jc == 0 ? 1. : 0.;
    if (jc == 0) return 0.;
    off = 1;
  }
  double Bx = b * (1. + cos(2. * PI * k1) + cos(2. * PI * k2));
  double By = b * (sin(2. * PI * k1) + sin(2. * PI * k2));
  double Bz = -g / 2.;
  if (o->tb_kind != TB_BN) Bz = -g / 2. - 2. * t2 * sin(phi0) * (sin(-2. * PI * k2 + 2. * PI * k1) + sin(2. * PI * k2) + sin(-2. * PI * k1));
  double B = sqrt(Bx * Bx + By * By + Bz * Bz);
  double phi = atan2(By, Bx) / 2.;
  double costh2 = sqrt((B + Bz) / 2. / B);
  double sinth2 = sqrt((B - Bz) / 2. / B);
  int i = ic - off, j = jc - off;
  if (i == 0) return j == 0 ? cexpi(phi) * sinth2 : -cexpi(-phi) * costh2;
  if (i == 1) return j == 0 ? cexpi(phi) * costh2 : cexpi(-phi) * sinth2;
  return 0;
}

/* headers/TightBinding.h:1256-1421 (dipolex/y/z) */
static cplx tb_dipole(const orc* o, int ic, int jc, int x) {
  double a = o->tb_a;
  switch (o->tb_kind) {
    case TB_HALDANE_N:
      if (x == 0) return ((ic == 0 && jc == 1) || (ic == 1 && jc == 0)) ? 0.0697595094 : 0.;
      if (x == 1) return (ic == 2 && jc == 2) ? a / sqrt(3.) : 0.;
      return 0.;
    case TB_HALDANE_B:
      if (x == 0) return ((ic == 0 && jc == 2) || (ic == 2 && jc == 0)) ? 0.0869151662 : 0.;
      if (x == 1) return ((ic == 2 && jc == 2) || (ic == 0 && jc == 0)) ? a / sqrt(3.) : 0.;
      return 0.;
    case TB_GEN2D:
      if (x == 0) {
        if ((ic == 0 && jc == 1) || (ic == 1 && jc == 0)) return o->tb_rchv;
        if ((ic == 0 && jc == 2) || (ic == 2 && jc == 0)) return o->tb_rchc;
        return 0.;
      }
      if (x == 1) {
        if (ic == 2 && jc == 2) return -a / sqrt(3.);
        if (ic == 0 && jc == 0 && fabs(o->tb_rchc) > 1.e-6) return -a / sqrt(3.);
        return 0.;
      }
      return 0.;
    case TB_BN:
      if (x == 1) return (ic == 1 && jc == 1) ? a / sqrt(3) : 0.;
      return 0.;
    case TB_COREBN_N:
      if (x == 0) return ((ic == 0 && jc == 1) || (ic == 1 && jc == 0)) ? 0.0697595094 : 0.;
      if (x == 1) return (ic == 2 && jc == 2) ? a / sqrt(3.) : 0.;
      return 0.;
    case TB_COREBN_B:
      if (x == 0) return ((ic == 0 && jc == 2) || (ic == 2 && jc == 0)) ? 0.0869151662 : 0.;
      if (x == 1) return ((ic == 2 && jc == 2) || (ic == 0 && jc == 0)) ? a / sqrt(3.) : 0.;
      return 0.;
    case TB_GRAPHENE:
      if (x == 1) return (ic == 1 && jc == 1) ? -2.68341111 : 0.;
      return 0.;
    case TB_GRAPHENE_COSTD:
    case TB_GRAPHENE_SYMD: {
      /* TightBinding.h:1272-1283, 1349-1357, 1401-1405 */
      if (x == 0) {
        cplx dx = 0.0780088 / sqrt(2.);
        if (ic <= 1 && jc > 1) return (ic == 0 || (ic == 1 && jc == 2)) ? dx : -dx;
        if (ic > 1 && jc <= 1) return conj((jc == 0 || (jc == 1 && ic == 2)) ? dx : -dx);
        return 0.;
      }
      if (x == 2 && o->tb_kind == TB_GRAPHENE_COSTD) return 0.;
      if (ic == 1 && jc == 1) return -2.68341111;
      if (ic > 1 && jc > 1) return ic == jc ? -2.68341111 / 2 : 2.68341111 / 2;
      return 0.;
    }
    case TB_GRAPHENE_ZURRON:
    case TB_BN1B:
      return 0.;
    case TB_DLGRAPHENE:
      /* TightBinding.h:1300-1308, 1376-1385, 1404-1413 */
      if (ic != jc) return 0.;
      if (x == 0) return (ic == 2 || ic == 3) ? o->tb_c : 0.;
      if (x == 1) return ic == 1 ? -a / sqrt(3) : ((ic == 2 || ic == 3) ? a / (2 * sqrt(3)) : 0.);
      return ic == 2 ? a / 2. : (ic == 3 ? -a / 2. : 0.);
    case TB_VAMPA:
      if (ic == jc) return 0.;
      return x == 2 ? 3.94 : 3.46;
    case TB_GES:
      return (x == 1 && ic == 1 && jc == 1) ? 0.52 * SPACE_A_AU : 0.;
    case TB_COREGRAPHENE:
      if (x == 0)
        return ((ic == 0 && jc == 2) || (ic == 1 && jc == 3) || (ic == 2 && jc == 0) || (ic == 3 && jc == 1)) ? 0.0780088 : 0.;
      if (x == 1) return (ic == jc && ic % 2 == 1) ? -2.68341111 : 0.;
      return 0.;
  }
  return 0.;
}

/* ------------------------------------------------------------ Wannier model */

/* headers/Wannier.h:47-148 (_tb.dat reader, Nch = 0) */
static int wannier_read(orc* o, const char* workdir) {
  char path[2 * EDUS_STRLEN + 16];
  snprintf(path, sizeof(path), "%s/%s_tb.dat", workdir ? workdir : ".", o->p.ref_coord);
  FILE* f = fopen(path, "r");
  if (!f) return EDUS_EIO;
  char line[4096];
  for (int i = 0; i < 4; i++)
    if (!fgets(line, sizeof(line), f)) goto fail;
  int nw, nr;
  if (fscanf(f, "%d %d", &nw, &nr) != 2) goto fail;
  if (nw != o->ncv) goto fail;
  o->nrpts = nr;
  int n = nw;
  double* ndeg = malloc(sizeof(double) * nr);
  o->Rvec = malloc(sizeof(double) * 3 * nr);
  o->HR = calloc((size_t)n * n * nr, sizeof(cplx));
  o->xR = calloc((size_t)n * n * nr, sizeof(cplx));
  o->yR = calloc((size_t)n * n * nr, sizeof(cplx));
  o->zR = calloc((size_t)n * n * nr, sizeof(cplx));
  for (int i = 0; i < nr; i++)
    if (fscanf(f, "%lf", &ndeg[i]) != 1) goto fail2;
  for (int iR = 0; iR < nr; iR++) {
    if (fscanf(f, "%lf %lf %lf", &o->Rvec[iR * 3], &o->Rvec[iR * 3 + 1], &o->Rvec[iR * 3 + 2]) != 3) goto fail2;
    for (int in = 0; in < n; in++)
      for (int im = 0; im < n; im++) {
        int t1, t2;
        double hr, hi;
        if (fscanf(f, "%d %d %lf %lf", &t1, &t2, &hr, &hi) != 4) goto fail2;
        o->HR[((size_t)im * n + in) * nr + iR] = hr / ndeg[iR] * ENERGY_EV_AU + I * (hi / ndeg[iR] * ENERGY_EV_AU);
      }
  }
  for (int iR = 0; iR < nr; iR++) {
    double R[3];
    if (fscanf(f, "%lf %lf %lf", &R[0], &R[1], &R[2]) != 3) goto fail2;
    for (int in = 0; in < n; in++)
      for (int im = 0; im < n; im++) {
        int t1, t2;
        double v[6];
        if (fscanf(f, "%d %d %lf %lf %lf %lf %lf %lf", &t1, &t2, &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]) != 8) goto fail2;
        size_t id = ((size_t)im * n + in) * nr + iR;
        o->xR[id] = v[0] / ndeg[iR] * SPACE_A_AU + I * (v[1] / ndeg[iR] * SPACE_A_AU);
        o->yR[id] = v[2] / ndeg[iR] * SPACE_A_AU + I * (v[3] / ndeg[iR] * SPACE_A_AU);
        o->zR[id] = v[4] / ndeg[iR] * SPACE_A_AU + I * (v[5] / ndeg[iR] * SPACE_A_AU);
      }
  }
  free(ndeg);
  fclose(f);
  return 0;
fail2:
  free(ndeg);
fail:
  fclose(f);
  return EDUS_EIO;
}

/* headers/Wannier.h:278-304 / :336-471: sum_R e^{2 pi i k.R} X(R) */
static cplx wannier_sum(const orc* o, const cplx* XR, int i, int j, const double* k) {
  cplx v = 0.;
  int nr = o->nrpts, n = o->ncv;
  for (int iR = 0; iR < nr; iR++) {
    double kR = 0.;
    for (int l = 0; l < 3; l++) kR += k[l] * o->Rvec[iR * 3 + l];
    kR *= 2 * PI;
    v += cexpi(kR) * XR[((size_t)i * n + j) * nr + iR];
  }
  return v;
}

/* ------------------------------------------------------------ Crystal model */

/* next line of f into buf; 0 at end of file */
static int cy_line(FILE* f, char* buf, int cap) { return fgets(buf, cap, f) != NULL; }

/* splits buf in place on blanks; returns the token count (at most cap) */
static int cy_split(char* buf, char** tok, int cap) {
  int n = 0;
  char* save = NULL;
  for (char* t = strtok_r(buf, " \t\r\n", &save); t && n < cap; t = strtok_r(NULL, " \t\r\n", &save)) tok[n++] = t;
  return n;
}

#define CY_LINE 65536
#define CY_TOK 512

/* headers/Crystal_interface.h:19-208 (Crystal::init): lattice, orbital count and
 * grid size from kmesh_data.dat, then H from hk_orthonormal.dat and the x, y Berry
 * connections from bc_betabetap_real.dat / bc_betabetap_imag.dat */
static int crystal_read(orc* o, const char* workdir) {
  char path[2 * EDUS_STRLEN + 32], path2[2 * EDUS_STRLEN + 32];
  char* buf = malloc(CY_LINE);
  char* tok[CY_TOK];
  int rc = EDUS_EIO, norb = 0, nkf = 0, n = o->ncv;
  const char* wd = workdir ? workdir : ".";
  FILE *f = NULL, *g = NULL;
  if (!buf) return EDUS_ENOMEM;
  snprintf(path, sizeof(path), "%s/kmesh_data.dat", wd);
  f = fopen(path, "r");
  if (!f) goto out;
  double v[4][2];
  for (int r = 0; r < 4; r++) {
    if (!cy_line(f, buf, CY_LINE) || !cy_line(f, buf, CY_LINE)) goto out;
    if (cy_split(buf, tok, CY_TOK) < 2) goto out;
    v[r][0] = atof(tok[0]);
    v[r][1] = atof(tok[1]);
  }
  memset(o->p.a, 0, sizeof(o->p.a));
  memset(o->p.b, 0, sizeof(o->p.b));
  o->p.a[1][1] = v[0][0];
  o->p.a[1][2] = v[0][1];
  o->p.a[2][1] = v[1][0];
  o->p.a[2][2] = v[1][1];
  o->p.a[0][0] = 15.;
  o->p.b[1][1] = v[2][0];
  o->p.b[1][2] = v[2][1];
  o->p.b[2][1] = v[3][0];
  o->p.b[2][2] = v[3][1];
  o->p.b[0][0] = 1. / 15.;
  for (;;) { /* up to the line whose last word is "basis" */
    if (!cy_line(f, buf, CY_LINE)) goto out;
    int nt = cy_split(buf, tok, CY_TOK);
    if (nt > 0 && !strcasecmp(tok[nt - 1], "basis")) break;
  }
  if (!cy_line(f, buf, CY_LINE) || cy_split(buf, tok, CY_TOK) < 1) goto out;
  norb = atoi(tok[0]);
  for (;;) { /* up to the line whose last word is "direction" */
    if (!cy_line(f, buf, CY_LINE)) goto out;
    int nt = cy_split(buf, tok, CY_TOK);
    if (nt > 0 && !strcasecmp(tok[nt - 1], "direction")) break;
  }
  if (!cy_line(f, buf, CY_LINE) || cy_split(buf, tok, CY_TOK) < 1) goto out;
  nkf = atoi(tok[0]);
  fclose(f);
  f = NULL;
  if (norb < n || nkf < 2) {
    rc = EDUS_EINVAL;
    goto out;
  }
  o->cy_nkf = nkf;
  size_t tab = (size_t)n * n * nkf * nkf;
  o->cyH = calloc(tab, sizeof(cplx));
  o->cyDx = calloc(tab, sizeof(cplx));
  o->cyDy = calloc(tab, sizeof(cplx));
  if (!o->cyH || !o->cyDx || !o->cyDy) {
    rc = EDUS_ENOMEM;
    goto out;
  }
#define CY_AT(T, i, j, k1, k2) (T)[(((size_t)(i) * n + (j)) * nkf + (k1)) * nkf + (k2)]
  snprintf(path, sizeof(path), "%s/hk_orthonormal.dat", wd);
  f = fopen(path, "r");
  if (!f) goto out;
  for (int k1 = 0; k1 < nkf; k1++)
    for (int k2 = 0; k2 < nkf; k2++) {
      for (int part = 0; part < 2; part++) { /* real rows, separator, imaginary rows */
        for (int i = 0; i < norb; i++) {
          if (!cy_line(f, buf, CY_LINE)) goto out;
          if (i >= n) continue;
          if (cy_split(buf, tok, CY_TOK) < i + 1) goto out;
          for (int j = 0; j <= i; j++) CY_AT(o->cyH, i, j, k1, k2) += part ? I * atof(tok[j]) : atof(tok[j]);
        }
        cy_line(f, buf, CY_LINE);
      }
      cy_line(f, buf, CY_LINE);
    }
  fclose(f);
  f = NULL;
  snprintf(path, sizeof(path), "%s/bc_betabetap_real.dat", wd);
  snprintf(path2, sizeof(path2), "%s/bc_betabetap_imag.dat", wd);
  f = fopen(path, "r");
  g = fopen(path2, "r");
  if (!f || !g) goto out;
  char* buf2 = malloc(CY_LINE);
  char* tok2[CY_TOK];
  if (!buf2) {
    rc = EDUS_ENOMEM;
    goto out;
  }
  for (int k1 = 0; k1 < nkf; k1++)
    for (int k2 = 0; k2 < nkf; k2++) {
      for (int x = 0; x < 2; x++) {
        cplx* T = x ? o->cyDy : o->cyDx;
        for (int i = 0; i < norb; i++) {
          if (!cy_line(f, buf, CY_LINE) || !cy_line(g, buf2, CY_LINE)) goto out2;
          if (i >= n) continue;
          if (cy_split(buf, tok, CY_TOK) < i + 1 || cy_split(buf2, tok2, CY_TOK) < i + 1) goto out2;
          for (int j = 0; j <= i; j++) CY_AT(T, i, j, k1, k2) = atof(tok[j]) + I * atof(tok2[j]);
        }
        cy_line(f, buf, CY_LINE);
        cy_line(g, buf2, CY_LINE);
      }
      cy_line(f, buf, CY_LINE);
      cy_line(g, buf2, CY_LINE);
    }
  rc = 0;
out2:
  free(buf2);
out:
  if (f) fclose(f);
  if (g) fclose(g);
  free(buf);
  return rc;
}

/* headers/Interpolation.h:86-146 (the two-dimensional fit: periodic padding, the
 * 16 coefficients a_ab = sum_rs M_ar M_bs p_rs of the 4 x 4 patch around the cell)
 * and :228-264 (cell location and the polynomial in dy, dz) */
static cplx crystal_fit(const orc* o, const cplx* T, int i, int j, const double* k) {
  static const double M[4][4] = {{0, 1, 0, 0}, {-0.5, 0, 0.5, 0}, {1, -2.5, 2, -0.5}, {-0.5, 1.5, -1.5, 0.5}};
  int n = o->ncv, nkf = o->cy_nkf;
  double sp = 1. / (nkf - 1);
  double dy = fmod((k[1] - (-0.5)) / sp, nkf), dz = fmod((k[2] - (-0.5)) / sp, nkf);
  if (dy < 0) dy += nkf;
  if (dz < 0) dz += nkf;
  int yi = (int)floor(dy), zi = (int)floor(dz);
  dy -= yi;
  dz -= zi;
  cplx p[4][4];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      int a1 = yi - 1 + r, a2 = zi - 1 + c;
      a1 = a1 >= 0 ? a1 % nkf : nkf + a1 % nkf;
      a2 = a2 >= 0 ? a2 % nkf : nkf + a2 % nkf;
      p[r][c] = CY_AT(T, i, j, a1, a2);
    }
  cplx cf[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      cplx acc = 0;
      for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) acc += M[a][r] * M[b][c] * p[r][c];
      cf[a][b] = acc;
    }
  double y2 = dy * dy, y3 = y2 * dy, z2 = dz * dz, z3 = z2 * dz;
  return (cf[0][0] + cf[0][1] * dz + cf[0][2] * z2 + cf[0][3] * z3) + (cf[1][0] + cf[1][1] * dz + cf[1][2] * z2 + cf[1][3] * z3) * dy +
         (cf[2][0] + cf[2][1] * dz + cf[2][2] * z2 + cf[2][3] * z3) * y2 + (cf[3][0] + cf[3][1] * dz + cf[3][2] * z2 + cf[3][3] * z3) * y3;
}

/* headers/Crystal_interface.h:212-270 (energy and dipoles; the upper triangle is the
 * conjugate of the fitted lower) */
static cplx crystal_elem(const orc* o, const cplx* T, int ic, int jc, const double* k) {
  if (jc < ic + 1) return crystal_fit(o, T, ic, jc, k);
  return conj(crystal_fit(o, T, jc, ic, k));
}
#undef CY_AT

/* ------------------------------------------------------------ model tabulation */

/* Source_Main/save_HUD.cpp:19-53 (+ headers/Wannier.h:477-551 energy_U) and
 * the gradient of the energy save_HUD.cpp:96-137. */
static int tabulate(orc* o) {
  int n = o->ncv, nk = o->nk;
  int isW = o->p.mode == EDUS_MODE_WANNIER;
  double S[EDUS_MAX_BANDS];
  for (int i = 0; i < n; i++) S[i] = 0;
  double gapc = o->p.conduction_shift;
  if (gapc > 1e-16)
    for (int i = 0; i < n; i++)
      if (i >= o->p.nb[1]) S[i] = gapc;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < nk; ik++) {
    const double* k = &o->kpt[ik * 3];
    cplx Hk[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Uk[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Dk[EDUS_MAX_BANDS * EDUS_MAX_BANDS * 3];
    if (isW) {
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++) {
          Hk[ic * n + jc] = wannier_sum(o, o->HR, ic, jc, k);
          if (ic == jc) Hk[ic * n + jc] = creal(Hk[ic * n + jc]);
          Dk[(ic * n + jc) * 3 + 0] = wannier_sum(o, o->xR, ic, jc, k);
          Dk[(ic * n + jc) * 3 + 1] = wannier_sum(o, o->yR, ic, jc, k);
          Dk[(ic * n + jc) * 3 + 2] = wannier_sum(o, o->zR, ic, jc, k);
          if (ic == jc)
            for (int x = 0; x < 3; x++) Dk[(ic * n + jc) * 3 + x] = creal(Dk[(ic * n + jc) * 3 + x]);
        }
      cplx A[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Z[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
      double ev[EDUS_MAX_BANDS];
      memcpy(A, Hk, sizeof(cplx) * n * n);
      eig_herm(n, A, ev, Z);
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++) Uk[ic * n + jc] = conj(Z[jc * n + ic]);
    } else if (o->p.mode == EDUS_MODE_CRYSTAL) {
      /* headers/Crystal_interface.h:272-304: dipoles in the order (z, x, y), real
       * diagonals; Uk = conj(eigenvectors)^T of the Hermitian H */
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++) {
          Hk[ic * n + jc] = crystal_elem(o, o->cyH, ic, jc, k);
          Dk[(ic * n + jc) * 3 + 0] = 0.;
          Dk[(ic * n + jc) * 3 + 1] = crystal_elem(o, o->cyDx, ic, jc, k);
          Dk[(ic * n + jc) * 3 + 2] = crystal_elem(o, o->cyDy, ic, jc, k);
          if (ic == jc)
            for (int x = 0; x < 3; x++) Dk[(ic * n + jc) * 3 + x] = creal(Dk[(ic * n + jc) * 3 + x]);
        }
      cplx A[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Z[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
      double ev[EDUS_MAX_BANDS];
      memcpy(A, Hk, sizeof(cplx) * n * n);
      eig_herm(n, A, ev, Z);
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++) Uk[ic * n + jc] = conj(Z[jc * n + ic]);
    } else {
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++) {
          Hk[ic * n + jc] = tb_energy(o, ic, jc, k);
          Uk[ic * n + jc] = tb_unitary(o, ic, jc, k);
          for (int x = 0; x < 3; x++) Dk[(ic * n + jc) * 3 + x] = tb_dipole(o, ic, jc, x);
        }
    }
    for (int ic = 0; ic < n; ic++)
      for (int jc = 0; jc < n; jc++) {
        cplx value = 0.;
        if (gapc > 1e-16)
          for (int ii = 0; ii < n; ii++) value += conj(Uk[ii * n + ic]) * S[ii] * Uk[ii * n + jc];
        o->H[IDX3(ik, ic, jc, n)] = Hk[ic * n + jc] + value;
        o->U[IDX3(ik, ic, jc, n)] = Uk[ic * n + jc];
        for (int x = 0; x < 3; x++) {
          cplx d = Dk[(ic * n + jc) * 3 + x];
          if (isW) d = 0.5 * (Dk[(ic * n + jc) * 3 + x] + Dk[(jc * n + ic) * 3 + x]);
          o->D[IDX4(ik, ic, jc, x, n)] = d;
        }
      }
  }
  for (int ik = 0; ik < nk; ik++)
    for (int ic = 0; ic < n; ic++)
      for (int jc = 0; jc < n; jc++) o->hU[IDX3(ik, ic, jc, n)] = conj(o->U[IDX3(ik, jc, ic, n)]);
  return 0;
}

/* ------------------------------------------------------------ velocity gauge
 * An option the reference does not have (its vector potential, Laser::A_crys
 * in headers/Laser.h:191-213, is only called from dead code). The length-gauge
 * equation drho(k)/dt = -i[H(k) + E.D(k), rho(k)] + E.grad_k rho(k) becomes,
 * for rho'(k, t) = rho(k + A(t), t) with A = -int E_pump dt,
 *   drho'(k)/dt = -i[H(k + A) + E.D(k + A), rho'(k)]
 * (the gradient term cancels against dA/dt = -E). Wannier models only: H and D
 * are the reference's Fourier sums (headers/Wannier.h:278-304,336-471,
 * 489-492, 577-578; Source_Main/save_HUD.cpp:47-51) at k + A. Observables at
 * k + A: populations in the eigenbasis of H(k + A), J1 from the reference's
 * stencil gradient of H(k + A) on the grid, J2 with H and D at k + A. */

static void field_at(const orc* o, double t, double EF[2][3]);

/* A(t) by 4-point Gauss-Legendre panels of at most 0.5 a.u. over [A_t, t]
 * (one panel per RK4 half step; the field period is hundreds of a.u.);
 * returns A in crystal coordinates */
static void vg_A(orc* o, double t, double Acrys[3]) {
  static const double gx[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
  static const double gw[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
  if (t < o->A_t) {
    o->A_t = -0.21 / TIME_AU_FS;
    o->A_cart[0] = o->A_cart[1] = o->A_cart[2] = 0.;
  }
  const int panels = (int)ceil((t - o->A_t) / 0.5);
  const double t0 = o->A_t;
  for (int p = 0; p < panels; p++) {
    const double a = t0 + (t - t0) * p / panels, b = t0 + (t - t0) * (p + 1) / panels;
    const double h = 0.5 * (b - a), m = 0.5 * (a + b);
    for (int q = 0; q < 4; q++) {
      double EF[2][3];
      field_at(o, m + h * gx[q], EF);
      for (int x = 0; x < 3; x++) o->A_cart[x] -= h * gw[q] * EF[0][x];
    }
  }
  o->A_t = t;
  cart_to_crys(o, o->A_cart, Acrys);
}

/* H and D of every k point at k + A(t) into o->H, o->D */
static void vg_tables(orc* o, double t) {
  int n = o->ncv;
  double Ac[3];
  vg_A(o, t, Ac);
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++) {
    double k[3];
    for (int l = 0; l < 3; l++) k[l] = o->kpt[ik * 3 + l] + Ac[l];
    cplx Dk[EDUS_MAX_BANDS * EDUS_MAX_BANDS * 3];
    for (int ic = 0; ic < n; ic++)
      for (int jc = 0; jc < n; jc++) {
        cplx h = wannier_sum(o, o->HR, ic, jc, k);
        if (ic == jc) h = creal(h);
        o->H[IDX3(ik, ic, jc, n)] = h;
        Dk[(ic * n + jc) * 3 + 0] = wannier_sum(o, o->xR, ic, jc, k);
        Dk[(ic * n + jc) * 3 + 1] = wannier_sum(o, o->yR, ic, jc, k);
        Dk[(ic * n + jc) * 3 + 2] = wannier_sum(o, o->zR, ic, jc, k);
        if (ic == jc)
          for (int x = 0; x < 3; x++) Dk[(ic * n + jc) * 3 + x] = creal(Dk[(ic * n + jc) * 3 + x]);
      }
    for (int ic = 0; ic < n; ic++)
      for (int jc = 0; jc < n; jc++)
        for (int x = 0; x < 3; x++)
          o->D[IDX4(ik, ic, jc, x, n)] = 0.5 * (Dk[(ic * n + jc) * 3 + x] + Dk[(jc * n + ic) * 3 + x]);
  }
}

/* Source_Main/save_HUD.cpp:96-137 (GradientEnergy of H) */
static void gradient_energy(orc* o, const cplx* Hs) {
  int n = o->ncv;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++)
    for (int i = 0; i < 3; i++)
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++) {
          cplx acc = 0;
          for (int b = 0; b < o->nnb; b++) {
            int kb = o->nbr[(size_t)ik * o->nnb + b];
            acc += o->weights[o->bshell[b]] * o->bvec[b][i] * (Hs[IDX3(kb, ic, jc, n)] - Hs[IDX3(ik, ic, jc, n)]);
          }
          o->GE[IDX4(ik, ic, jc, i, n)] = acc;
        }
}

/* if_resolution.cpp:154-169: renormalised gradient, upper triangle + conj mirror */
static void gradient_energy_renorm(orc* o, const cplx* Hs) {
  int n = o->ncv;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++)
    for (int i = 0; i < 3; i++)
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic; jc < n; jc++) {
          cplx acc = 0;
          for (int b = 0; b < o->nnb; b++) {
            int kb = o->nbr[(size_t)ik * o->nnb + b];
            acc += o->weights[o->bshell[b]] * o->bvec[b][i] * (Hs[IDX3(kb, ic, jc, n)] - Hs[IDX3(ik, ic, jc, n)]);
          }
          o->GE[IDX4(ik, ic, jc, i, n)] = acc;
          o->GE[IDX4(ik, jc, ic, i, n)] = conj(acc);
        }
}

/* headers/InitialPopulation.h:2-39 */
static void initial_population(orc* o) {
  int n = o->ncv;
  for (int ik = 0; ik < o->nk; ik++)
    for (int ia = 0; ia < n; ia++)
      for (int ib = 0; ib < n; ib++) {
        cplx acc = 0;
        for (int ii = 0; ii < o->nbands; ii++) acc += o->U[IDX3(ik, ii, ia, n)] * conj(o->U[IDX3(ik, ii, ib, n)]);
        o->P0[IDX3(ik, ia, ib, n)] = acc;
      }
}

/* headers/InitParameters.h:203-224 (Initialize_T) + main_MPI.cpp:66-77 */
static void init_T(orc* o) {
  int n = o->ncv, nch = o->nch;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) o->T[i][j] = 0;
  for (int ic = nch; ic < n; ic++)
    for (int jc = nch; jc < n; jc++) o->T[ic][jc] = (ic == jc) ? o->p.T1 : o->p.T2;
  for (int ic = 0; ic < nch; ic++) {
    for (int jc = 0; jc < nch; jc++) o->T[ic][jc] = o->p.Tch;
    for (int jc = nch; jc < n; jc++) o->T[ic][jc] = o->p.Tch / 2.;
  }
  for (int ic = 0; ic < n; ic++)
    for (int jc = ic + 1; jc < n; jc++) o->T[jc][ic] = o->T[ic][jc];
  o->n_diss = 0;
  for (int ic = 0; ic < n; ic++)
    for (int jc = 0; jc < n; jc++)
      if (fabs(o->T[ic][jc]) > 1e-24) {
        o->diss_i[o->n_diss] = ic;
        o->diss_j[o->n_diss] = jc;
        o->n_diss++;
      }
}

/* ------------------------------------------------------------ laser */

/* headers/Laser.h:56-76 envelopes, :128-144 E(t) */
static void laser_E(const edus_laser* L, double t, double E[3]) {
  double env = 0.;
  if (L->envelope_kind == EDUS_ENV_GAUSS) {
    double d = t - L->t0;
    env = (d * d < 40 * L->sigma * L->sigma) ? L->E0 * exp(-d * d / (2 * L->sigma * L->sigma)) : 0.;
  } else if (L->envelope_kind == EDUS_ENV_SIN2) {
    if (t >= L->t0 && t <= L->tf) {
      double s = sin(PI * (t - L->t0) / (L->tf - L->t0));
      env = L->E0 * (s * s);
    }
  } else if (L->envelope_kind == EDUS_ENV_PW) {
    double tr = 0.;
    if (t >= L->t0 && t < L->w1)
      tr = (t - L->t0) / (L->w1 - L->t0);
    else if (t >= L->w1 && t < L->w2)
      tr = 1.;
    else if (t >= L->w2 && t <= L->tf)
      tr = (t - L->tf) / (L->w2 - L->tf);
    env = L->E0 * tr;
  }
  double p1 = L->envelope_only ? 1. : sin(L->wl * (t - L->t0) + L->phase);
  double p2 = L->envelope_only ? 1. : cos(L->wl * (t - L->t0) + L->phase);
  for (int i = 0; i < 3; i++) E[i] = env * (p1 * L->pol1[i] + p2 * L->pol2[i]);
}

/* Source_Main/RungeKutta.cpp:24-30: pump sum and half probe */
static void field_at(const orc* o, double t, double EF[2][3]) {
  for (int i = 0; i < 3; i++) EF[0][i] = 0.;
  for (int ip = 0; ip < o->p.n_pumps; ip++) {
    double e[3];
    laser_E(&o->p.pump[ip], t, e);
    for (int i = 0; i < 3; i++) EF[0][i] += e[i];
  }
  double e2[3];
  laser_E(&o->p.probe, t, e2);
  for (int i = 0; i < 3; i++) EF[1][i] = .5 * e2[i];
}

static int field_nonzero(double EF[2][3]) {
  double Emax = 0;
  for (int a = 0; a < 2; a++)
    for (int i = 0; i < 3; i++) Emax += EF[a][i] * EF[a][i];
  return sqrt(Emax) > 1e-20;
}

/* ------------------------------------------------------------ Coulomb */

/* headers/integrationWeight.h:139-175 (get_trig_coef) */
static void trig_tables(orc* o) {
  int nc = o->ncut, nk = o->nk;
  int a1 = o->p.sample_110 ? 0 : 1, a2 = o->p.sample_110 ? 1 : 2;
  for (int m = 0; m < nc; m++)
    for (int ik = 0; ik < nk; ik++) {
      double mkx = 2 * PI * m * o->kpt[ik * 3 + a1];
      double nky = 2 * PI * m * o->kpt[ik * 3 + a2];
      o->cos_m1[m * nk + ik] = cos(mkx);
      o->sin_m1[m * nk + ik] = sin(mkx);
      o->cos_m2[m * nk + ik] = cos(nky);
      o->sin_m2[m * nk + ik] = sin(nky);
    }
}

/* Source_Main/Fourier_Coulomb.cpp:505-622 (Read_Coulomb_from_files) */
static int read_cplx_rows(const char* path, int rows, int cols, cplx* dst) {
  FILE* f = fopen(path, "r");
  if (!f) return EDUS_EIO;
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < cols; c++) {
      double re, im;
      if (fscanf(f, "%lf %lf", &re, &im) != 2) {
        fclose(f);
        return EDUS_EIO;
      }
      dst[(size_t)r * cols + c] = re + I * im;
    }
  fclose(f);
  return 0;
}

static int coulomb_read(orc* o, const char* workdir) {
  int n = o->ncv, nc2 = o->ncut * o->ncut, n2 = n * n;
  char path[3 * EDUS_STRLEN];
  const char* wd = workdir ? workdir : ".";
  const char* lab = o->p.coulomb_label;
  snprintf(path, sizeof(path), "%s/Output/Coulomb/V_Hartree_%s.txt", wd, lab);
  FILE* f = fopen(path, "r");
  if (!f) return EDUS_EIO;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      if (fscanf(f, "%lf", &o->VH[i][j]) != 1) {
        fclose(f);
        return EDUS_EIO;
      }
  fclose(f);
  const char* nm[4] = {"A", "B", "C", "D"};
  cplx* dst[4] = {o->cA, o->cB, o->cC, o->cD};
  for (int q = 0; q < 4; q++) {
    snprintf(path, sizeof(path), "%s/Output/Coulomb/%s_coeff%s.txt", wd, nm[q], lab);
    int rc = read_cplx_rows(path, nc2, n2, dst[q]);
    if (rc) return rc;
  }
  snprintf(path, sizeof(path), "%s/Output/Coulomb/Screen_const_%s.txt", wd, lab);
  return read_cplx_rows(path, n2, 1, o->screen);
}

/* headers/Coulomb.h:273-503 (Calculate_X_coefficients_MPI), one rank:
 * forward trig transform of P, Hartree term at mm=0, combine with A,B,C,D. */
static void coulomb_coeffs(orc* o, const cplx* P) {
  int n = o->ncv, nk = o->nk, nc = o->ncut;
  double N_BZ = (double)nk;
  double wk = 1.0 / N_BZ;
  const int nth = NBLK;
  cplx* part = malloc(sizeof(cplx) * 4 * n * n * nth);
  for (int mm = 0; mm < nc * nc; mm++) {
    int m = mm / nc, nn = mm % nc;
    double corr = -4 * PI * PI * (m * m + nn * nn) / (N_BZ * 27);
    memset(part, 0, sizeof(cplx) * 4 * n * n * nth);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nth; t++) {
      const int T = nth;
      int len = nk / T, left = nk % T;
      int beg = len * t + (t < left ? t : left);
      int end = beg + len + (t < left ? 1 : 0);
      cplx* fcc = part + (size_t)4 * n * n * t;
      cplx *fcs = fcc + n * n, *fsc = fcs + n * n, *fss = fsc + n * n;
      for (int ik = beg; ik < end; ik++) {
        double cc = o->cos_m1[m * nk + ik] * o->cos_m2[nn * nk + ik];
        double cs = o->cos_m1[m * nk + ik] * o->sin_m2[nn * nk + ik];
        double sc = o->sin_m1[m * nk + ik] * o->cos_m2[nn * nk + ik];
        double ss = o->sin_m1[m * nk + ik] * o->sin_m2[nn * nk + ik];
        for (int ic = 0; ic < n; ic++)
          for (int jc = ic; jc < n; jc++) {
            cplx Pc = wk * P[IDX3(ik, ic, jc, n)];
            fcc[ic * n + jc] += Pc * cc * (1. + corr);
            fcs[ic * n + jc] += Pc * cs * (1. + corr);
            fsc[ic * n + jc] += Pc * sc * (1. + corr);
            fss[ic * n + jc] += Pc * ss * (1. + corr);
          }
      }
    }
    cplx f[4][EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    memset(f, 0, sizeof(f));
    for (int t = 0; t < nth; t++)
      for (int q = 0; q < 4; q++)
        for (int e = 0; e < n * n; e++) f[q][e] += part[(size_t)4 * n * n * t + q * n * n + e];
    cplx *fcc = f[0], *fcs = f[1], *fsc = f[2], *fss = f[3];
    if (mm == 0) {
      for (int ic = 0; ic < n; ic++) {
        o->EH[ic] = 0.;
        for (int jc = 0; jc < n; jc++) o->EH[ic] += creal(fcc[jc * n + jc]) * o->VH[ic][jc];
        o->EH[ic] -= o->EH0[ic];
      }
    }
    cplx Amn = 0, Bmn = 0, Cmn = 0, Dmn = 0;
    size_t base = (size_t)mm * n * n;
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic; jc < n; jc++) {
        int d = ic * n + jc, od = jc * n + ic;
        if (ic == jc) {
          Amn = o->cA[(size_t)mm * n * n + 0];
          Dmn = o->cD[(size_t)mm * n * n + 0];
        } else {
          Amn = o->cA[(size_t)mm * n * n + d];
          Bmn = o->cB[(size_t)mm * n * n + d];
          Cmn = o->cC[(size_t)mm * n * n + d];
          Dmn = o->cD[(size_t)mm * n * n + d];
        }
        o->Xcc[base + d] = (Amn * fcc[d] + Dmn * fss[d]) - o->Xcc0[base + d];
        if (jc != ic) {
          o->Xcc[base + d] += (Bmn * fcs[d] + Cmn * fsc[d]);
          o->Xcc[base + od] = conj(o->Xcc[base + d]);
        }
        o->Xcs[base + d] = (Amn * fcs[d] - Dmn * fsc[d]) - o->Xcs0[base + d];
        if (jc != ic) {
          o->Xcs[base + d] += (-Bmn * fcc[d] + Cmn * fss[d]);
          o->Xcs[base + od] = conj(o->Xcs[base + d]);
        }
        o->Xsc[base + d] = (Amn * fsc[d] - Dmn * fcs[d]) - o->Xsc0[base + d];
        if (jc != ic) {
          o->Xsc[base + d] += (Bmn * fss[d] - Cmn * fcc[d]);
          o->Xsc[base + od] = conj(o->Xsc[base + d]);
        }
        o->Xss[base + d] = (Amn * fss[d] + Dmn * fcc[d]) - o->Xss0[base + d];
        if (jc != ic) {
          o->Xss[base + d] += (-Bmn * fsc[d] - Cmn * fcs[d]);
          o->Xss[base + od] = conj(o->Xss[base + d]);
        }
      }
  }
  free(part);
}

/* headers/Coulomb.h:510-541 (Calculate_X_MPI) for one k */
static void coulomb_X(const orc* o, int ik, cplx* Xk) {
  int n = o->ncv, nk = o->nk, nc = o->ncut;
  for (int e = 0; e < n * n; e++) Xk[e] = 0;
  for (int mm = 0; mm < nc * nc; mm++) {
    int m = mm / nc, nn = mm % nc;
    double cc = o->cos_m1[m * nk + ik] * o->cos_m2[nn * nk + ik];
    double cs = o->cos_m1[m * nk + ik] * o->sin_m2[nn * nk + ik];
    double sc = o->sin_m1[m * nk + ik] * o->cos_m2[nn * nk + ik];
    double ss = o->sin_m1[m * nk + ik] * o->sin_m2[nn * nk + ik];
    size_t base = (size_t)mm * n * n;
    for (int ic = 0; ic < n; ic++)
      for (int jc = 0; jc < n; jc++) {
        size_t id = base + ic * n + jc;
        cplx alpha = o->Xcc[id] * cc + o->Xcs[id] * cs + o->Xsc[id] * sc + o->Xss[id] * ss;
        Xk[jc * n + ic] -= alpha;
      }
  }
}

/* headers/RungeKutta.h:69-138: renormalised H for one k (Wannier basis) */
static void coulomb_hk(const orc* o, int ik, const cplx* P, cplx* Hk) {
  int n = o->ncv;
  cplx X[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  coulomb_X(o, ik, X);
  if (o->n_cond_coul > pow(10, -20)) {
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic; jc < n; jc++) {
        int lin = (ic != jc) ? ic * n + jc : 0;
        X[ic * n + jc] -= conj(o->screen[lin]) * (P[IDX3(ik, jc, ic, n)] - o->PW0[IDX3(ik, jc, ic, n)]);
        if (ic != jc) X[jc * n + ic] = conj(X[ic * n + jc]);
      }
  }
  for (int ic = 0; ic < n; ic++) {
    X[ic * n + ic] = creal(X[ic * n + ic]);
    for (int jc = ic; jc < n; jc++) {
      Hk[ic * n + jc] = o->H[IDX3(ik, ic, jc, n)] + X[ic * n + jc];
      if (ic == jc) Hk[ic * n + ic] += o->EH[ic];
      if (ic != jc) Hk[jc * n + ic] = conj(Hk[ic * n + jc]);
    }
  }
}

/* headers/InitParameters.h:264-333 (get_P_in_dia_vect): P_d = conj(U) P U^T
 * with a real diagonal, for every k */
static void p_in_dia(const orc* o, const cplx* P, cplx* Pd) {
  int n = o->ncv;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++) {
    const cplx* U = &o->U[IDX3(ik, 0, 0, n)];
    cplx Pf[EDUS_MAX_BANDS * EDUS_MAX_BANDS], M[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic; jc < n; jc++) {
        Pf[ic * n + jc] = P[IDX3(ik, ic, jc, n)];
        if (ic != jc) Pf[jc * n + ic] = conj(Pf[ic * n + jc]);
      }
    for (int ii = 0; ii < n; ii++)
      for (int jc = 0; jc < n; jc++) {
        cplx m = 0;
        for (int jj = 0; jj < n; jj++) m += Pf[ii * n + jj] * U[jc * n + jj];
        M[jc * n + ii] = m;
      }
    for (int ic = 0; ic < n; ic++)
      for (int jc = 0; jc < n; jc++) {
        cplx v = 0;
        for (int ii = 0; ii < n; ii++) v += conj(U[ic * n + ii]) * M[jc * n + ii];
        Pd[IDX3(ik, ic, jc, n)] = v;
      }
    for (int ic = 0; ic < n; ic++) Pd[IDX3(ik, ic, ic, n)] = creal(Pd[IDX3(ik, ic, ic, n)]);
  }
}

/* headers/RungeKutta.h:96-138: renormalised H for one k, Coulomb in the
 * diagonal basis (screening of that basis, then X_W = U^dagger X_d U,
 * get_Xd_in_Wannier_vect, headers/InitParameters.h:339-373) */
static void coulomb_hk_diag(const orc* o, int ik, cplx* Hk) {
  int n = o->ncv;
  cplx X[EDUS_MAX_BANDS * EDUS_MAX_BANDS], M[EDUS_MAX_BANDS * EDUS_MAX_BANDS], XW[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  coulomb_X(o, ik, X);
  const cplx* Pd = &o->Pd[IDX3(ik, 0, 0, n)];
  for (int ic = 0; ic < n; ic++) {
    double pb = ic < o->nbands ? 1.0 : 0.0;
    X[ic * n + ic] -= o->screen[0] * (Pd[ic * n + ic] - pb);
    for (int jc = ic + 1; jc < n; jc++) {
      X[ic * n + jc] -= conj(o->screen[1]) * Pd[jc * n + ic];
      X[jc * n + ic] = conj(X[ic * n + jc]);
    }
  }
  const cplx* U = &o->U[IDX3(ik, 0, 0, n)];
  for (int ii = 0; ii < n; ii++)
    for (int jc = 0; jc < n; jc++) {
      cplx m = 0;
      for (int jj = 0; jj < n; jj++) m += X[ii * n + jj] * U[jj * n + jc];
      M[ii * n + jc] = m;
    }
  for (int ic = 0; ic < n; ic++)
    for (int jc = 0; jc < n; jc++) {
      cplx v = 0;
      for (int ii = 0; ii < n; ii++) v += conj(U[ii * n + ic]) * M[ii * n + jc];
      XW[ic * n + jc] = v;
    }
  for (int ic = 0; ic < n; ic++) {
    XW[ic * n + ic] = creal(XW[ic * n + ic]);
    for (int jc = ic; jc < n; jc++) {
      Hk[ic * n + jc] = o->H[IDX3(ik, ic, jc, n)] + XW[ic * n + jc];
      if (ic == jc) Hk[ic * n + ic] += o->EH[ic];
      if (ic != jc) Hk[jc * n + ic] = conj(Hk[ic * n + jc]);
    }
  }
}

/* Coulomb coefficients of the state (the eigenbasis state in the diagonal basis) */
static void coulomb_update(orc* o, const cplx* P) {
  if (o->p.diag_basis) {
    p_in_dia(o, P, o->Pd);
    coulomb_coeffs(o, o->Pd);
  } else {
    coulomb_coeffs(o, P);
  }
}

static void coulomb_hk_any(const orc* o, int ik, const cplx* P, cplx* Hk) {
  if (o->p.diag_basis)
    coulomb_hk_diag(o, ik, Hk);
  else
    coulomb_hk(o, ik, P, Hk);
}

/* ------------------------------------------------------------ RHS */

/* headers/RungeKutta.h:7-297 (get_derivative_Df), Wannier-basis Coulomb */
static void rhs(orc* o, const cplx* P, cplx* Pv, double EF[2][3], double wx2, int e_non0) {
  int n = o->ncv, nch = o->nch;
  if (o->p.coulomb) coulomb_update(o, P);
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++) {
    cplx Hk[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    if (o->p.coulomb) {
      coulomb_hk_any(o, ik, P, Hk);
      for (int e = 0; e < n * n; e++) o->Hr[(size_t)ik * n * n + e] = Hk[e];
    } else {
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic; jc < n; jc++) {
          Hk[ic * n + jc] = o->H[IDX3(ik, ic, jc, n)];
          if (ic != jc) Hk[jc * n + ic] = conj(Hk[ic * n + jc]);
        }
    }
    const cplx* Pk = &P[IDX3(ik, 0, 0, n)];
    cplx* pv = &Pv[IDX3(ik, 0, 0, n)];
    const cplx* Dk = &o->D[IDX4(ik, 0, 0, 0, n)];
    /* populations (RungeKutta.h:158-173) */
    for (int ic = 0; ic < n; ic++) {
      cplx beta = 0.;
      for (int j = 0; j < n; j++) {
        int w = (ic >= nch && j < nch) || (ic < nch && j >= nch);
        cplx h = Hk[ic * n + j] + EF[w][0] * Dk[(ic * n + j) * 3 + 0] + EF[w][1] * Dk[(ic * n + j) * 3 + 1] +
                 EF[w][2] * Dk[(ic * n + j) * 3 + 2];
        beta += h * Pk[ic * n + j];
      }
      pv[ic * n + ic] = 2. * cimag(beta);
    }
    /* coherences (RungeKutta.h:184-212) */
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic + 1; jc < n; jc++) {
        cplx beta = 0.;
        for (int j = 0; j < n; j++) {
          int w1 = (jc >= nch && j < nch) || (jc < nch && j >= nch);
          int w2 = (ic >= nch && j < nch) || (ic < nch && j >= nch);
          cplx a = (Hk[jc * n + j] + EF[w1][0] * Dk[(jc * n + j) * 3 + 0] + EF[w1][1] * Dk[(jc * n + j) * 3 + 1] +
                    EF[w1][2] * Dk[(jc * n + j) * 3 + 2]) *
                   Pk[ic * n + j];
          cplx b = (Hk[ic * n + j] + EF[w2][0] * Dk[(ic * n + j) * 3 + 0] + EF[w2][1] * Dk[(ic * n + j) * 3 + 1] +
                    EF[w2][2] * Dk[(ic * n + j) * 3 + 2]) *
                   Pk[jc * n + j];
          beta += (0. + a) - conj(b);
        }
        pv[ic * n + jc] = -I * beta;
        if (ic < nch && jc >= nch) pv[ic * n + jc] += -I * (-wx2 * Pk[ic * n + jc]);
      }
    /* dissipation (RungeKutta.h:219-254) */
    if (o->n_diss > 0) {
      const cplx* Uk = &o->U[IDX3(ik, 0, 0, n)];
      const cplx* hUk = &o->hU[IDX3(ik, 0, 0, n)];
      cplx Mk[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
      for (int e = 0; e < n * n; e++) Mk[e] = 0;
      for (int t = 0; t < o->n_diss; t++) {
        int ii = o->diss_i[t], jj = o->diss_j[t];
        for (int i = 0; i < n; i++)
          for (int j = 0; j < n; j++) Mk[ii * n + jj] += conj(Uk[ii * n + i]) * Uk[jj * n + j] * Pk[i * n + j];
      }
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic; jc < n; jc++) {
          for (int t = 0; t < o->n_diss; t++) {
            int ii = o->diss_i[t], jj = o->diss_j[t];
            pv[ic * n + jc] -= hUk[jc * n + jj] * conj(Uk[ic * n + ii]) * o->T[ii][jj] * Mk[ii * n + jj];
          }
          cplx Tii = 0.;
          for (int i = 0; i < o->nbands; i++) Tii += hUk[jc * n + i] * conj(hUk[ic * n + i]) * o->T[i][i];
          pv[ic * n + jc] += Tii;
        }
    }
    /* k gradient (RungeKutta.h:258-276) */
    if (e_non0) {
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic; jc < n; jc++) {
          cplx g = 0.;
          for (int b = 0; b < o->nnb; b++) {
            int kb = o->nbr[(size_t)ik * o->nnb + b];
            for (int i = 0; i < 3; i++) g += o->weights[o->bshell[b]] * EF[0][i] * o->bvec[b][i] * P[IDX3(kb, ic, jc, n)];
          }
          pv[ic * n + jc] += g;
        }
    }
    /* hermitize (RungeKutta.h:283-294) */
    for (int ic = 0; ic < n; ic++) {
      pv[ic * n + ic] = creal(pv[ic * n + ic]);
      for (int jc = ic + 1; jc < n; jc++) pv[jc * n + ic] = conj(pv[ic * n + jc]);
    }
  }
}

/* headers/RungeKutta.h:301-328 / :331-355 */
static void rk_ad(orc* o, const cplx* P0, cplx* P1, const cplx* Pv, double dt) {
  size_t tot = (size_t)o->nk * o->ncv * o->ncv;
#pragma omp parallel for schedule(static)
  for (size_t e = 0; e < tot; e++) P1[e] = P0[e] + Pv[e] * dt;
}
static void rk_ac(orc* o, cplx* P0, const cplx* Pv, double dt) {
  size_t tot = (size_t)o->nk * o->ncv * o->ncv;
#pragma omp parallel for schedule(static)
  for (size_t e = 0; e < tot; e++) P0[e] += Pv[e] * dt;
}

/* ------------------------------------------------------------ observables */

/* headers/InitParameters.h:264-335 (get_P_in_dia_vect), diagonal only */
static void pop_diag(int n, const cplx* Pk, const cplx* Uk, double* out) {
  cplx Pp[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Mk[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  for (int ic = 0; ic < n; ic++)
    for (int jc = ic; jc < n; jc++) {
      Pp[ic * n + jc] = Pk[ic * n + jc];
      if (ic != jc) Pp[jc * n + ic] = conj(Pp[ic * n + jc]);
    }
  for (int ii = 0; ii < n; ii++)
    for (int jc = 0; jc < n; jc++) {
      cplx acc = 0;
      for (int jj = 0; jj < n; jj++) acc += Pp[ii * n + jj] * Uk[jc * n + jj];
      Mk[jc * n + ii] = acc;
    }
  for (int ic = 0; ic < n; ic++) {
    cplx acc = 0;
    for (int ii = 0; ii < n; ii++) acc += conj(Uk[ic * n + ii]) * Mk[ic * n + ii];
    out[ic] = creal(acc);
  }
}

/* headers/Observables_MPI.h:217-484 (PrintLossesMPI_exciton), :668-775
 * (Current1/2), :559-598 (TransientAbs). Uses o->Hr for Coulomb. */
static void observables(orc* o, const cplx* P, edus_obs* ob) {
  int n = o->ncv, nk = o->nk, ncc = o->nbands, nch = o->nch;
  const int nth = NBLK;
  double* popp = calloc((size_t)nth * n, sizeof(double));
  double* pmax = calloc(nth, sizeof(double));
  double* pmin = malloc(sizeof(double) * nth);
  cplx* j1p = calloc((size_t)nth * 3, sizeof(cplx));
  cplx* j2p = calloc((size_t)nth * 3, sizeof(cplx));
  cplx* tap = calloc((size_t)nth * 3, sizeof(cplx));
  cplx* plp = calloc((size_t)nth * 3, sizeof(cplx));
  for (int t = 0; t < nth; t++) pmin[t] = 1.0;
  if (o->p.coulomb && o->p.current) gradient_energy_renorm(o, o->Hr);
  if (o->vg && o->p.current) gradient_energy_renorm(o, o->H);
  const cplx* Hs = o->p.coulomb ? o->Hr : o->H;
#pragma omp parallel for schedule(static)
  for (int t = 0; t < nth; t++) {
    const int T = nth;
    int len = nk / T, left = nk % T;
    int beg = len * t + (t < left ? t : left);
    int end = beg + len + (t < left ? 1 : 0);
    for (int ik = beg; ik < end; ik++) {
      const cplx* Pk = &P[IDX3(ik, 0, 0, n)];
      cplx Uex[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
      if (o->p.coulomb || o->vg) {
        cplx A[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Z[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
        double ev[EDUS_MAX_BANDS];
        memcpy(A, o->vg ? &o->H[(size_t)ik * n * n] : &o->Hr[(size_t)ik * n * n], sizeof(cplx) * n * n);
        eig_herm(n, A, ev, Z);
        for (int ic = 0; ic < n; ic++)
          for (int jc = 0; jc < n; jc++) Uex[ic * n + jc] = conj(Z[jc * n + ic]);
      } else {
        memcpy(Uex, &o->U[IDX3(ik, 0, 0, n)], sizeof(cplx) * n * n);
      }
      double pd[EDUS_MAX_BANDS];
      pop_diag(n, Pk, Uex, pd);
      for (int ic = 0; ic < n; ic++) {
        double Pik = pd[ic];
        popp[t * n + ic] += Pik;
        if (ic < ncc) {
          if (fabs(1. - Pik) > pmax[t]) pmax[t] = fabs(1. - Pik);
          if ((1. - Pik) < pmin[t]) pmin[t] = 1. - Pik;
        } else {
          if (fabs(Pik) > pmax[t]) pmax[t] = fabs(Pik);
          if (Pik < pmin[t]) pmin[t] = Pik;
        }
      }
      /* polarisation (an extension, no reference counterpart): Tr(D_x rho) =
         sum_ij D_x,ij P_ij with P[k][i][j] = rho_ji */
      for (int ic = 0; ic < n; ic++)
        for (int jc = 0; jc < n; jc++)
          for (int x = 0; x < 3; x++) plp[t * 3 + x] += o->D[IDX4(ik, ic, jc, x, n)] * Pk[ic * n + jc];
      if (o->p.current) {
        for (int ic = 0; ic < n; ic++)
          for (int jc = 0; jc < n; jc++)
            for (int x = 0; x < 3; x++) j1p[t * 3 + x] += Pk[ic * n + jc] * o->GE[IDX4(ik, ic, jc, x, n)];
        for (int ic = 0; ic < n; ic++)
          for (int jc = 0; jc < n; jc++)
            for (int kc = 0; kc < n; kc++)
              for (int x = 0; x < 3; x++)
                j2p[t * 3 + x] += Pk[ic * n + jc] * Hs[IDX3(ik, ic, kc, n)] * conj(o->D[IDX4(ik, jc, kc, x, n)]);
      }
    }
  }
  /* CalculateTransientAbs runs on the master thread: one sequential sum */
  if (o->p.tabs)
    for (int ik = 0; ik < nk; ik++)
      for (int ic = 0; ic < nch; ic++)
        for (int jc = nch; jc < n; jc++)
          for (int x = 0; x < 3; x++) tap[x] -= 2. * o->D[IDX4(ik, ic, jc, x, n)] * P[IDX3(ik, ic, jc, n)];
  double nktot_inv = 1. / nk;
  double popg[EDUS_MAX_BANDS];
  double pmx = 0, pmn = 1.0;
  cplx J1[3] = {0, 0, 0}, J2[3] = {0, 0, 0}, TA[3] = {0, 0, 0}, PL[3] = {0, 0, 0};
  for (int ic = 0; ic < n; ic++) popg[ic] = 0;
  for (int t = 0; t < nth; t++) {
    if (pmx < pmax[t]) pmx = pmax[t];
    if (pmn > pmin[t]) pmn = pmin[t];
    for (int ic = 0; ic < n; ic++) popg[ic] += popp[t * n + ic] * nktot_inv;
    for (int x = 0; x < 3; x++) {
      J1[x] += j1p[t * 3 + x];
      J2[x] += j2p[t * 3 + x];
      PL[x] += plp[t * 3 + x];
    }
  }
  for (int x = 0; x < 3; x++) TA[x] = tap[x];
  double ptrace = -ncc;
  for (int ic = 0; ic < n; ic++) {
    ptrace += popg[ic];
    if (ic < ncc) popg[ic] = 1.0 - popg[ic];
  }
  double ncond = 0;
  for (int ic = 0; ic < n; ic++)
    if (popg[ic] > ncond) ncond = popg[ic];
  double sc = o->dk[0] * o->dk[1] * o->dk[2] / o->det_a;
  memset(ob, 0, sizeof(*ob));
  for (int ic = 0; ic < n; ic++) ob->pop[ic] = popg[ic];
  ob->trace_dev = ptrace;
  ob->p_cond_max = pmx;
  ob->p_min = pmn;
  ob->n_cond = ncond;
  for (int x = 0; x < 3; x++) {
    cplx j1 = J1[x] * sc, j2 = J2[x] * sc;
    ob->J1[2 * x] = creal(j1);
    ob->J1[2 * x + 1] = cimag(j1);
    ob->J2[x] = -2. * cimag(j2);
    cplx ta = TA[x] * (fabs(o->jac) * o->dk[0] * o->dk[1] * o->dk[2]);
    ob->tabs[2 * x] = creal(ta) / nk;
    ob->tabs[2 * x + 1] = cimag(ta) / nk;
    ob->pol[2 * x] = creal(PL[x]) / nk;
    ob->pol[2 * x + 1] = cimag(PL[x]) / nk;
  }
  free(plp);
  free(popp);
  free(pmax);
  free(pmin);
  free(j1p);
  free(j2p);
  free(tap);
}

/* ------------------------------------------------------------ time loop */

/* Source_Main/RungeKutta.cpp:1-197 (one RK4 step, incl. E_non0 bookkeeping) */
static void step_rk4_ring(orc* o, int store_ring);
static void step_rk4(orc* o) { step_rk4_ring(o, 0); }
/* store_ring: RK4 start-up of Adams–Bashforth (an option the reference does
 * not have; its AB starts from a zero history): the first-stage derivative is
 * kept in the AB ring so the multistep formula has a true history. */
static void step_rk4_ring(orc* o, int store_ring) {
  int n = o->ncv;
  double dt = o->dt, dt6 = dt / 6.0, dt3 = dt / 3.0, dt2 = dt / 2.0;
  double wx2 = o->p.probe.wl;
  if (o->p.dynamical_dt)
    for (int ik = 0; ik < o->nk; ik++)
      for (int ic = 0; ic < n; ic++) o->Psave_diag[(size_t)ik * n + ic] = o->P0[IDX3(ik, ic, ic, n)];
  double t = o->time_loop;
  /* velocity gauge: H, D at k + A(stage time), no k-gradient term */
  const int grad = o->vg ? 0 : o->e_non0;
  field_at(o, t, o->EF);
  if (o->vg) vg_tables(o, t);
  rhs(o, o->P0, o->Pv, o->EF, wx2, grad);
  if (store_ring) memcpy(o->ring + (size_t)o->nk * n * n * o->ring_idx[0], o->Pv, sizeof(cplx) * (size_t)o->nk * n * n);
  rk_ad(o, o->P0, o->P1, o->Pv, dt6);
  rk_ad(o, o->P0, o->P2, o->Pv, dt2);
  field_at(o, t + dt2, o->EF);
  if (o->vg) vg_tables(o, t + dt2);
  rhs(o, o->P2, o->Pv, o->EF, wx2, grad);
  rk_ac(o, o->P1, o->Pv, dt3);
  rk_ad(o, o->P0, o->P2, o->Pv, dt2);
  rhs(o, o->P2, o->Pv, o->EF, wx2, grad);
  rk_ac(o, o->P1, o->Pv, dt3);
  rk_ad(o, o->P0, o->P2, o->Pv, dt);
  field_at(o, t + dt, o->EF);
  if (o->vg) vg_tables(o, t + dt);
  rhs(o, o->P2, o->Pv, o->EF, wx2, grad);
  rk_ad(o, o->P1, o->P0, o->Pv, dt6);
  if (o->p.dynamical_dt)
    for (size_t e = 0; e < (size_t)o->nk * n; e++) o->Pprev_diag[e] = o->Psave_diag[e];
  o->e_non0 = field_nonzero(o->EF);
}

/* Source_Main/Linear_Multistep_ODE_solvers.cpp:1-93 + headers/ODE_solver.h:66-98,152-181 */
static void step_ab(orc* o) {
  int n = o->ncv, p = o->p.order;
  static const double c1[1] = {1.};
  static const double c2[2] = {3.0 / 2.0, -1.0 / 2.0};
  static const double c3[3] = {23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0};
  static const double c4[4] = {55.0 / 24.0, -59.0 / 24.0, 37.0 / 24.0, -9.0 / 24.0};
  static const double c5[5] = {1901.0 / 720.0, -2774.0 / 720.0, 2616.0 / 720.0, -1274.0 / 720.0, 251.0 / 720.0};
  const double* coef = p == 1 ? c1 : p == 2 ? c2 : p == 3 ? c3 : p == 4 ? c4 : c5;
  field_at(o, o->time_loop, o->EF);
  o->e_non0 = field_nonzero(o->EF);
  int fill = o->ring_idx[p - 1];
  for (int s = p - 1; s > 0; s--) o->ring_idx[s] = o->ring_idx[s - 1];
  o->ring_idx[0] = fill;
  if (o->p.ab_rk4_startup && o->it < p - 1) {
    step_rk4_ring(o, 1);
    return;
  }
  rhs(o, o->P0, o->Pv, o->EF, o->p.probe.wl, o->e_non0);
  size_t st = (size_t)o->nk * n * n;
  memcpy(o->ring + st * o->ring_idx[0], o->Pv, sizeof(cplx) * st);
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++)
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic; jc < n; jc++) {
        cplx d = 0.0;
        for (int s = 0; s < p; s++) d += coef[s] * o->ring[st * o->ring_idx[s] + IDX3(ik, ic, jc, n)];
        o->P0[IDX3(ik, ic, jc, n)] += o->dt * d;
        if (ic != jc) o->P0[IDX3(ik, jc, ic, n)] = conj(o->P0[IDX3(ik, ic, jc, n)]);
      }
}

/* Source_Main/Taylor_DE_solver_deriv_Polynom.cpp:1-177 */
static void step_taylor(orc* o) {
  int n = o->ncv, TO = o->p.order;
  field_at(o, o->time_loop, o->EF);
  o->e_non0 = field_nonzero(o->EF);
  int fill = o->ring_idx[TO - 1];
  for (int s = TO - 1; s > 0; s--) o->ring_idx[s] = o->ring_idx[s - 1];
  o->ring_idx[0] = fill;
  rhs(o, o->P0, o->Pv, o->EF, o->p.probe.wl, o->e_non0);
  if (o->p.dynamical_dt)
    for (int ik = 0; ik < o->nk; ik++)
      for (int ic = 0; ic < n; ic++) o->Pprev_diag[(size_t)ik * n + ic] = o->P0[IDX3(ik, ic, ic, n)];
  size_t st = (size_t)o->nk * n * n;
  memcpy(o->ring + st * o->ring_idx[0], o->Pv, sizeof(cplx) * st);
  int m = TO - 1;
  double ti[16], tau[256], tinv[256];
  ti[0] = o->dt_prev[0];
  for (int i = 1; i < m; i++) ti[i] = ti[i - 1] + o->dt_prev[i - 1];
  double scale = pow(10, 7);
  for (int i = 0; i < m; i++)
    for (int q = 0; q < m; q++) tau[i * m + q] = scale * pow(ti[i], (q + 1));
  inv_gj(m, tau, tinv);
  for (int i = 0; i < m * m; i++) tinv[i] *= scale;
  double dt = o->dt;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++)
    for (int e = 0; e < n * n; e++) {
      cplx dP[16], al[16];
      cplx f0 = o->ring[st * o->ring_idx[0] + (size_t)ik * n * n + e];
      for (int i = 0; i < m; i++) dP[i] = f0 - o->ring[st * o->ring_idx[i + 1] + (size_t)ik * n * n + e];
      for (int i = 0; i < m; i++) {
        cplx acc = 0;
        for (int q = 0; q < m; q++) acc += tinv[i * m + q] * dP[q];
        al[i] = acc;
      }
      cplx d = f0 * dt;
      for (int i = 1; i < TO; i++) d += pow(dt, i + 1) * al[i - 1] / (double)(i + 1);
      o->P0[(size_t)ik * n * n + e] += d;
    }
}

/* Source_Main/dyn_dt_evolution.cpp:64-133 (max_dP and dt update) */
static void adapt_dt(orc* o) {
  int n = o->ncv;
  double mx = 0.0;
  for (int ik = 0; ik < o->nk; ik++)
    for (int ic = 0; ic < n; ic++) {
      double v = 2 * cabs(o->Pprev_diag[(size_t)ik * n + ic] - o->P0[IDX3(ik, ic, ic, n)]) /
                 (o->P_cond_max + o->n_cond + cabs(o->P0[IDX3(ik, ic, ic, n)]) + 1.0e-7);
      if (v > mx) mx = v;
    }
  double eps = o->p.eps_step_abs;
  if ((mx > eps) && (o->dt > 0.01))
    o->dt *= eps / mx;
  else if (o->dt < o->dt0)
    o->dt *= 1.02;
  if (o->p.solver == EDUS_SOLVER_TAYLOR) {
    for (int i = o->p.order - 1; i > 0; i--) o->dt_prev[i] = o->dt_prev[i - 1];
    o->dt_prev[0] = o->dt;
  }
}

static void record(orc* o, edus_obs* ob) {
  observables(o, o->P0, ob);
  ob->t = o->time_loop;
  for (int i = 0; i < 3; i++) {
    ob->EF_pump[i] = o->EF[0][i];
    ob->EF_probe[i] = o->EF[1][i];
  }
  ob->dt = o->dt;
  o->n_cond = ob->n_cond;
  o->n_cond_coul = ob->n_cond;
  o->P_cond_max_loc = ob->p_cond_max;
  o->P_min = ob->p_min;
}

/* Source_Main/const_dt_evolution.cpp:1-54 and dyn_dt_evolution.cpp:1-183 */
int orc_run(orc* o, int max_steps, edus_obs* log, int log_cap, int* n_log) {
  int nl = 0;
  int steps = 0;
  int res = o->p.it_resolution > 0 ? o->p.it_resolution : 1;
  int taylor = o->p.solver == EDUS_SOLVER_TAYLOR;
  int ab = o->p.solver == EDUS_SOLVER_AB && !o->p.dynamical_dt;
  if (!o->p.dynamical_dt) {
    while (o->it <= o->itfi) {
      if (max_steps >= 0 && steps >= max_steps) break;
      if (o->it % res == 0) {
        edus_obs ob;
        record(o, &ob);
        if (log && nl < log_cap) log[nl] = ob;
        nl++;
      }
      if (taylor)
        step_taylor(o);
      else if (ab)
        step_ab(o);
      else
        step_rk4(o);
      if (o->it % (10 * res) == 0) o->P_cond_max = o->P_cond_max_loc;
      o->time_loop += o->dt;
      o->it += 1;
      steps++;
    }
  } else {
    while (o->time_loop < o->p.t_fin) {
      if (max_steps >= 0 && steps >= max_steps) break;
      if (o->it % res == 0) {
        edus_obs ob;
        record(o, &ob);
        if (log && nl < log_cap) log[nl] = ob;
        nl++;
        o->P_cond_max = o->P_cond_max_loc;
      }
      if (taylor)
        step_taylor(o);
      else
        step_rk4(o);
      adapt_dt(o);
      o->time_loop += o->dt;
      o->it += 1;
      steps++;
    }
  }
  if (n_log) *n_log = nl;
  return 0;
}

/* ------------------------------------------------------------ setup */

static void* xcalloc(size_t n, size_t s) {
  void* p = calloc(n ? n : 1, s);
  return p;
}

int orc_create(const edus_params* p, const char* workdir, orc** out) {
  orc* o = xcalloc(1, sizeof(orc));
  if (!o) return EDUS_ENOMEM;
  o->p = *p;
  o->nch = p->nb[0];
  o->nv = p->nb[1];
  o->ncv = p->nb[0] + p->nb[1] + p->nb[2];
  o->nbands = p->nb[0] + p->nb[1];
  int n = o->ncv;
  if (n < 1 || n > EDUS_MAX_BANDS) {
    free(o);
    return EDUS_EINVAL;
  }
  o->nk = p->nk[0] * p->nk[1] * p->nk[2];
  o->n1 = p->nk[1];
  o->n2 = p->nk[2];
  int rc = 0;
  if (p->mode == EDUS_MODE_CRYSTAL) { /* Source_Main/input.cpp:57: the lattice comes from the crystal files */
    rc = crystal_read(o, workdir);
    if (rc) goto fail;
  }
  rc = set_crys_to_cart(o);
  if (rc) goto fail;
  /* det_a (Source_Main/input.cpp:63-73) */
  const double(*la)[3] = o->p.a;
  if (!p->sample_110)
    o->det_a = fabs(la[1][1] * la[2][2] - la[1][2] * la[2][1]);
  else
    o->det_a = fabs(la[0][0] * la[1][1] - la[0][1] * la[1][0]);
  o->kpt = xcalloc((size_t)o->nk * 3, sizeof(double));
  rc = make_grid(o);
  if (rc) goto fail;
  rc = calc_weights(o);
  if (rc) goto fail;
  o->nbr = xcalloc((size_t)o->nk * o->nnb, sizeof(int));
  rc = calc_indices(o);
  if (rc) goto fail;
  size_t st = (size_t)o->nk * n * n;
  o->H = xcalloc(st, sizeof(cplx));
  o->U = xcalloc(st, sizeof(cplx));
  o->hU = xcalloc(st, sizeof(cplx));
  o->D = xcalloc(st * 3, sizeof(cplx));
  o->GE = xcalloc(st * 3, sizeof(cplx));
  if (p->mode == EDUS_MODE_WANNIER) {
    rc = wannier_read(o, workdir);
  } else if (p->mode == EDUS_MODE_TB) {
    rc = tb_init(o);
  }
  if (rc) goto fail;
  rc = tabulate(o);
  if (rc) goto fail;
  if (p->current) gradient_energy(o, o->H);
  init_T(o);
  o->P0 = xcalloc(st, sizeof(cplx));
  o->P1 = xcalloc(st, sizeof(cplx));
  o->P2 = xcalloc(st, sizeof(cplx));
  o->Pv = xcalloc(st, sizeof(cplx));
  o->Pprev_diag = xcalloc((size_t)o->nk * n, sizeof(cplx));
  o->Psave_diag = xcalloc((size_t)o->nk * n, sizeof(cplx));
  initial_population(o);
  int ord = p->order > 0 ? p->order : 5;
  if (p->solver != EDUS_SOLVER_RK4) {
    o->ring = xcalloc(st * ord, sizeof(cplx));
    for (int i = 0; i < ord; i++) o->ring_idx[i] = i;
  }
  o->dt = p->dt;
  o->dt0 = p->dt;
  for (int i = 0; i < 16; i++) o->dt_prev[i] = p->dt;
  o->it = 0;
  o->time_loop = -0.21 / TIME_AU_FS;
  o->itfi = (int)((p->t_fin - o->time_loop) / p->dt);
  o->e_non0 = 1;
  o->n_cond = p->dynamical_dt ? pow(10, -16) : 0;
  if (p->velocity_gauge) {
    if (p->mode != EDUS_MODE_WANNIER || p->solver != EDUS_SOLVER_RK4 || p->dynamical_dt || p->coulomb ||
        p->conduction_shift > 1e-16 || o->n_diss > 0) {
      orc_free(o);
      return EDUS_EUNSUPPORTED;
    }
    o->vg = 1;
    o->A_t = o->time_loop;
  }
  o->P_cond_max = 0;
  if (p->coulomb) {
    o->ncut = p->ncut;
    size_t c2 = (size_t)o->ncut * o->ncut * n * n;
    o->cA = xcalloc(c2, sizeof(cplx));
    o->cB = xcalloc(c2, sizeof(cplx));
    o->cC = xcalloc(c2, sizeof(cplx));
    o->cD = xcalloc(c2, sizeof(cplx));
    o->Xcc = xcalloc(c2, sizeof(cplx));
    o->Xcs = xcalloc(c2, sizeof(cplx));
    o->Xsc = xcalloc(c2, sizeof(cplx));
    o->Xss = xcalloc(c2, sizeof(cplx));
    o->Xcc0 = xcalloc(c2, sizeof(cplx));
    o->Xcs0 = xcalloc(c2, sizeof(cplx));
    o->Xsc0 = xcalloc(c2, sizeof(cplx));
    o->Xss0 = xcalloc(c2, sizeof(cplx));
    o->cos_m1 = xcalloc((size_t)o->ncut * o->nk, sizeof(double));
    o->sin_m1 = xcalloc((size_t)o->ncut * o->nk, sizeof(double));
    o->cos_m2 = xcalloc((size_t)o->ncut * o->nk, sizeof(double));
    o->sin_m2 = xcalloc((size_t)o->ncut * o->nk, sizeof(double));
    o->PW0 = xcalloc(st, sizeof(cplx));
    o->Hr = xcalloc(st, sizeof(cplx));
    if (!p->read_from_files) {
      rc = EDUS_EUNSUPPORTED;
      goto fail;
    }
    o->Pd = xcalloc(st, sizeof(cplx));
    rc = coulomb_read(o, workdir);
    if (rc) goto fail;
    trig_tables(o);
    memcpy(o->Hr, o->H, sizeof(cplx) * st);
    /* main_MPI.cpp:276-337: equilibrium coefficients (diagonal basis: of the
     * equilibrium state in the eigenbasis, 1 on the filled bands) */
    if (p->diag_basis) {
      for (int ik = 0; ik < o->nk; ik++)
        for (int ic = 0; ic < o->nbands; ic++) o->Pd[IDX3(ik, ic, ic, n)] = 1.0;
      coulomb_coeffs(o, o->Pd);
    } else {
      coulomb_coeffs(o, o->P0);
    }
    memcpy(o->Xcc0, o->Xcc, sizeof(cplx) * c2);
    memcpy(o->Xcs0, o->Xcs, sizeof(cplx) * c2);
    memcpy(o->Xsc0, o->Xsc, sizeof(cplx) * c2);
    memcpy(o->Xss0, o->Xss, sizeof(cplx) * c2);
    for (int i = 0; i < n; i++) o->EH0[i] = o->EH[i];
    memcpy(o->PW0, o->P0, sizeof(cplx) * st);
  }
  *out = o;
  return 0;
fail:
  orc_free(o);
  return rc;
}

void orc_free(orc* o) {
  if (!o) return;
  void* ptrs[] = {o->kpt, o->nbr, o->H, o->U, o->hU, o->D, o->GE, o->Rvec, o->HR, o->xR, o->yR, o->zR,
                  o->P0, o->P1, o->P2, o->Pv, o->Pgrad, o->ring, o->Pprev_diag, o->Psave_diag, o->cA, o->cB,
                  o->cC, o->cD, o->Xcc, o->Xcs, o->Xsc, o->Xss, o->Xcc0, o->Xcs0, o->Xsc0, o->Xss0,
                  o->cos_m1, o->sin_m1, o->cos_m2, o->sin_m2, o->PW0, o->Hr, o->Pd, o->cyH, o->cyDx, o->cyDy};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
  free(o);
}

int orc_info(const orc* o, edus_problem_info* out) {
  memset(out, 0, sizeof(*out));
  out->ncv = o->ncv;
  out->nch = o->nch;
  out->nv = o->nv;
  out->nc = o->p.nb[2];
  out->nk = o->nk;
  out->n1 = o->n1;
  out->n2 = o->n2;
  out->nshell = o->nshell;
  out->nnb = o->nnb;
  out->nrpts = o->nrpts;
  out->n_diss = o->n_diss;
  out->nsteps = o->itfi + 1;
  int res = o->p.it_resolution > 0 ? o->p.it_resolution : 1;
  out->nprint = o->itfi / res + 1;
  out->t_start = -0.21 / TIME_AU_FS;
  out->det_a = o->det_a;
  out->jacobian = o->jac;
  for (int i = 0; i < 3; i++) out->dk[i] = o->dk[i];
  return 0;
}

static int copy_named(const orc* o, const char* name, void** ptr, size_t* nb) {
  size_t st = (size_t)o->nk * o->ncv * o->ncv;
  static double wbuf[MAXNB];
  if (!strcmp(name, "kpt")) {
    *ptr = o->kpt;
    *nb = sizeof(double) * 3 * o->nk;
  } else if (!strcmp(name, "H")) {
    *ptr = o->H;
    *nb = sizeof(cplx) * st;
  } else if (!strcmp(name, "U")) {
    *ptr = o->U;
    *nb = sizeof(cplx) * st;
  } else if (!strcmp(name, "D")) {
    *ptr = o->D;
    *nb = sizeof(cplx) * st * 3;
  } else if (!strcmp(name, "GE")) {
    *ptr = o->GE;
    *nb = sizeof(cplx) * st * 3;
  } else if (!strcmp(name, "P0")) {
    *ptr = o->P0;
    *nb = sizeof(cplx) * st;
  } else if (!strcmp(name, "Hr")) {
    *ptr = o->Hr;
    *nb = o->Hr ? sizeof(cplx) * st : 0;
  } else if (!strcmp(name, "nbr")) {
    *ptr = o->nbr;
    *nb = sizeof(int) * o->nk * o->nnb;
  } else if (!strcmp(name, "bvec")) {
    *ptr = (void*)o->bvec;
    *nb = sizeof(double) * 3 * o->nnb;
  } else if (!strcmp(name, "weights")) {
    for (int b = 0; b < o->nnb; b++) wbuf[b] = o->weights[o->bshell[b]];
    *ptr = wbuf;
    *nb = sizeof(double) * o->nnb;
  } else {
    return EDUS_EINVAL;
  }
  return 0;
}

int orc_get(const orc* o, const char* name, void* dst, size_t nbytes) {
  void* ptr;
  size_t nb;
  if (copy_named(o, name, &ptr, &nb)) return EDUS_EINVAL;
  if (nb != nbytes) return EDUS_EINVAL;
  memcpy(dst, ptr, nb);
  return 0;
}

int orc_set(orc* o, const char* name, const void* src, size_t nbytes) {
  void* ptr;
  size_t nb;
  if (copy_named(o, name, &ptr, &nb)) return EDUS_EINVAL;
  if (nb != nbytes) return EDUS_EINVAL;
  memcpy(ptr, src, nb);
  return 0;
}

int orc_rhs(orc* o, const double* P, double* Pv, const double EF[6], double wx2, int e_non0) {
  double ef[2][3];
  for (int i = 0; i < 3; i++) {
    ef[0][i] = EF[i];
    ef[1][i] = EF[3 + i];
  }
  rhs(o, (const cplx*)P, (cplx*)Pv, ef, wx2, e_non0);
  return 0;
}

int orc_coulomb_hk(orc* o, const double* P, double* hk) {
  if (!o->p.coulomb) return EDUS_EINVAL;
  coulomb_update(o, (const cplx*)P);
  int n = o->ncv;
#pragma omp parallel for schedule(static)
  for (int ik = 0; ik < o->nk; ik++) coulomb_hk_any(o, ik, (const cplx*)P, (cplx*)hk + (size_t)ik * n * n);
  return 0;
}

int orc_observables(orc* o, const double* P, edus_obs* out) {
  observables(o, (const cplx*)P, out);
  return 0;
}

int orc_clock(const orc* o, int* it, double* t, double* dt) {
  if (it) *it = o->it;
  if (t) *t = o->time_loop;
  if (dt) *dt = o->dt;
  return 0;
}

/* ------------------------------------------------- Coulomb coefficient generator */

/* headers/Coulomb.h:60-83 (Coloumb_THh_F) */
static double gen_v(double q_mod, double qTF, double eps_area, double r0, int rk) {
  double Num = 2 * PI, Den;
  if (rk)
    Den = eps_area * sqrt(q_mod + qTF * qTF) * (sqrt(q_mod) * r0 + 1.0);
  else
    Den = eps_area * sqrt(q_mod + qTF * qTF);
  return Num / Den;
}

/* headers/Coulomb.h:87-157 (Create_Wq_with_G_sum): Wq[n][n] at (qx, qy) */
static void gen_wq(const orc* o, double qx, double qy, const int* G, int ng, const double* disp, double qTF, double eps_area,
                   int hartree, cplx* Wq) {
  int n = o->ncv;
  for (int i = 0; i < n * n; i++) Wq[i] = 0;
  for (int g = 0; g < ng; g++) {
    double c[3], x[3];
    if (o->p.sample_110) {
      c[0] = qx + G[2 * g];
      c[1] = qy + G[2 * g + 1];
      c[2] = 0.0;
    } else {
      c[0] = 0.0;
      c[1] = qx + G[2 * g];
      c[2] = qy + G[2 * g + 1];
    }
    crys_to_cart(o, c, x);
    double Vq;
    if (hartree && ((double)G[2 * g] + (double)G[2 * g + 1]) < 1e-16)
      Vq = 0.0;
    else
      Vq = gen_v(x[0] * x[0] + x[1] * x[1] + x[2] * x[2], qTF, eps_area, o->p.r0, o->p.rytova_keldysh);
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic; jc < n; jc++) {
        if (ic + jc == 0) Wq[0] += Vq;
        if (jc != ic) {
          double phi = 0.0;
          for (int i = 0; i < 3; i++) phi += x[i] * (disp[ic * 3 + i] - disp[jc * 3 + i]);
          Wq[ic * n + jc] += Vq * cexp(I * phi);
        }
      }
    for (int ic = 1; ic < n; ic++) Wq[ic * n + ic] = Wq[0];
  }
}

/* Source_Main/Fourier_Coulomb.cpp:95-500 with the Simpson grid of
 * headers/integrationWeight.h:5-15. what: bit 0 the Hartree table, bit 1 the
 * Fourier coefficients A..D, bit 2 the screening constant (needs bit 1).
 * n_sum / n_sum_screen: grid points per axis (the reference: 4999, 39999). */
int orc_coulomb_generate(const edus_params* p, const char* workdir, int what, int n_sum, int n_sum_screen, double* A,
                         double* B, double* C, double* D, double* screen, double* VH, int* g_num) {
  edus_params q = *p;
  q.coulomb = 0;
  orc* o = NULL;
  int rc = orc_create(&q, workdir, &o);
  if (rc) return rc;
  const int n = o->ncv, n2 = n * n, ncut = p->ncut;
  /* Displacement_orb: diagonal dipoles at k = (0, 0.3, 0.1) (Fourier_Coulomb.cpp:41-67) */
  double disp[EDUS_MAX_BANDS * 3];
  {
    double kc[3] = {0.0, 0.3, 0.1};
    if (p->sample_110) {
      kc[0] = 0.3;
      kc[1] = 0.1;
      kc[2] = 0.0;
    }
    for (int ic = 0; ic < n; ic++)
      for (int x = 0; x < 3; x++) {
        cplx d;
        if (p->mode == EDUS_MODE_WANNIER) {
          const cplx* R = x == 0 ? o->xR : (x == 1 ? o->yR : o->zR);
          d = wannier_sum(o, R, ic, ic, kc);
        } else {
          d = tb_dipole(o, ic, ic, x);
        }
        disp[ic * 3 + x] = creal(d);
      }
  }
  double det_b = p->sample_110 ? fabs(p->b[0][0] * p->b[1][1] - p->b[0][1] * p->b[1][0])
                               : fabs(p->b[1][1] * p->b[2][2] - p->b[1][2] * p->b[2][1]);
  double eps_area = p->epsilon_static * o->det_a;
  double gdist = p->G_distance * sqrt(det_b);
  /* G list (Fourier_Coulomb.cpp:113-136) */
  int bord = (int)(sqrt(9999.0 * 9999.0) / 2);
  int cap = 1 << 20, ng = 0;
  int* G = malloc(sizeof(int) * 2 * cap);
  for (int ix = -bord; ix <= bord; ix++)
    for (int iy = -bord; iy <= bord; iy++) {
      double c[3] = {0.0, (double)ix, (double)iy}, x[3];
      if (p->sample_110) {
        c[0] = ix;
        c[1] = iy;
        c[2] = 0.0;
      }
      crys_to_cart(o, c, x);
      if (sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) < gdist) {
        if (ng == cap) {
          cap *= 2;
          G = realloc(G, sizeof(int) * 2 * cap);
        }
        G[2 * ng] = ix;
        G[2 * ng + 1] = iy;
        ng++;
      }
    }
  if (g_num) *g_num = ng;
  cplx Wq[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
  if (what & 1) {
    /* Hartree table (Fourier_Coulomb.cpp:166-214) */
    gen_wq(o, 0.0, 0.0, G, ng, disp, p->qTF, eps_area, 1, Wq);
    cplx V[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    memcpy(V, Wq, sizeof(cplx) * n2);
    for (int ic = 0; ic < n; ic++) {
      if (ic > 0) V[ic * n + ic] = V[0];
      for (int jc = ic; jc < n; jc++) {
        V[jc * n + ic] = creal(V[ic * n + jc]);
        V[ic * n + jc] = V[jc * n + ic];
      }
    }
    for (int i = 0; i < n2; i++) VH[i] = creal(V[i]);
  }
  cplx* cAc = calloc((size_t)ncut * ncut * n2, sizeof(cplx));
  cplx* cBc = calloc((size_t)ncut * ncut * n2, sizeof(cplx));
  cplx* cCc = calloc((size_t)ncut * ncut * n2, sizeof(cplx));
  cplx* cDc = calloc((size_t)ncut * ncut * n2, sizeof(cplx));
  if (what & 2) {
    /* Simpson grid (headers/integrationWeight.h:5-15) and the coefficient sums (Fourier_Coulomb.cpp:233-275) */
    double h = 1.0 / (n_sum - 1), hs = 3.0 * (n_sum - 1);
    double* qg = malloc(sizeof(double) * n_sum);
    double* sp = malloc(sizeof(double) * n_sum);
    for (int i = 0; i < n_sum; i++) qg[i] = -0.5 + i * h;
    sp[0] = 1 / hs;
    for (int i = 1; i < n_sum; i += 2) sp[i] = 4.0 / hs;
    for (int i = 2; i < n_sum; i += 2) sp[i] = 2.0 / hs;
    sp[n_sum - 1] = 1 / hs;
    for (long iq = 0; iq < (long)n_sum * n_sum; iq++) {
      int ix = (int)(iq / n_sum), iy = (int)(iq % n_sum);
      double spxy = sp[ix] * sp[iy], qx = qg[ix], qy = qg[iy];
      gen_wq(o, qx, qy, G, ng, disp, p->qTF, eps_area, 0, Wq);
      for (int mm = 0; mm < ncut * ncut; mm++) {
        int m = mm / ncut, nn = mm % ncut;
        double mq = 2 * PI * m * qx, nq = 2 * PI * nn * qy;
        double tmc = cos(mq), tms = sin(mq), tnc = cos(nq), tns = sin(nq);
        double dA = 4 * spxy * tmc * tnc, dD = 4 * spxy * tms * tns, dB = 4 * spxy * tmc * tns, dC = 4 * spxy * tms * tnc;
        double fac = (m == 0 && nn == 0) ? 0.25 : ((m == 0 || nn == 0) ? 0.5 : 1.0);
        for (int ic = 0; ic < n; ic++)
          for (int jc = ic; jc < n; jc++) {
            int il = ic * n + jc;
            cplx Vq = Wq[il];
            if (ic == 0 && jc == 0) {
              cAc[(size_t)mm * n2] += creal(Vq * dA * fac);
              cDc[(size_t)mm * n2] += creal(Vq * dD * fac);
            }
            if (jc != ic) {
              cAc[(size_t)mm * n2 + il] += creal(dA * Vq * fac);
              cBc[(size_t)mm * n2 + il] += I * cimag(dB * Vq * fac);
              cCc[(size_t)mm * n2 + il] += I * cimag(dC * Vq * fac);
              cDc[(size_t)mm * n2 + il] += creal(dD * Vq * fac);
            }
          }
      }
    }
    free(qg);
    free(sp);
    for (size_t i = 0; i < (size_t)ncut * ncut * n2; i++) {
      A[2 * i] = creal(cAc[i]);
      A[2 * i + 1] = cimag(cAc[i]);
      B[2 * i] = creal(cBc[i]);
      B[2 * i + 1] = cimag(cBc[i]);
      C[2 * i] = creal(cCc[i]);
      C[2 * i + 1] = cimag(cCc[i]);
      D[2 * i] = creal(cDc[i]);
      D[2 * i + 1] = cimag(cDc[i]);
    }
  }
  if ((what & 4) && (what & 2)) {
    /* screening constant (Fourier_Coulomb.cpp:369-470), order 0 */
    int N = n_sum_screen;
    double h = 1.0 / (N - 1), dk2 = 1. / ((double)N * N);
    double q_peak = p->qTF < 0.02 ? 0.02 : p->qTF;
    cplx sum[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    for (int i = 0; i < n2; i++) sum[i] = 0;
    for (long iq = 0; iq < (long)N * N; iq++) {
      double qx = -0.5 + (iq / N) * h, qy = -0.5 + (iq % N) * h;
      double c[3] = {0.0, qx, qy}, x[3];
      if (p->sample_110) {
        c[0] = qx;
        c[1] = qy;
        c[2] = 0.0;
      }
      crys_to_cart(o, c, x);
      double q_mod = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
      if (!(q_mod < q_peak * q_peak && q_mod > pow(10, -17))) continue;
      gen_wq(o, qx, qy, G, ng, disp, 0.0, eps_area, 0, Wq);
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic; jc < n; jc++) {
          int il = ic * n + jc;
          cplx VF = 0.0;
          for (int m = 0; m < ncut; m++)
            for (int nn = 0; nn < ncut; nn++) {
              double tmc = cos(2 * PI * m * qx), tms = sin(2 * PI * m * qx);
              double tnc = cos(2 * PI * nn * qy), tns = sin(2 * PI * nn * qy);
              size_t ix = (size_t)(nn + ncut * m) * n2 + il;
              VF += cAc[ix] * tmc * tnc + cBc[ix] * tmc * tns + cCc[ix] * tms * tnc + cDc[ix] * tms * tns;
            }
          sum[il] += (Wq[il] - VF) * dk2;
        }
    }
    for (int i = 0; i < n2; i++) {
      screen[2 * i] = creal(sum[i]);
      screen[2 * i + 1] = cimag(sum[i]);
    }
  }
  free(cAc);
  free(cBc);
  free(cCc);
  free(cDc);
  free(G);
  orc_free(o);
  return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* unused helpers kept for completeness of the constant table */
double orc_const_c(void) { return C_LIGHT + 0 * ENERGY_AU_EV + 0 * SPACE_AU_A; }
