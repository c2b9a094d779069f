// eig.cuh — small dense Hermitian eigensolver for device code (one matrix per thread).
#pragma once
#include "dev.cuh"

namespace edus {

// Hermitian eigenvectors by cyclic Jacobi; Z columns are eigenvectors,
// eigenvalues ascending (Armadillo eig_sym in Observables_MPI.h:294).
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

}  // namespace edus
