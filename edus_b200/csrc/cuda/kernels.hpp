// kernels.hpp — host-side launch API of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include "../../../include/edus_b200.h"
#include "dev.cuh"

namespace edus {

using ObsRecord = edus_obs;

// Device buffers of the Coulomb mean field (separable truncated transform).
struct CoulDev {
  double2* g = nullptr;        // [n1][2][ncut][ntri] row transform of rho
  const double* t1c = nullptr; // [ncut][n1] cos(2 pi m k1)
  const double* t1s = nullptr;
  const double* t2c = nullptr; // [ncut][n2] cos(2 pi n k2)
  const double* t2s = nullptr;
  const double* t2T = nullptr; // [n2][2 ncut] cos then sin, transposed for the row pass
  const double* t1P = nullptr; // [2][ncut][n1|1] cos / sin rows padded to an odd stride
  const double2* A = nullptr;  // [ncut^2][ntri] coefficients, diagonal rule applied
  const double2* B = nullptr;
  const double2* C = nullptr;
  const double2* D = nullptr;
  const unsigned char* is_diag = nullptr;  // [ntri]
  const int* diag_of = nullptr;            // [ntri] band of a diagonal element
  double2* fdiag = nullptr;                // [n] f_cc(0,0) of the diagonal
};

cudaError_t launch_rhs(const DevTables& tb, const DevConsts* cst, const StageArgs& a, cudaStream_t s);
cudaError_t coulomb_prepare(const DevTables& tb);
size_t coulomb_t2T_count(int n2, int ncut);
size_t coulomb_t1P_count(int n1, int ncut);
cudaError_t launch_coulomb(const DevTables& tb, const CoulDev& c, const double2* rho, double2* h, double2* Xout,
                           const double2* X0, cudaStream_t s);
// Elements (ic, jc), (ic, ic), (jc, jc) of rho in the eigenbasis of tb.U for
// every k: out[3][nk].
// With dyn (adaptive step on the device), out is the base of the snapshot
// slots and the slot is dyn->snap_slot (nothing when it is negative).
cudaError_t launch_snapshot(const DevTables& tb, const double2* rho, int ic, int jc, double2* out, cudaStream_t s,
                            const DynStep* dyn = nullptr);
// Ascending eigenvalues of the Hermitian planes hr at every k: out[n][nk]
// (slot dyn->snap_slot of out with dyn, as above).
cudaError_t launch_band_energies(const DevTables& tb, const double2* hr, double* out, cudaStream_t s,
                                 const DynStep* dyn = nullptr);
// d = a + dt * v elementwise (n complex entries; d may alias a).
cudaError_t launch_axpy(const double2* a, const double2* v, double dt, double2* d, size_t n, cudaStream_t s);
// Coulomb in the diagonal basis, up to 4 bands: the state in the eigenbasis of
// tb.U (upper planes), and the screened mean-field term rotated back to the
// Wannier basis from the inverse-transform rows tb.h.
cudaError_t launch_pdiag(const DevTables& tb, const double2* rho, double2* pd, cudaStream_t s);
cudaError_t launch_coulomb_xw(const DevTables& tb, const DevConsts* cst, const double2* pd, double2* xw, cudaStream_t s);
// Velocity gauge: H(k + A), D(k + A) of a Wannier model at every k point
// (vgauge.cu). coef: [4][ntri][nr] upper-triangle coefficients of H(R) and of
// the symmetric dipoles (r_x(R) + r_x(R)^T) / 2; A in crystal coordinates.
struct VgArgs {
  int n = 0, ntri = 0, nk = 0, nr = 0;
  const double* kpt = nullptr;    // [nk][3] crystal coordinates
  const double* Rvec = nullptr;   // [nr][3]
  const double2* coef = nullptr;  // [4][ntri][nr]
  double A[3] = {0, 0, 0};
  double2* H = nullptr;           // out [ntri][nk]
  double2* D = nullptr;           // out [3][ntri][nk]
};
cudaError_t launch_vg_tables(const VgArgs& a, cudaStream_t s);
int obs_parts(int nk);
size_t obs_part_bytes();
cudaError_t launch_observables(const DevTables& tb, const DevConsts* cst, const double2* rho, const double2* hr,
                               int want_current, int want_tabs, void* part, unsigned int* done, double scaleJ,
                               double scaleTA, const ObsRecord& rec, ObsRecord* log, double* ncond_dev,
                               double* pcmax_dev, cudaStream_t s, const DynStep* dyn = nullptr);

}  // namespace edus
