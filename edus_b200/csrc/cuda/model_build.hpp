// model_build.hpp — launcher of the device-side Wannier model build.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

namespace edus {
namespace batch {

struct ModelBuildArgs {
  int n, ntri, nk, nr, nnb, nbands, nv;
  int only_h;             // contraction of H alone (D untouched)
  double scissor;         // conduction-band shift (bands{conduction_shift}), 0 = off
  const double* kpt;      // [nk][3] crystal coordinates
  const double* Rvec;     // [nr][3]
  const double2* coef;    // [4][ntri][nr]: H(R), then (r_ij(R) + r_ji(R)) / 2 for x, y, z
  const int* nbr;         // [nnb][nk]
  const double* gb;       // [nnb][3] w_b * b_x
  double2* H;             // [ntri][nk]   out (FP64)
  double2* D;             // [3][ntri][nk] out
  double2* U;             // [n*n][nk]    out
  double2* GE;            // [3][ntri][nk] out, or null
  double2* P0;            // [ntri][nk]   out: initial state
};

cudaError_t build_wannier_model(const ModelBuildArgs& a, cudaStream_t s);
// Second half of the build on a given a.H (FP64): eigenbasis, scissor, rho0, dH/dk.
cudaError_t finish_wannier_model(const ModelBuildArgs& a, cudaStream_t s);
// FP64 H(k) alone (a.only_h) and its b-vector stencil dH/dk into a.GE.
cudaError_t wannier_h_and_gradient(const ModelBuildArgs& a, cudaStream_t s);
cudaError_t planes_to_float(const double2* src, float2* dst, size_t count, cudaStream_t s);
// out[i][k] = Re H[idx(i,i)][k] for the upper-triangle planes of an n-band model
cudaError_t planes_diagonal(const double2* H, double* out, int n, int nk, cudaStream_t s);

}  // namespace batch
}  // namespace edus
