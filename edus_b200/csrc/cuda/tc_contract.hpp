// tc_contract.hpp — tensor-core (tcgen05, split TF32) Wannier contraction.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include <algorithm>

namespace edus {
namespace batch {

struct TcArgs {
  int n, ntri, nk, nr;
  const double* kpt;     // [nk][3]
  const double* Rvec;    // [nr][3]
  const float* Bw;       // [8 ntri][Kp] split coefficients [hi | lo | hi | lo] (host-built)
  const double2* hdiagR; // [n][nr] H_ii(R) for the FP64 band energies
  float* Aw;             // scratch [nk][Kp] split phases
  double* Cw;            // scratch [nk][8 ntri] GEMM result (FP64 sum of FP32 slices)
  float2* H32;           // out [ntri][nk]
  float2* D32;           // out [3][ntri][nk]
  double* Hdiag;         // out [n][nk] FP64 band energies
  double2* Hused;        // out [ntri][nk] FP64 matrix the dynamics uses (for the eigensolve)
  int* err;              // device error word (bounded waits)
};

// K depth of the split GEMM (4 x 2 nr, padded to the K slice)
int tc_pad_k(int nr);
cudaError_t tc_contract(const TcArgs& a, cudaStream_t s);

}  // namespace batch
}  // namespace edus
