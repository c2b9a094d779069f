// tc_contract.hpp — tensor-core (tcgen05, exact BF16 slices) Wannier contraction.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstring>
#include <stddef.h>

#include <algorithm>

namespace edus {
namespace batch {

struct TcArgs {
  int n, ntri, nk, nr;
  const double* kpt;     // [nk][3]
  const double* Rvec;    // [nr][3]
  const uint16_t* Bw;    // [8 ntri][Kp] coefficient slices (BF16), one K segment per slice pair (host-built)
  const double2* hdiagR; // [n][nr] H_ii(R) for the FP64 band energies
  uint16_t* Aw;          // scratch [nk][Kp] phase slices (BF16), one K segment per slice pair
  double* Cw;            // scratch [nk][8 ntri] GEMM result (FP64 sum of FP32 slices)
  float2* H32;           // out [ntri][nk]
  float2* D32;           // out [3][ntri][nk]
  double* Hdiag;         // out [n][nk] FP64 band energies
  double2* Hused;        // out [ntri][nk] FP64 matrix the dynamics uses (for the eigensolve)
  int* err;              // device error word (bounded waits)
};

// Exact-slice form of the contraction. Every operand y (half a phase cos / sin,
// or a coefficient divided by its column's power-of-two scale) lies in
// [-1/2, 1/2] and is cut into kTcSlices slices of at most 8 significant bits,
// slice s a multiple of 2^-(8 s + 8) and at most 128 in magnitude:
// y = sum_s slice_s(y) + O(2^-33); every slice is exact in BF16. The GEMM runs
// one K segment per slice pair
// (a, b) with a + b < kTcSlices; inside a segment every product is an integer
// times one power of two, at most 2^14 in magnitude, so the tensor core's FP32
// sums over a segment of up to 1024 are exact and the FP64 sum of the segments
// is the contraction to about 2^-32 of its terms.
constexpr int kTcSlices = 4;
constexpr int kTcPairs = 10;  // (a, b) with a + b <= 3
__host__ __device__ constexpr int tc_pair_a(int p) {
  return p == 0 ? 0 : p == 1 ? 0 : p == 2 ? 1 : p == 3 ? 0 : p == 4 ? 1 : p == 5 ? 2 : p == 6 ? 0 : p == 7 ? 1 : p == 8 ? 2 : 3;
}
__host__ __device__ constexpr int tc_pair_b(int p) {
  return p == 0 ? 0 : p == 1 ? 1 : p == 2 ? 0 : p == 3 ? 2 : p == 4 ? 1 : p == 5 ? 0 : p == 6 ? 3 : p == 7 ? 2 : p == 8 ? 1 : 0;
}
// slice s of y in [-1, 1] (FP64 arithmetic, exact at every step)
__host__ __device__ inline double tc_slice(double y, int s) {
  double r = y, v = 0.;
  double scale = 256.;
  for (int t = 0; t <= s; t++) {
    v = rint(r * scale) / scale;
    r -= v;
    scale *= 256.;
  }
  return v;
}
// BF16 bit pattern of a value with at most 8 significant bits (exact: the low
// 16 bits of its FP32 pattern are zero)
__host__ __device__ inline uint16_t tc_bf16(double v) {
  const float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  return (uint16_t)(u >> 16);
}
// K segment length (2 nr padded to the 64-deep K slice) and the GEMM depth
int tc_seg_k(int nr);
int tc_pad_k(int nr);
cudaError_t tc_contract(const TcArgs& a, cudaStream_t s);

// Velocity gauge on the tensor cores: H(k + A), D(k + A) of every k point for
// every RK4 stage as the exact-slice GEMM above. The phase slices of the grid
// (A' = [cos | sin](2 pi k.R) / 2) are cut once; each stage cuts the
// coefficient slices of c_A(R) = e^{2 pi i A.R} c(R) on the device (column
// scales fixed from |c(R)|, which bounds |Re c_A| and |Im c_A| for every A),
// runs the GEMM and scatters FP64 planes (diagonal imaginary parts zero).
struct TcVgArgs {
  int n = 0, ntri = 0, nk = 0, nr = 0;
  const double* kpt = nullptr;       // [nk][3]
  const double* Rvec = nullptr;      // [nr][3]
  const double2* coef = nullptr;     // [4][ntri][nr]: H(R), (r_x(R) + r_x(R)^T) / 2 upper entries
  const double* colscale = nullptr;  // [8 ntri] power-of-two scale of each GEMM column
  double A[3] = {0, 0, 0};           // crystal coordinates
  uint16_t* Aw = nullptr;            // [nk][Kp] phase slices (tc_vg_prepare)
  uint16_t* Bw = nullptr;            // [8 ntri][Kp] coefficient slices (zero padded once)
  double* Cw = nullptr;              // [nk][8 ntri]
  double2* H = nullptr;              // out [ntri][nk]
  double2* D = nullptr;              // out [3][ntri][nk]
  int* err = nullptr;                // device error word (bounded waits)
  // TMA descriptors of Aw and Bw (tc_vg_maps); without them the cp.async form runs
  bool tma = false;
  CUtensorMap mapA{}, mapB{};
};
cudaError_t tc_vg_prepare(const TcVgArgs& a, cudaStream_t s);
// Encode the TMA descriptors of a.Aw, a.Bw (sets a.tma on success).
cudaError_t tc_vg_maps(TcVgArgs& a);
// A TMA-staged GEMM form (warp-specialised by default, single-issuer with
// EDUS_TC_GEMM=tma) is used unless EDUS_TC_GEMM=cpasync.
bool tc_gemm_tma_wanted();
cudaError_t tc_vg_stage(const TcVgArgs& a, cudaStream_t s);

}  // namespace batch
}  // namespace edus
