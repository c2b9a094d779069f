// model_build.cu — Wannier model tables built on the device for a batch
// instance (the per-k tabulation of Source_Main/save_HUD.cpp:19-53 over
// headers/Wannier.h:278-304,336-471, plus the eigenbasis, the initial state of
// headers/InitialPopulation.h:2-39 and GradientEnergy of save_HUD.cpp:96-137).
//
//   k_wan_contract  H(k) = sum_R e^{2 pi i k.R} H(R) and the symmetrised dipole
//                   D(k) = sum_R e^{2 pi i k.R} (r_ij(R) + r_ji(R)) / 2, the
//                   imaginary part of every diagonal entry zeroed
//                   (Wannier.h:489-492, save_HUD.cpp:47-51). Phases of a tile of
//                   k points are staged in shared memory and reused by every
//                   output element.
//   k_wan_eig       eigenvectors of H(k) (ascending), U = Z^dagger, the optional
//                   conduction-band scissor H += U^dagger S U, and the initial
//                   state rho0 = sum over filled bands of the U-row projectors.
//   k_wan_ge        dH/dk by the b-vector stencil: sum_b w_b b (H(k+b) - H(k)).
#include "batch.cuh"
#include "eig.cuh"
#include "model_build.hpp"

namespace edus {
namespace batch {
namespace {

constexpr int kContractKT = 8;
constexpr int kContractThreads = 256;

__global__ void __launch_bounds__(kContractThreads) k_wan_contract(ModelBuildArgs a) {
  extern __shared__ double2 ph[];  // [kContractKT][nr]
  const int k0 = blockIdx.x * kContractKT;
  const int nr = a.nr, nk = a.nk, ntri = a.ntri, n = a.n;
  for (int q = threadIdx.x; q < kContractKT * nr; q += blockDim.x) {
    const int kl = q / nr, r = q - kl * nr;
    const int k = min(k0 + kl, nk - 1);
    const double kR = a.kpt[k * 3 + 0] * a.Rvec[r * 3 + 0] + a.kpt[k * 3 + 1] * a.Rvec[r * 3 + 1] + a.kpt[k * 3 + 2] * a.Rvec[r * 3 + 2];
    double s, c;
    sincospi(2.0 * kR, &s, &c);
    ph[q] = make_double2(c, s);
  }
  __syncthreads();
  const int nout = (a.only_h ? 1 : 4) * ntri * kContractKT;
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int kl = o % kContractKT, ce = o / kContractKT;  // ce = comp * ntri + e
    const int k = k0 + kl;
    if (k >= nk) continue;
    const int comp = ce / ntri, e = ce - comp * ntri;
    const double2* cf = a.coef + (size_t)ce * nr;
    const double2* p = ph + kl * nr;
    double2 acc = cz();
    for (int r = 0; r < nr; r++) acc = cadd(acc, cmul(p[r], cf[r]));
    // diagonal entries are real (Wannier.h:489-492)
    bool diag = false;
    for (int i = 0; i < n; i++) diag = diag || (e == i * n - (i * (i - 1)) / 2);
    if (diag) acc.y = 0.;
    if (comp == 0)
      a.H[(size_t)e * nk + k] = acc;
    else
      a.D[((size_t)(comp - 1) * ntri + e) * nk + k] = acc;
  }
}

template <int N>
__global__ void __launch_bounds__(64) k_wan_eig(ModelBuildArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = a.nk;
  if (k >= nk) return;
  auto up = [](int i, int j) { return i * N - (i * (i - 1)) / 2 + (j - i); };
  double2 A[N * N], Z[N * N];
  for (int i = 0; i < N; i++)
    for (int j = i; j < N; j++) {
      const double2 v = a.H[(size_t)up(i, j) * nk + k];
      A[i * N + j] = v;
      A[j * N + i] = cconj(v);
    }
  eig_herm_dev<N>(A, Z);
  // U[i][j] = conj(Z[j][i]) (rows are eigenvectors, as the host build stores them)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) a.U[((size_t)i * N + j) * nk + k] = cconj(Z[j * N + i]);
  auto U = [&](int i, int j) { return cconj(Z[j * N + i]); };
  if (a.scissor > 1e-16)
    for (int i = 0; i < N; i++)
      for (int j = i; j < N; j++) {
        double2 v = cz();
        for (int ii = 0; ii < N; ii++)
          if (ii >= a.nv) v = cadd(v, cscale(cmul(cconj(U(ii, i)), U(ii, j)), a.scissor));
        const size_t o = (size_t)up(i, j) * nk + k;
        a.H[o] = cadd(a.H[o], v);
      }
  for (int ia = 0; ia < N; ia++)
    for (int ib = ia; ib < N; ib++) {
      double2 acc = cz();
      for (int ii = 0; ii < a.nbands; ii++) acc = cadd(acc, cmul(U(ii, ia), cconj(U(ii, ib))));
      a.P0[(size_t)up(ia, ib) * nk + k] = acc;
    }
}

__global__ void k_wan_ge(ModelBuildArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = blockIdx.y;
  const int nk = a.nk;
  if (k >= nk) return;
  const double2 h0 = a.H[(size_t)e * nk + k];
  double2 g[3] = {cz(), cz(), cz()};
  for (int b = 0; b < a.nnb; b++) {
    const int kb = a.nbr[(size_t)b * nk + k];
    const double2 d = csub(a.H[(size_t)e * nk + kb], h0);
    for (int x = 0; x < 3; x++) g[x] = cadd(g[x], cscale(d, a.gb[b * 3 + x]));
  }
  for (int x = 0; x < 3; x++) a.GE[((size_t)x * a.ntri + e) * nk + k] = g[x];
}

__global__ void k_to_float(const double2* __restrict__ src, float2* __restrict__ dst, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

__global__ void k_diag(const double2* __restrict__ H, double* __restrict__ out, int n, int nk) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (k < nk) out[(size_t)i * nk + k] = H[(size_t)(i * n - (i * (i - 1)) / 2) * nk + k].x;
}

}  // namespace

cudaError_t planes_diagonal(const double2* H, double* out, int n, int nk, cudaStream_t s) {
  k_diag<<<dim3((nk + 255) / 256, n), 256, 0, s>>>(H, out, n, nk);
  return cudaGetLastError();
}

cudaError_t build_wannier_model(const ModelBuildArgs& a, cudaStream_t s) {
  const size_t smem = sizeof(double2) * kContractKT * a.nr;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_wan_contract, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_wan_contract<<<(a.nk + kContractKT - 1) / kContractKT, kContractThreads, smem, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_wannier_model(a, s);
}

cudaError_t finish_wannier_model(const ModelBuildArgs& a, cudaStream_t s) {
  cudaError_t e;
  const int blocks = (a.nk + 63) / 64;
  switch (a.n) {
    case 2: k_wan_eig<2><<<blocks, 64, 0, s>>>(a); break;
    case 3: k_wan_eig<3><<<blocks, 64, 0, s>>>(a); break;
    case 4: k_wan_eig<4><<<blocks, 64, 0, s>>>(a); break;
    case 5: k_wan_eig<5><<<blocks, 64, 0, s>>>(a); break;
    case 8: k_wan_eig<8><<<blocks, 64, 0, s>>>(a); break;
    case 16: k_wan_eig<16><<<blocks, 64, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (a.GE) {
    k_wan_ge<<<dim3((a.nk + 127) / 128, a.ntri), 128, 0, s>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t wannier_h_and_gradient(const ModelBuildArgs& a, cudaStream_t s) {
  const size_t smem = sizeof(double2) * kContractKT * a.nr;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_wan_contract, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_wan_contract<<<(a.nk + kContractKT - 1) / kContractKT, kContractThreads, smem, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !a.GE) return e;
  k_wan_ge<<<dim3((a.nk + 127) / 128, a.ntri), 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t planes_to_float(const double2* src, float2* dst, size_t count, cudaStream_t s) {
  if (!count) return cudaSuccess;
  const int blocks = (int)std::min<size_t>((count + 255) / 256, 148 * 16);
  k_to_float<<<blocks, 256, 0, s>>>(src, dst, count);
  return cudaGetLastError();
}

}  // namespace batch
}  // namespace edus
