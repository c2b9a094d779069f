// tc_contract.cu — the Wannier Fourier sums H(k), D(k) on the tcgen05 tensor
// cores (kind::tf32 with exact integer slices) for mixed-precision batch
// instances.
//
// Real form of the complex sums: with A[k][.] = [cos(2 pi k.R_r) | sin(2 pi k.R_r)]
// (K = 2 nr) and, per output element, the column pair
//   re: [ Re c_r ; -Im c_r ],   im: [ Im c_r ; Re c_r ],
// out = A . B^T gives Re / Im of sum_r e^{2 pi i k.R_r} c_r. Both operands are
// cut into 9-bit slices on a power-of-two scale (tc_contract.hpp): the GEMM
// depth holds one segment of 2 nr (padded to 32) per slice pair (a, b) with
// a + b <= 3. Within a 32-deep K slice every product is an integer times a
// common power of two and at most 2^16, so the tensor core's FP32 sums are
// exact; the slices are added in FP64 registers. The result is the FP64 sum to
// about 2^-32 of the terms, so the FP32 tables stored from it equal those of
// the FP64 CUDA-core build up to the last rounding.
//
// GEMM kernel: one CTA (4 warps) per 128 x 32 tile of C; per 32-deep slice of
// K the block stages A and B in shared memory in the K-major canonical layout
// without swizzle (16-byte rows of 4 TF32, 8-row core matrices 128 bytes
// apart, the two 16-byte halves of one MMA's K = 8 slice one whole operand
// apart), one elected thread issues four tcgen05.mma (M 128, N 32, K 8) and
// commits them to an mbarrier that the block waits on (bounded) before the
// next slice overwrites shared memory. The slice's accumulator (128 lanes x 32
// FP32 columns of TMEM) is read back with tcgen05.ld.32x32b by each warp's lane
// quarter into FP64 registers.
#include <stdint.h>

#include "batch.cuh"
#include "dev.cuh"
#include "tc_contract.hpp"

namespace edus {
namespace batch {
namespace {

constexpr int TM = 128, TN = 32, TK = 32;  // CTA tile and K slice (TF32 elements)
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 32;

// A' rows: phases of k point m over the R vectors; segment p holds slice
// tc_pair_a(p) of [cos | sin], zero padded to the segment length. One phase
// is evaluated once and written to every segment.
__global__ void k_phase_split(const double* __restrict__ kpt, const double* __restrict__ Rvec, int nk, int nr, int kseg,
                              int kpad, float* __restrict__ A) {
  const int m = blockIdx.x;
  const int K = 2 * nr;
  float* row = A + (size_t)m * kpad;
  for (int q = threadIdx.x; q < kseg; q += blockDim.x) {
    float sl[kTcSlices] = {0.f, 0.f, 0.f, 0.f};
    if (m < nk && q < K) {
      const int r = q < nr ? q : q - nr;
      const double kR = kpt[m * 3 + 0] * Rvec[r * 3 + 0] + kpt[m * 3 + 1] * Rvec[r * 3 + 1] + kpt[m * 3 + 2] * Rvec[r * 3 + 2];
      double sn, co;
      sincospi(2.0 * kR, &sn, &co);
      const double y = q < nr ? co : sn;
#pragma unroll
      for (int t = 0; t < kTcSlices; t++) sl[t] = (float)tc_slice(y, t);  // at most 9 significant bits: exact in TF32
    }
#pragma unroll
    for (int p = 0; p < kTcPairs; p++) row[(size_t)p * kseg + q] = sl[tc_pair_a(p)];
  }
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, legacy LBO mode, no swizzle (layout type 0)
  return d;
}

// kind::tf32, D FP32, A and B TF32 K-major, M = 128, N = 32
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

// C (FP64) = A' B'^T. Every 32-deep slice starts a fresh TMEM accumulator and is
// added into FP64 registers, so FP32 rounding spans only 32 exact products.
__global__ void __launch_bounds__(kThreads, 1) k_tc_gemm(const float* __restrict__ A, const float* __restrict__ B, double* __restrict__ C,
                                                         int M, int N, int Kp, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  float* sA = reinterpret_cast<float*>(smem);              // [TK / 4 chunks][TM rows][4]
  float* sB = sA + TM * TK;                                // [TK / 4][TN][4]
  __shared__ unsigned long long bar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) mbar_init(&bar, 1);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
  double acc[TN];
#pragma unroll
  for (int c = 0; c < TN; c++) acc[c] = 0.;
  bool ok = true;
  uint32_t phase = 0;
  for (int k0 = 0; k0 < Kp; k0 += TK) {
    // stage the slice: row r, 16-byte chunk c -> chunk-major, rows contiguous
    for (int q = tid; q < TM * (TK / 4); q += kThreads) {
      const int r = q % TM, c = q / TM;
      const float4 v = (m0 + r < M) ? *reinterpret_cast<const float4*>(A + (size_t)(m0 + r) * Kp + k0 + 4 * c)
                                    : make_float4(0.f, 0.f, 0.f, 0.f);
      *reinterpret_cast<float4*>(sA + (c * TM + r) * 4) = v;
    }
    for (int q = tid; q < TN * (TK / 4); q += kThreads) {
      const int r = q % TN, c = q / TN;
      const float4 v = (n0 + r < N) ? *reinterpret_cast<const float4*>(B + (size_t)(n0 + r) * Kp + k0 + 4 * c)
                                    : make_float4(0.f, 0.f, 0.f, 0.f);
      *reinterpret_cast<float4*>(sB + (c * TN + r) * 4) = v;
    }
    // generic-proxy shared stores -> visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int j = 0; j < TK / 8; j++) {
        // K = 8 slice j: chunks 2j, 2j+1; LBO = one chunk plane, SBO = 8 rows x 16 bytes
        const uint64_t da = smem_desc(aBase + (uint32_t)(2 * j * TM * 16), TM * 16, 128);
        const uint64_t db = smem_desc(bBase + (uint32_t)(2 * j * TN * 16), TN * 16, 128);
        const uint32_t accum = j > 0 ? 1u : 0u;  // each slice starts from zero
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(kIdesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&bar)) : "memory");
    }
    // the MMAs have read this slice and written TMEM once the barrier completes its phase
    const bool done = mbar_wait(&bar, phase, err);
    phase ^= 1;
    if (__syncthreads_or(!done)) {  // a wait that ran out ends the block, uniformly
      ok = false;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    // warp w reads TMEM lanes 32w..32w+31 (rows m0 + 32w + lane), all TN columns
#pragma unroll
    for (int c0 = 0; c0 < TN; c0 += 8) {
      uint32_t v[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int u = 0; u < 8; u++) acc[c0 + u] += (double)__uint_as_float(v[u]);
    }
    // the next slice's MMAs overwrite TMEM and its staging overwrites shared memory
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  }
  if (ok) {
    const int row = m0 + warp * 32 + lane;
    if (row < M)
#pragma unroll
      for (int c = 0; c < TN; c++)
        if (n0 + c < N) C[(size_t)row * N + n0 + c] = acc[c];
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// C[k][col] (col = (comp * ntri + e) * 2 + re/im) -> FP32 planes H [ntri][nk], D [3][ntri][nk];
// diagonal imaginary parts are zero (Wannier.h:489-492)
__global__ void k_scatter(const double* __restrict__ C, int nk, int n, int ntri, int ncols, float2* __restrict__ H,
                          float2* __restrict__ D) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int ce = blockIdx.y;  // comp * ntri + e
  if (k >= nk) return;
  const int comp = ce / ntri, e = ce - comp * ntri;
  float2 v = make_float2((float)C[(size_t)k * ncols + 2 * ce], (float)C[(size_t)k * ncols + 2 * ce + 1]);
  bool diag = false;
  for (int i = 0; i < n; i++) diag = diag || (e == i * n - (i * (i - 1)) / 2);
  if (diag) v.y = 0.f;
  if (comp == 0)
    H[(size_t)e * nk + k] = v;
  else
    D[((size_t)(comp - 1) * ntri + e) * nk + k] = v;
}

// FP64 band energies: Re sum_r e^{2 pi i k.R_r} H_ii(R_r), and the FP64 matrix the
// eigensolve uses: the tensor-core off-diagonal (as stored, FP32), diagonal from here.
__global__ void k_diag64(const double* __restrict__ kpt, const double* __restrict__ Rvec, const double2* __restrict__ hdiagR,
                         const float2* __restrict__ H32, int nk, int n, int nr, double* __restrict__ Hdiag,
                         double2* __restrict__ Hused) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (k >= nk) return;
  double acc = 0.;
  for (int r = 0; r < nr; r++) {
    const double kR = kpt[k * 3 + 0] * Rvec[r * 3 + 0] + kpt[k * 3 + 1] * Rvec[r * 3 + 1] + kpt[k * 3 + 2] * Rvec[r * 3 + 2];
    double s, c;
    sincospi(2.0 * kR, &s, &c);
    const double2 h = hdiagR[(size_t)i * nr + r];
    acc += c * h.x - s * h.y;
  }
  Hdiag[(size_t)i * nk + k] = acc;
  for (int j = i; j < n; j++) {
    const int e = i * n - (i * (i - 1)) / 2 + (j - i);
    Hused[(size_t)e * nk + k] = (j == i) ? make_double2(acc, 0.) : make_double2(H32[(size_t)e * nk + k].x, H32[(size_t)e * nk + k].y);
  }
}

}  // namespace

size_t tc_gemm_smem() { return sizeof(float) * (TM + TN) * TK + 1024; }

int tc_seg_k(int nr) { return ((2 * nr + TK - 1) / TK) * TK; }
int tc_pad_k(int nr) { return kTcPairs * tc_seg_k(nr); }

cudaError_t tc_contract(const TcArgs& a, cudaStream_t s) {
  const int kpad = tc_pad_k(a.nr);
  const int ncols = 8 * a.ntri;
  k_phase_split<<<a.nk, 256, 0, s>>>(a.kpt, a.Rvec, a.nk, a.nr, tc_seg_k(a.nr), kpad, a.Aw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // about 55 KB of shared memory per CTA keeps at most four CTAs, 512 TMEM columns, per SM
  const size_t smem = std::max(tc_gemm_smem(), (size_t)56 * 1024);
  if ((e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
  dim3 grid((a.nk + TM - 1) / TM, (ncols + TN - 1) / TN);
  k_tc_gemm<<<grid, kThreads, smem, s>>>(a.Aw, a.Bw, a.Cw, a.nk, ncols, kpad, a.err);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_scatter<<<dim3((a.nk + 255) / 256, 4 * a.ntri), 256, 0, s>>>(a.Cw, a.nk, a.n, a.ntri, ncols, a.H32, a.D32);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_diag64<<<dim3((a.nk + 127) / 128, a.n), 128, 0, s>>>(a.kpt, a.Rvec, a.hdiagR, a.H32, a.nk, a.n, a.nr, a.Hdiag, a.Hused);
  return cudaGetLastError();
}

}  // namespace batch
}  // namespace edus
