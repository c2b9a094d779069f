// tc_contract.cu — the Wannier Fourier sums H(k), D(k) on the tcgen05 tensor
// cores (kind::f16 with exact BF16 integer slices) for mixed-precision batch
// instances.
//
// Real form of the complex sums: with A[k][.] = [cos(2 pi k.R_r) | sin(2 pi k.R_r)] / 2
// (K = 2 nr) and, per output element, the column pair
//   re: [ Re c_r ; -Im c_r ],   im: [ Im c_r ; Re c_r ]  (times 2),
// out = A . B^T gives Re / Im of sum_r e^{2 pi i k.R_r} c_r. Both operands are
// cut into 8-bit slices on a power-of-two scale (tc_contract.hpp): the GEMM
// depth holds one segment of 2 nr (padded to 64) per slice pair (a, b) with
// a + b <= 3. Within a segment every product is an integer times a common
// power of two and at most 2^14, so the tensor core's FP32 sums over a segment
// (at most 1024 deep) are exact; the segments are added in FP64 registers. The
// result is the FP64 sum to about 2^-32 of the terms, so the FP32 tables stored
// from it equal those of the FP64 CUDA-core build up to the last rounding.
//
// Three forms of the GEMM give the same sums bit for bit. k_tc_gemm_ws (the
// default) and k_tc_gemm_tma (EDUS_TC_GEMM=tma) move 128 x 64 and 64 x 64
// operand tiles by TMA into 128-byte swizzled stages, four deep, with the
// loads, MMAs and read-back on separate warps or all issued by thread 0
// (below). k_tc_gemm (EDUS_TC_GEMM=cpasync): one
// CTA (4 warps) per 128 x 32 tile of C. The 64-deep K slices
// (128-byte rows of BF16) are staged with cp.async into two shared-memory
// stages in the K-major canonical layout without swizzle (16-byte chunks of 8
// BF16, 8-row core matrices 128 bytes apart, the two 16-byte halves of one
// MMA's K = 16 one whole operand apart): slice s + 1 loads while the tensor
// core works on slice s. One elected thread issues four tcgen05.mma (M 128,
// N 32, K 16) per slice and commits them to the stage's mbarrier. Segments
// alternate between two TMEM accumulators (128 lanes x 32 FP32 columns each);
// a finished segment is read back with tcgen05.ld.32x32b into FP64 registers
// while the next one accumulates. All waits are bounded.
#include <cuda.h>
#include <stdint.h>

#include <cstdlib>
#include <cstring>

#include "batch.cuh"
#include "dev.cuh"
#include "tc_contract.hpp"

namespace edus {
namespace batch {
namespace {

constexpr int TM = 128, TN = 32, TK = 64;  // CTA tile and K slice (BF16 elements: 128-byte rows)
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 32;

// A' rows: phases of k point m over the R vectors; segment p holds slice
// tc_pair_a(p) of [cos | sin], zero padded to the segment length. One phase
// is evaluated once and written to every segment.
__global__ void k_phase_split(const double* __restrict__ kpt, const double* __restrict__ Rvec, int nk, int nr, int kseg,
                              int kpad, uint16_t* __restrict__ A) {
  const int m = blockIdx.x;
  const int K = 2 * nr;
  uint16_t* row = A + (size_t)m * kpad;
  for (int q = threadIdx.x; q < kseg; q += blockDim.x) {
    uint16_t sl[kTcSlices] = {0, 0, 0, 0};
    if (m < nk && q < K) {
      const int r = q < nr ? q : q - nr;
      const double kR = kpt[m * 3 + 0] * Rvec[r * 3 + 0] + kpt[m * 3 + 1] * Rvec[r * 3 + 1] + kpt[m * 3 + 2] * Rvec[r * 3 + 2];
      double sn, co;
      sincospi(2.0 * kR, &sn, &co);
      const double y = 0.5 * (q < nr ? co : sn);  // in [-1/2, 1/2]: every slice at most 128 in magnitude
#pragma unroll
      for (int t = 0; t < kTcSlices; t++) sl[t] = tc_bf16(tc_slice(y, t));  // at most 8 significant bits: exact in BF16
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
// kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9 and 10-12 = 1), K-major, M = 128, N = 32
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

// C (FP64) = A' B'^T. Each K segment (one slice pair) accumulates in FP32 in
// one of two TMEM regions, exactly (every product is an integer times the
// segment's power of two, at most 2^14, and a segment is at most 1024 deep);
// the segment is read back into FP64 registers while the next segment's MMAs
// run in the other region. The 32-deep K slices are staged with cp.async into
// two shared-memory stages: slice s + 1 loads while the tensor core works on
// slice s. Every wait is bounded; a wait that runs out ends the block
// uniformly after its own copies and MMAs have drained.
__device__ __forceinline__ void tc_cp16(uint32_t dst, const void* src, bool pred) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(pred ? 16 : 0) : "memory");
}

__global__ void __launch_bounds__(kThreads, 1) k_tc_gemm(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B, double* __restrict__ C,
                                                         int M, int N, int Kp, int kseg, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr uint32_t kStageA = TM * TK * 2, kStageB = TN * TK * 2, kStage = kStageA + kStageB;
  __shared__ unsigned long long bar[2];  // MMAs of the slices staged in stage 0 / 1 have completed
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(2 * kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t base = smem_u32(smem);
  const int S = Kp / TK, SEG = kseg / TK;
  double acc[TN];
#pragma unroll
  for (int c = 0; c < TN; c++) acc[c] = 0.;

  // slice s -> stage b: row r, 16-byte chunk c at (c * rows + r) * 16 (K-major core matrices)
  auto load = [&](int s, int b) {
    const int k0 = s * TK;
    const uint32_t sa = base + (uint32_t)b * kStage, sb = sa + kStageA;
    for (int q = tid; q < TM * (TK / 8); q += kThreads) {
      const int r = q % TM, c = q / TM;
      const bool in = m0 + r < M;
      tc_cp16(sa + (uint32_t)((c * TM + r) * 16), in ? (const void*)(A + (size_t)(m0 + r) * Kp + k0 + 8 * c) : (const void*)A, in);
    }
    for (int q = tid; q < TN * (TK / 8); q += kThreads) {
      const int r = q % TN, c = q / TN;
      const bool in = n0 + r < N;
      tc_cp16(sb + (uint32_t)((c * TN + r) * 16), in ? (const void*)(B + (size_t)(n0 + r) * Kp + k0 + 8 * c) : (const void*)B, in);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // segment p's accumulator (TMEM region p & 1) into FP64 registers: warp w reads
  // lanes 32w..32w+31 (rows m0 + 32w + lane), all TN columns
  auto readout = [&](int p) {
    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
    for (int c0 = 0; c0 < TN; c0 += 8) {
      uint32_t v[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((p & 1) * kTmemCols + c0);
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int u = 0; u < 8; u++) acc[c0 + u] += (double)__uint_as_float(v[u]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
  };
  // the MMAs of slice s have completed (commit number s >> 1 on bar[s & 1])
  auto mma_done = [&](int s) { return mbar_wait(&bar[s & 1], (uint32_t)((s >> 1) & 1), err); };

  bool ok = true;
  int issued = -1;  // last slice whose MMAs were committed
  load(0, 0);
  for (int s = 0; s < S; s++) {
    const int b = s & 1;
    if (s + 1 < S) {
      // stage b ^ 1 was last read by the MMAs of slice s - 1
      if (s >= 1) ok = mma_done(s - 1) && ok;
      if (__syncthreads_or(!ok)) break;
      load(s + 1, b ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    // this thread's copies of slice s are in; make every thread's visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t sa = base + (uint32_t)b * kStage, sb = sa + kStageA;
      const uint32_t dtm = tmem + (uint32_t)(((s / SEG) & 1) * kTmemCols);
#pragma unroll
      for (int j = 0; j < TK / 16; j++) {
        // K = 16 slice j: chunks 2j, 2j+1; LBO = one chunk plane, SBO = 8 rows x 16 bytes
        const uint64_t da = smem_desc(sa + (uint32_t)(2 * j * TM * 16), TM * 16, 128);
        const uint64_t db = smem_desc(sb + (uint32_t)(2 * j * TN * 16), TN * 16, 128);
        const uint32_t accum = (j > 0 || s % SEG != 0) ? 1u : 0u;  // each segment starts from zero
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtm),
            "l"(da), "l"(db), "r"(kIdesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&bar[b])) : "memory");
    }
    issued = s;
    // the previous segment is complete once slice s - 1's MMAs are: read it back while
    // this segment's MMAs run in the other region
    // (the readout is warp-collective: the block decides on the wait together)
    if (s > 0 && s % SEG == 0) {
      const bool d = mma_done(s - 1);
      if (__syncthreads_or(!d)) {
        ok = false;
        break;
      }
      readout((s - 1) / SEG);
    }
  }
  if (__syncthreads_or(!ok)) ok = false;
  if (ok && issued == S - 1) {
    const bool d = mma_done(S - 1);
    if (__syncthreads_or(!d)) ok = false;
    else readout((S - 1) / SEG);
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (!__syncthreads_or(!ok)) {
    const int row = m0 + warp * 32 + lane;
    if (row < M)
#pragma unroll
      for (int c = 0; c < TN; c++)
        if (n0 + c < N) C[(size_t)row * N + n0 + c] = acc[c];
  } else if (issued >= 0) {
    // drain: the last committed MMAs must finish before their TMEM is released (bounded)
    mma_done(issued);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTmemCols));
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

// ------------------------------------------------------------------ TMA-staged GEMM
// The same exact-slice GEMM with its operand tiles moved by TMA
// (cp.async.bulk.tensor.2d, no multicast; both tensor maps cover this GPU's
// own buffers) in the 128-byte swizzled K-major layout: one box of 64 BF16
// (128 bytes) x 128 rows of A' and one of 64 x 64 rows of B' per 64-deep K
// slice, each landing as 8-row x 128-byte swizzle atoms 1024 bytes apart; the
// MMA descriptors address K step j of the slice at +32 j bytes inside the
// atom. N tile 64, four shared-memory stages; thread 0 issues the MMAs of
// slice s, then the loads of slice s + 3 once slice s - 1's MMAs have freed
// their stage, so three slices are in flight while the tensor core works.
// Every wait is bounded; on a timeout the block waits (bounded) for its issued
// loads and MMAs, releases TMEM and ends.
constexpr int TN2 = 64, kStages2 = 4;
constexpr uint32_t kTmemCols2 = 64;
constexpr uint32_t kIdesc2 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN2 >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
               "l"(map), "r"(x), "r"(y), "r"(bar)
               : "memory");
}

// K-major operand in 128-byte swizzle atoms (8 rows x 128 bytes, 1024-byte
// aligned, atoms 1024 bytes apart along M / N): stride byte offset 1024, the
// leading offset unused (encoded 1), layout type 2 (128-byte swizzle)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  d |= (uint64_t)2 << 61;  // 128-byte swizzle
  return d;
}

__global__ void __launch_bounds__(kThreads, 1) k_tc_gemm_tma(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                                                             double* __restrict__ C, int M, int N, int Kp, int kseg, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr uint32_t kStageA = TM * TK * 2, kStageB = TN2 * TK * 2, kStage = kStageA + kStageB;
  __shared__ unsigned long long full[kStages2], mmab[kStages2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN2;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(2 * kTmemCols2));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int b = 0; b < kStages2; b++) {
      mbar_init(&full[b], 1);
      mbar_init(&mmab[b], 1);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t base = (smem_u32(smem) + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
  const int S = Kp / TK, SEG = kseg / TK;
  double acc[TN2];
#pragma unroll
  for (int c = 0; c < TN2; c++) acc[c] = 0.;

  // slice s into stage b: one 64 x 128 box of A', one 64 x 64 box of B' (rows past M, N read as zero)
  auto issue_load = [&](int s, int b) {
    const uint32_t sa = base + (uint32_t)b * kStage, sb = sa + kStageA;
    mbar_expect_tx(&full[b], kStage);
    tma_load_2d(sa, &mapA, s * TK, m0, smem_u32(&full[b]));
    tma_load_2d(sb, &mapB, s * TK, n0, smem_u32(&full[b]));
  };
  auto readout = [&](int p) {
    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
    for (int c0 = 0; c0 < TN2; c0 += 8) {
      uint32_t v[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((p & 1) * kTmemCols2 + c0);
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int u = 0; u < 8; u++) acc[c0 + u] += (double)__uint_as_float(v[u]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
  };
  // completion number (s / kStages2) of a stage's barrier belongs to slice s
  auto mma_done = [&](int s) { return mbar_wait(&mmab[s % kStages2], (uint32_t)((s / kStages2) & 1), err); };
  auto loaded = [&](int s) { return mbar_wait(&full[s % kStages2], (uint32_t)((s / kStages2) & 1), err); };

  bool ok = true;
  int issued = -1, loads = 0;  // last slice whose MMAs were committed; slices whose loads were issued
  if (tid == 0)
    for (; loads < kStages2 - 1 && loads < S; loads++) issue_load(loads, loads);
  for (int s = 0; s < S; s++) {
    if (tid == 0) {
      if (ok) ok = loaded(s);
      if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t sa = base + (uint32_t)(s % kStages2) * kStage, sb = sa + kStageA;
        const uint32_t dtm = tmem + (uint32_t)(((s / SEG) & 1) * kTmemCols2);
#pragma unroll
        for (int j = 0; j < TK / 16; j++) {
          // K step j: 16 BF16 = 32 bytes into every 128-byte swizzled row
          const uint64_t da = sw128_desc(sa + (uint32_t)(32 * j));
          const uint64_t db = sw128_desc(sb + (uint32_t)(32 * j));
          const uint32_t accum = (j > 0 || s % SEG != 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtm),
              "l"(da), "l"(db), "r"(kIdesc2), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mmab[s % kStages2]))
                     : "memory");
        issued = s;
      }
      // refill: slice s + 3 goes to the stage slice s - 1 used, once its MMAs are done
      // (slice s's MMAs are queued behind them meanwhile)
      if (ok && loads < S) {
        if (loads >= kStages2) ok = mma_done(loads - kStages2);
        if (ok) {
          issue_load(loads, loads % kStages2);
          loads++;
        }
      }
    }
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    // the previous segment is complete with slice s - 1: read it while this one accumulates
    if (s > 0 && s % SEG == 0) {
      const bool d = mma_done(s - 1);
      if (__syncthreads_or(!d)) {
        ok = false;
        break;
      }
      readout((s - 1) / SEG);
    }
  }
  if (__syncthreads_or(!ok)) ok = false;
  if (ok) {
    const bool d = mma_done(S - 1);
    if (__syncthreads_or(!d)) ok = false;
    else readout((S - 1) / SEG);
  }
  if (!__syncthreads_or(!ok)) {
    const int row = m0 + warp * 32 + lane;
    if (row < M)
#pragma unroll
      for (int c = 0; c < TN2; c++)
        if (n0 + c < N) C[(size_t)row * N + n0 + c] = acc[c];
  } else if (tid == 0) {
    // drain (bounded): issued loads land and committed MMAs finish before the stages and TMEM go away
    for (int s = issued + 1; s < loads; s++) loaded(s);
    if (issued >= 0) mma_done(issued);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTmemCols2));
}

// ------------------------------------------------------- warp-specialised form
// The TMA-staged GEMM with its roles on separate warps, so that loads, MMAs and
// the FP64 read-back of finished segments overlap instead of taking turns on
// thread 0 between block barriers: warp 4 (one lane) issues the TMA loads of
// slice s into stage s % 4 once the MMAs of slice s - 4 have released it;
// warp 5 (one lane) issues the MMAs of slice s once its stage is full, into
// the TMEM accumulator of its segment's parity, after the read-back of the
// segment two back has freed that accumulator, and commits them to the
// stage's "empty" barrier and, at a segment's end, to the accumulator's
// "full" barrier; warps 0-3 read each finished segment (32 TMEM lanes each)
// into FP64 registers and arrive on the accumulator's "free" barrier. The
// sums are those of the other forms, in the same order. Every wait is bounded;
// a role that times out raises a shared abort flag and stops, the others stop
// at their next wait, and before TMEM and shared memory are released the
// producer waits (bounded) for its last loads and the MMA lane for its last
// commit.
constexpr int kWsThreads = 192;

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(kWsThreads, 2) k_tc_gemm_ws(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                                                              double* __restrict__ C, int M, int N, int Kp, int kseg, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr uint32_t kStageA = TM * TK * 2, kStageB = TN2 * TK * 2, kStage = kStageA + kStageB;
  __shared__ unsigned long long full[kStages2], empty[kStages2], accf[2], acce[2];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, loads_issued, last_commit;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN2;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(2 * kTmemCols2));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 32) {
    for (int b = 0; b < kStages2; b++) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);  // one arrival per read-back warp
    }
    abort_flag = 0;
    loads_issued = 0;
    last_commit = -1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t base = (smem_u32(smem) + 1023u) & ~1023u;
  const int S = Kp / TK, SEG = kseg / TK, P = S / SEG;
  volatile int* abortp = &abort_flag;
  double acc[TN2];
#pragma unroll
  for (int c = 0; c < TN2; c++) acc[c] = 0.;

  if (warp == 4) {
    if (lane == 0) {
      int s = 0;
      for (; s < S; s++) {
        const int st = s % kStages2;
        if (*abortp) break;
        if (s >= kStages2 && !mbar_wait(&empty[st], (uint32_t)(((s / kStages2) - 1) & 1), err)) {
          *abortp = 1;
          break;
        }
        const uint32_t sa = base + (uint32_t)st * kStage, sb = sa + kStageA;
        mbar_expect_tx(&full[st], kStage);
        tma_load_2d(sa, &mapA, s * TK, m0, smem_u32(&full[st]));
        tma_load_2d(sb, &mapB, s * TK, n0, smem_u32(&full[st]));
      }
      loads_issued = s;
    }
  } else if (warp == 5) {
    if (lane == 0) {
      int last = -1;
      for (int s = 0; s < S; s++) {
        const int st = s % kStages2, p = s / SEG, buf = p & 1;
        if (*abortp) break;
        if (!mbar_wait(&full[st], (uint32_t)((s / kStages2) & 1), err)) {
          *abortp = 1;
          break;
        }
        // a segment's first slice reuses the accumulator of the segment two back: wait for its read-back
        if (s % SEG == 0 && p >= 2 && !mbar_wait(&acce[buf], (uint32_t)(((p / 2) - 1) & 1), err)) {
          *abortp = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t sa = base + (uint32_t)st * kStage, sb = sa + kStageA;
        const uint32_t dtm = tmem + (uint32_t)(buf * kTmemCols2);
#pragma unroll
        for (int j = 0; j < TK / 16; j++) {
          const uint64_t da = sw128_desc(sa + (uint32_t)(32 * j));
          const uint64_t db = sw128_desc(sb + (uint32_t)(32 * j));
          const uint32_t accum = (j > 0 || s % SEG != 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtm),
              "l"(da), "l"(db), "r"(kIdesc2), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&empty[st]))
                     : "memory");
        if (s % SEG == SEG - 1)
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&accf[buf]))
                       : "memory");
        last = s;
      }
      last_commit = last;
    }
  } else {
    // read-back warps: TMEM lanes 32 warp .. 32 warp + 31 are rows m0 + 32 warp + lane
    for (int p = 0; p < P; p++) {
      const int buf = p & 1;
      const bool ok = !*abortp && mbar_wait(&accf[buf], (uint32_t)((p / 2) & 1), err);
      if (__any_sync(0xffffffffu, !ok)) {
        if (lane == 0) *abortp = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int c0 = 0; c0 < TN2; c0 += 8) {
        uint32_t v[8];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * kTmemCols2 + c0);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                     : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int u = 0; u < 8; u++) acc[c0 + u] += (double)__uint_as_float(v[u]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[buf]);
    }
  }
  __syncthreads();
  if (!*abortp) {
    if (warp < 4) {
      const int row = m0 + warp * 32 + lane;
      if (row < M)
#pragma unroll
        for (int c = 0; c < TN2; c++)
          if (n0 + c < N) C[(size_t)row * N + n0 + c] = acc[c];
    }
  } else if (tid == 128) {
    // the last loads issued (one per stage at most is outstanding) land before the stages go away
    for (int s = loads_issued - kStages2 < 0 ? 0 : loads_issued - kStages2; s < loads_issued; s++)
      mbar_wait(&full[s % kStages2], (uint32_t)((s / kStages2) & 1), err);
  } else if (tid == 160 && last_commit >= 0) {
    // the last committed MMAs finish before their TMEM is released
    mbar_wait(&empty[last_commit % kStages2], (uint32_t)((last_commit / kStages2) & 1), err);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTmemCols2));
}

// Velocity gauge: coefficient slices of c_A(R) = e^{2 pi i A.R} c(R), one thread per
// (column, K entry); column 2 ce + part holds [Re c_A ; -Im c_A] (part 0) or
// [Im c_A ; Re c_A] (part 1), pre-multiplied by 2 scale as the host build's slices
__global__ void k_vg_bslices(const double2* __restrict__ coef, const double* __restrict__ Rvec, const double* __restrict__ colscale,
                             double A0, double A1, double A2, int ntri, int nr, int kseg, int kpad, uint16_t* __restrict__ B) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;  // K entry
  const int col = blockIdx.y;                          // 2 (comp * ntri + e) + part
  const int K = 2 * nr;
  if (q >= K) return;
  const int ce = col / 2, part = col % 2;
  const int r = q < nr ? q : q - nr;
  const double* R = Rvec + (size_t)r * 3;
  double s, c;
  sincospi(2.0 * (A0 * R[0] + A1 * R[1] + A2 * R[2]), &s, &c);
  const double2 cf = coef[(size_t)ce * nr + r];
  const double re = c * cf.x - s * cf.y, im = c * cf.y + s * cf.x;
  const double v = part == 0 ? (q < nr ? re : -im) : (q < nr ? im : re);
  const double scale = colscale[col];
  uint16_t* row = B + (size_t)col * kpad;
#pragma unroll
  for (int p = 0; p < kTcPairs; p++) row[(size_t)p * kseg + q] = tc_bf16(2.0 * scale * tc_slice(v / scale, tc_pair_b(p)));
}

// C[k][col] -> FP64 planes H [ntri][nk], D [3][ntri][nk]; diagonal imaginary parts zero
__global__ void k_scatter64(const double* __restrict__ C, int nk, int n, int ntri, int ncols, double2* __restrict__ H,
                            double2* __restrict__ D) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int ce = blockIdx.y;
  if (k >= nk) return;
  const int comp = ce / ntri, e = ce - comp * ntri;
  double2 v = make_double2(C[(size_t)k * ncols + 2 * ce], C[(size_t)k * ncols + 2 * ce + 1]);
  bool diag = false;
  for (int i = 0; i < n; i++) diag = diag || (e == i * n - (i * (i - 1)) / 2);
  if (diag) v.y = 0.;
  if (comp == 0)
    H[(size_t)e * nk + k] = v;
  else
    D[((size_t)(comp - 1) * ntri + e) * nk + k] = v;
}

}  // namespace

size_t tc_gemm_smem() { return 2 * sizeof(uint16_t) * (TM + TN) * TK + 1024; }

int tc_seg_k(int nr) { return ((2 * nr + TK - 1) / TK) * TK; }
int tc_pad_k(int nr) { return kTcPairs * tc_seg_k(nr); }

cudaError_t tc_gemm_run(const uint16_t* Aw, const uint16_t* Bw, double* Cw, int M, int ncols, int kpad, int kseg, int* err,
                        const CUtensorMap* mapA, const CUtensorMap* mapB, cudaStream_t s);
bool tc_gemm_tma_wanted();
cudaError_t tc_gemm_maps(const uint16_t* Aw, const uint16_t* Bw, int M, int ncols, int kpad, CUtensorMap* mapA, CUtensorMap* mapB);

cudaError_t tc_contract(const TcArgs& a, cudaStream_t s) {
  const int kpad = tc_pad_k(a.nr);
  const int ncols = 8 * a.ntri;
  k_phase_split<<<a.nk, 256, 0, s>>>(a.kpt, a.Rvec, a.nk, a.nr, tc_seg_k(a.nr), kpad, a.Aw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  CUtensorMap mA, mB;
  const bool tma = tc_gemm_tma_wanted() && tc_gemm_maps(a.Aw, a.Bw, a.nk, ncols, kpad, &mA, &mB) == cudaSuccess;
  if ((e = tc_gemm_run(a.Aw, a.Bw, a.Cw, a.nk, ncols, kpad, tc_seg_k(a.nr), a.err, tma ? &mA : nullptr, tma ? &mB : nullptr, s)) !=
      cudaSuccess)
    return e;
  k_scatter<<<dim3((a.nk + 255) / 256, 4 * a.ntri), 256, 0, s>>>(a.Cw, a.nk, a.n, a.ntri, ncols, a.H32, a.D32);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_diag64<<<dim3((a.nk + 127) / 128, a.n), 128, 0, s>>>(a.kpt, a.Rvec, a.hdiagR, a.H32, a.nk, a.n, a.nr, a.Hdiag, a.Hused);
  return cudaGetLastError();
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                   const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// rows x Kp BF16 operand (K contiguous; Kp a multiple of 64), boxes of 64 x
// box_rows in 128-byte swizzle atoms; out-of-range rows read as zero
cudaError_t encode_operand(CUtensorMap* map, const uint16_t* ptr, int rows, int Kp, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * sizeof(uint16_t)};
  const cuuint32_t box[2] = {(cuuint32_t)TK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

size_t tma_gemm_smem() { return (size_t)kStages2 * (TM + TN2) * TK * 2 + 1024; }

}  // namespace

cudaError_t tc_vg_prepare(const TcVgArgs& a, cudaStream_t s) {
  const int kpad = tc_pad_k(a.nr);
  k_phase_split<<<a.nk, 256, 0, s>>>(a.kpt, a.Rvec, a.nk, a.nr, tc_seg_k(a.nr), kpad, a.Aw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(a.Bw, 0, sizeof(uint16_t) * (size_t)8 * a.ntri * kpad, s)) != cudaSuccess) return e;
  const size_t smem = std::max(tc_gemm_smem(), (size_t)56 * 1024);
  if ((e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_tc_gemm_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_gemm_smem())) != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tc_gemm_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_gemm_smem());
}

// GEMM form: the warp-specialised TMA form by default (76.8 us against 110 us
// for the single-issuer TMA form and 229 us for the cp.async form on the 96 x 96
// 8-band contraction); EDUS_TC_GEMM=tma selects the single-issuer TMA form,
// EDUS_TC_GEMM=cpasync the cp.async form (all three give bit-identical sums:
// every segment's FP32 sums are exact).
int tc_gemm_form() {
  const char* form = std::getenv("EDUS_TC_GEMM");
  if (form && std::strcmp(form, "cpasync") == 0) return 0;
  if (form && std::strcmp(form, "tma") == 0) return 1;
  return 2;
}
bool tc_gemm_tma_wanted() { return tc_gemm_form() != 0; }

cudaError_t tc_gemm_maps(const uint16_t* Aw, const uint16_t* Bw, int M, int ncols, int kpad, CUtensorMap* mapA, CUtensorMap* mapB) {
  cudaError_t e = encode_operand(mapA, Aw, M, kpad, TM);
  if (e == cudaSuccess) e = encode_operand(mapB, Bw, ncols, kpad, TN2);
  return e;
}

// C = A' B'^T over the slice-pair segments: the TMA form with the given tensor maps, else the cp.async form
cudaError_t tc_gemm_run(const uint16_t* Aw, const uint16_t* Bw, double* Cw, int M, int ncols, int kpad, int kseg, int* err,
                        const CUtensorMap* mapA, const CUtensorMap* mapB, cudaStream_t s) {
  cudaError_t e;
  if (mapA && mapB && tc_gemm_form() == 2) {
    if ((e = cudaFuncSetAttribute(k_tc_gemm_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_gemm_smem())) != cudaSuccess)
      return e;
    dim3 grid((M + TM - 1) / TM, (ncols + TN2 - 1) / TN2);
    k_tc_gemm_ws<<<grid, kWsThreads, tma_gemm_smem(), s>>>(*mapA, *mapB, Cw, M, ncols, kpad, kseg, err);
  } else if (mapA && mapB) {
    if ((e = cudaFuncSetAttribute(k_tc_gemm_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_gemm_smem())) != cudaSuccess)
      return e;
    dim3 grid((M + TM - 1) / TM, (ncols + TN2 - 1) / TN2);
    k_tc_gemm_tma<<<grid, kThreads, tma_gemm_smem(), s>>>(*mapA, *mapB, Cw, M, ncols, kpad, kseg, err);
  } else {
    // about 55 KB of shared memory per CTA keeps at most four CTAs (256 of the 512 TMEM columns) per SM
    const size_t smem = std::max(tc_gemm_smem(), (size_t)56 * 1024);
    if ((e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
    dim3 grid((M + TM - 1) / TM, (ncols + TN - 1) / TN);
    k_tc_gemm<<<grid, kThreads, smem, s>>>(Aw, Bw, Cw, M, ncols, kpad, kseg, err);
  }
  return cudaGetLastError();
}

cudaError_t tc_vg_maps(TcVgArgs& a) {
  const cudaError_t e = tc_gemm_maps(a.Aw, a.Bw, a.nk, 8 * a.ntri, tc_pad_k(a.nr), &a.mapA, &a.mapB);
  a.tma = e == cudaSuccess;
  return e;
}

cudaError_t tc_vg_stage(const TcVgArgs& a, cudaStream_t s) {
  const int kpad = tc_pad_k(a.nr), kseg = tc_seg_k(a.nr), ncols = 8 * a.ntri;
  k_vg_bslices<<<dim3((2 * a.nr + 127) / 128, ncols), 128, 0, s>>>(a.coef, a.Rvec, a.colscale, a.A[0], a.A[1], a.A[2], a.ntri,
                                                                   a.nr, kseg, kpad, a.Bw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = tc_gemm_run(a.Aw, a.Bw, a.Cw, a.nk, ncols, kpad, kseg, a.err, a.tma ? &a.mapA : nullptr, a.tma ? &a.mapB : nullptr, s)) !=
      cudaSuccess)
    return e;
  k_scatter64<<<dim3((a.nk + 255) / 256, 4 * a.ntri), 256, 0, s>>>(a.Cw, a.nk, a.n, a.ntri, ncols, a.H, a.D);
  return cudaGetLastError();
}

}  // namespace batch
}  // namespace edus
