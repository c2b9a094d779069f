// dev.cuh — device-side types shared by the FP64 kernels and their launchers.
//
// Device layout (all resident in HBM for the whole solve):
//   state planes    rho[e][k], e over the upper triangle i <= j of the n x n
//                   density matrix in the reference's P[k][i][j] convention
//                   (lower triangle = conj, exact because every update the
//                   reference applies preserves Hermiticity bit for bit).
//   H, GE           Hermitian -> upper triangle planes.
//   D               symmetric (save_HUD.cpp:47-51, TB dipoles) -> upper planes.
//   U               full n x n planes (only for dissipation / populations).
//   nbr             [b][k] neighbour table of the k-gradient stencil.
// Planes are [element][k] so one thread per k reads coalesced 16-byte words.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace edus {

// ------------------------------------------------------------- complex helpers
__host__ __device__ __forceinline__ double2 cz() { return make_double2(0., 0.); }
__host__ __device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// -i * a
__host__ __device__ __forceinline__ double2 cmi(double2 a) { return make_double2(a.y, -a.x); }

__host__ __device__ __forceinline__ int tri_index(int i, int j, int n) {
  // i <= j, row-major upper triangle
  return i * n - (i * (i - 1)) / 2 + (j - i);
}

// ------------------------------------------------------------- async bulk copies
// 1-D TMA bulk copies global -> shared completing on an mbarrier. Addresses
// and sizes must be multiples of 16 bytes. Waits are bounded: a wait that runs
// out records kErrTimeout in *err and returns false instead of spinning on.
constexpr int kErrTimeout = 1;
constexpr int kBulkWaitIters = 1 << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t phase, int* err, int iters = kBulkWaitIters) {
  for (int it = 0; it < iters; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (done) return true;
  }
  if (err) atomicExch(err, kErrTimeout);
  return false;
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may start as the previous kernel in the
// stream retires. pdl_wait() returns once that kernel has completed and its
// writes are visible; kernels do independent set-up (trig tables into shared
// memory) before it and touch nothing the previous kernel writes until after
// it. No kernel triggers its dependents early: measured on the 120 x 120
// Coulomb step, an early trigger let waiting blocks of the next kernel occupy
// SM slots and cost 16 %, the implicit trigger at retirement gains 4 %. Both
// calls are no-ops for a normal launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Launch with programmatic stream serialization (PDL).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr int kMaxBands = 16;
constexpr int kMaxTri = kMaxBands * (kMaxBands + 1) / 2;
constexpr int kMaxNb = 64;
constexpr int kMaxOrder = 8;
constexpr int kMaxNcut = 64;

// Static problem tables on the device.
struct DevTables {
  int n, ntri, nk, nnb, n1, n2, nch, nbands;
  const double2* H;    // [ntri][nk]
  const double2* D;    // [3][ntri][nk]
  const double2* U;    // [n*n][nk] or null
  const double2* GE;   // [3][ntri][nk] or null
  const int* nbr;      // [nnb][nk]
  int n_diss;
  // 1: D is Hermitian (the Crystal interface keeps its Berry connections as
  // read, headers/Crystal_interface.h:266-268): D_ji = conj(D_ij). 0: D is
  // symmetric (the reference's 1/2 (D + D^T) of Wannier and tight-binding
  // models, Source_Main/save_HUD.cpp:47-51): D_ji = D_ij. Only the upper
  // triangle is stored either way.
  int herm_dip;
  // Coulomb (null when off)
  int ncut;
  const double2* h;      // [n1][2][ncut][ntri] inverse-transform rows
  const double* t2c;     // [ncut][n2] cos(2 pi n k2)
  const double* t2s;     // [ncut][n2] sin(2 pi n k2)
  const double2* fdiag;  // [n] f_cc(0,0) diagonal (Hartree input)
  const double2* PW0;    // [ntri][nk] initial state (screen correction)
  const double* ncond;   // device scalar: Coulomb_set.n_cond
  int* err;              // device error word (kErrTimeout from bounded waits)
};

// Per-problem constants small enough for a kernel parameter block.
struct DevConsts {
  double wb[kMaxNb];          // weight of the shell of each b
  double bvec[kMaxNb][3];     // Cartesian b
  double T[kMaxBands * kMaxBands];
  int diss_i[kMaxBands * kMaxBands], diss_j[kMaxBands * kMaxBands];
  double VH[kMaxBands * kMaxBands];
  double EH0[kMaxBands];
  double2 screen[kMaxTri];    // conj(Screen_const) per upper element (diag uses [0])
  double2 screen_d00;         // diagonal basis: Screen_const[0][0]
  double2 screen_d01c;        // diagonal basis: conj(Screen_const[0][1])
};

enum StageOp : int {
  OP_PV = 0,       // dst = Pv
  OP_RK_FIRST = 1, // acc = base + c1 Pv ; dst = base + c2 Pv
  OP_RK_MID = 2,   // acc += c1 Pv       ; dst = base + c2 Pv
  OP_RK_LAST = 3,  // dst = acc + c1 Pv
  OP_AB = 4,       // ring[slot0] = Pv ; dst = src + dt * sum coef[s] ring[idx[s]]
  OP_TAYLOR = 5,   // ring[slot0] = Pv ; dst = src + Taylor increment
};

struct DynStep;

// Everything one fused RHS + update launch needs that changes per stage.
struct StageArgs {
  const double2* src;   // state the RHS is evaluated on
  double2* dst;
  const double2* base;  // P0 for the RK stage updates
  double2* acc;         // P1 accumulator
  double2* ring;        // [order][ntri][nk]
  double2* hr_out;      // Hk_renorm output [ntri][nk] (Coulomb) or null
  double EF[2][3];
  double wx2;
  int e_non0;
  int op;
  double c1, c2;
  int order;            // AB / Taylor order
  int ring_idx[kMaxOrder];
  double coef[kMaxOrder];     // AB coefficients
  double tinv[kMaxOrder * kMaxOrder];  // Taylor tau^-1 (scaled)
  double tpow[kMaxOrder];     // pow(dt, i+1)
  double dt;
  // adaptive dt: max over k of the population change, written as uint64 bits
  unsigned long long* maxdp;
  double pcond_plus_ncond;  // P_cond_max + n_cond
  int stage_rows;           // set by the launcher: k-grid rows of Coulomb tables staged per block
  // Coulomb in the diagonal basis: the mean-field term already rotated back to
  // the Wannier basis, [ntri][nk] (null: the Wannier-basis term from tb.h)
  const double2* xw;
  // adaptive step on the device: when set, the stage's field (dyn->EF[dyn_field]),
  // coefficients (dyn->c[dyn_stage]), dt, Taylor tables, e_non0 and
  // P_cond_max + n_cond come from *dyn, and the launch does nothing once the
  // run has ended (dyn->active == 0)
  const DynStep* dyn;
  int dyn_stage, dyn_field;
};

}  // namespace edus
