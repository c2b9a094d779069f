// batch_kernels.cu — persistent RK4 stage and observable kernels over the tile
// table of a batch (one class of band count N per launch).
//
// Element-parallel like the single-solve kernel: thread (k, e) of a tile owns
// one upper-triangle element e = (i, j) of one k point; the block exchanges
// rho and H~ through shared memory. Blocks are 1-D and padded to whole warps;
// padding threads only take part in barriers.
//
// Precision: FP64 mode reproduces headers/RungeKutta.h:141-294 in double.
// Mixed mode stores H, D, GE, U as FP32 and evaluates H~, the commutator and
// the k-gradient sum in FP32 on the deviation from the initial state
// rho - rho_eq (rho_eq kept in FP64); rho, the RK4 stage arithmetic and all
// observables stay in FP64.
#include <type_traits>

#include "batch.cuh"

namespace edus {
namespace batch {
namespace {

template <int N>
struct TriB {
  static constexpr int NT = N * (N + 1) / 2;
  static __device__ __forceinline__ int idx(int i, int j) { return i * N - (i * (i - 1)) / 2 + (j - i); }
  static __device__ __forceinline__ void ij(int e, int& i, int& j) {
    int r = e;
    i = 0;
    while (r >= N - i) {
      r -= N - i;
      i++;
    }
    j = i + r;
  }
};

constexpr int pad32(int x) { return (x + 31) / 32 * 32; }

// complex arithmetic generic over float2 / double2 (same expressions as dev.cuh)
template <class C>
__device__ __forceinline__ C xmk(decltype(C::x) a, decltype(C::x) b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <class C>
__device__ __forceinline__ C xadd(C a, C b) { return xmk<C>(a.x + b.x, a.y + b.y); }
template <class C>
__device__ __forceinline__ C xsub(C a, C b) { return xmk<C>(a.x - b.x, a.y - b.y); }
template <class C>
__device__ __forceinline__ C xmul(C a, C b) { return xmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <class C>
__device__ __forceinline__ C xscale(C a, decltype(C::x) s) { return xmk<C>(a.x * s, a.y * s); }
template <class C>
__device__ __forceinline__ C xconj(C a) { return xmk<C>(a.x, -a.y); }
template <class C>
__device__ __forceinline__ C xmi(C a) { return xmk<C>(a.y, -a.x); }

template <class To, class From>
__device__ __forceinline__ To cvt(From a) { return xmk<To>((decltype(To::x))a.x, (decltype(To::x))a.y); }

// Commutator sum beta = sum_l H~_jl P_il - conj(H~_il P_jl) as fused
// multiply-adds into eight independent partial sums (products with H~_j and
// with H~_i, real and imaginary parts, even and odd l), so that no dependency
// chain is longer than N multiply-adds; batch_pipe.cu uses the same order.
template <class C>
struct CommAcc {
  using R = decltype(C::x);
  R ax[2] = {0, 0}, ay[2] = {0, 0}, bx[2] = {0, 0}, by[2] = {0, 0};
  __device__ __forceinline__ void add(int par, C hj, C pi, C hi, C pj) {
    ax[par] = fma(hj.x, pi.x, ax[par]);
    ax[par] = fma(-hj.y, pi.y, ax[par]);
    ay[par] = fma(hj.x, pi.y, ay[par]);
    ay[par] = fma(hj.y, pi.x, ay[par]);
    bx[par] = fma(hi.x, pj.x, bx[par]);
    bx[par] = fma(-hi.y, pj.y, bx[par]);
    by[par] = fma(hi.x, pj.y, by[par]);
    by[par] = fma(hi.y, pj.x, by[par]);
  }
  // H~_j.P_i - conj(H~_i.P_j)
  __device__ __forceinline__ C sum() const {
    C r;
    r.x = (ax[0] + ax[1]) - (bx[0] + bx[1]);
    r.y = (ay[0] + ay[1]) + (by[0] + by[1]);
    return r;
  }
};

template <bool MIX>
struct Types {
  using S = double2;  // storage of H, D, GE, U
  using C = double2;  // commutator arithmetic
};
template <>
struct Types<true> {
  using S = float2;
  using C = float2;
};

__device__ __forceinline__ bool field_on(const double* E) {
  double s = 0;
  for (int q = 0; q < 6; q++) s += E[q] * E[q];
  return sqrt(s) > 1e-20;
}

// ------------------------------------------------------------------ RK4 stage
// Stage s of Source_Main/RungeKutta.cpp:20-165 for every active instance:
//   s=0: P1 = P0 + dt/6 k1, Pa = P0 + dt/2 k1     (field at t)
//   s=1: P1 += dt/3 k2,     Pb = P0 + dt/2 k2     (field at t + dt/2)
//   s=2: P1 += dt/3 k3,     Pa = P0 + dt k3       (stage-2 field reused)
//   s=3: P0 = P1 + dt/6 k4                        (field at t + dt)
// Resident blocks per SM the register budget is sized for: register profile 0
// aims at about 36 warps per SM (56 registers), profile 1 at 24 warps (up to
// 80-96 registers, fewer spills). The autotuner picks one per class.
constexpr int min_blocks(int nthr, int occ) {
  const int target = occ == 0 ? 1152 : 768;
  return target / nthr > 0 ? target / nthr : 1;
}

// Shared-memory exchange of one tile: full n x n matrices (the lower triangle
// written as the conjugate / mirrored entry), element (r, c) of k point kl at
// [r * RS + c * KT + kl], so every operand of the commutator is a constant
// offset from a per-thread row pointer. The tile's field, gradient
// coefficients and neighbour indices are written one tile ahead.
// Row r of a shared matrix starts at r * RS(N, KT), RS = KT mod 2 KT: the
// elements (i, j), (i, j + 1), ... that one bank phase of a warp serves (16
// threads of 8-byte entries, 8 threads of 16-byte entries) then read their
// KT-long runs of row j from disjoint banks.
template <int N, int KT>
struct Rows {
  static constexpr int RS = N * KT + ((N % 2) ? 0 : KT);
  static constexpr int SIZE = N * RS;
};

template <int N, int KT, bool MIX>
struct StageSmem {
  using C = typename Types<MIX>::C;
  static constexpr int SZ = Rows<N, KT>::SIZE;
  C P[SZ];                          // FP64: rho; mixed: rho - rho_eq
  C H[SZ];                          // H~ = H + E . D (mixed: off-diagonal part)
  double Ed[MIX ? N * KT : 1];      // mixed: diagonal of H~ in FP64
  double E[2][3];                   // field of the stage: pump, probe / 2
  double G[kBatchMaxNb];            // w_b (E_pump . b) per neighbour
  int nb[kBatchMaxNb][KT];          // k + b of the tile's k points
  int on;                           // k-gradient on (E_non0)
  int active;                       // the tile's instance is inside its time grid
};

// k + b of the k-gradient stencil: from the lattice steps of the stencil
// (every b of a Monkhorst-Pack grid is a fixed step (d1, d2) with periodic
// wrap, verified against the neighbour table at admission), else the table.
__device__ __forceinline__ int neighbour(const Inst* I, int k, int b) {
  if (!I->lattice) return I->nbr[(size_t)b * I->nk + k];
  const int i1 = k / I->n2, i2 = k - i1 * I->n2;
  int j1 = i1 + I->off[b][0], j2 = i2 + I->off[b][1];
  j1 += j1 < 0 ? I->n1 : (j1 >= I->n1 ? -I->n1 : 0);
  j2 += j2 < 0 ? I->n2 : (j2 >= I->n2 ? -I->n2 : 0);
  return j1 * I->n2 + j2;
}

// Per-tile set-up of smem slot s for tile tl at step it (written before the
// barrier of the preceding tile, read after it).
template <int N, int KT, bool MIX>
__device__ __forceinline__ void tile_setup(StageSmem<N, KT, MIX>& s, const View& v, const Tile& tl, int it, int stage) {
  const Inst* I = v.insts + tl.inst;
  const bool active = it >= 0 && it <= I->itfi;
  const int tid = threadIdx.x;
  if (tid == 0) s.active = active;
  if (!active) return;
  const int nk = I->nk, nsel = I->nsel;
  const FieldRow* fr = I->field + it;
  const double* Es = stage == 0 ? fr->Et : (stage == 3 ? fr[1].Et : fr->Eh);
  if (tid < nsel) {
    const int b = I->bsel[tid];
    s.G[tid] = I->wb[b] * (Es[0] * I->bvec[b][0] + Es[1] * I->bvec[b][1] + Es[2] * I->bvec[b][2]);
  }
  if (tid == 0) {
    for (int q = 0; q < 6; q++) s.E[q / 3][q % 3] = Es[q];
    s.on = (it == 0) || field_on(fr->Et);
  }
  for (int q = tid; q < nsel * KT; q += blockDim.x) {
    const int c = q / KT, kq = tl.k0 + q % KT;
    s.nb[c][q % KT] = kq < nk ? neighbour(I, kq, I->bsel[c]) : 0;
  }
}

template <int N, int KT, bool MIX, int OCC>
__global__ void __launch_bounds__(pad32(KT* TriB<N>::NT), min_blocks(pad32(KT* TriB<N>::NT), OCC))
    k_bstage(View v, int stage, int parity) {
  constexpr int NT = TriB<N>::NT;
  using S = typename Types<MIX>::S;
  using C = typename Types<MIX>::C;
  using R = decltype(C::x);
  __shared__ StageSmem<N, KT, MIX> sm[2];  // double buffered by tile: one barrier per tile
  const int tid = threadIdx.x;
  const int kl = tid % KT, e = tid / KT;
  const bool lane_ok = e < NT;
  int i = 0, j = 0;
  if (lane_ok) TriB<N>::ij(e, i, j);
  const int ntiles = *v.ntiles;
  if ((int)blockIdx.x >= ntiles) return;  // uniform over the block
  int buf = 0;
  Tile tl = v.tiles[blockIdx.x];
  int it = v.it[parity][tl.inst];
  tile_setup(sm[0], v, tl, it, stage);
  __syncthreads();
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    StageSmem<N, KT, MIX>& s = sm[buf];
    StageSmem<N, KT, MIX>& sn = sm[buf ^ 1];
    buf ^= 1;
    const Inst* I = v.insts + tl.inst;
    const bool active = s.active;
    const int nk = I->nk, nch = I->nch, nsel = I->nsel, fmask = I->fmask;
    const int k = tl.k0 + kl;
    const bool valid = active && lane_ok && k < nk;
    const double2* src = stage == 0 ? I->P0 : (stage == 2 ? I->Pb : I->Pa);
    // mixed: the stage inputs of stages 1-3 are FP32 deviations in the same planes
    const float2* src32 = reinterpret_cast<const float2*>(stage == 2 ? I->Pb : I->Pa);
    const size_t o = (size_t)e * nk + k;
    double2 p1v = cz(), p0v = cz(), Pe = cz();
    double Hii = 0.;
    S He = xmk<S>(0, 0), De[3] = {xmk<S>(0, 0), xmk<S>(0, 0), xmk<S>(0, 0)};
    S We[3] = {xmk<S>(0, 0), xmk<S>(0, 0), xmk<S>(0, 0)};
    C G = xmk<C>(0, 0);
    if (valid) {
      // every global load of the tile is issued here, the stencil gathers included
      Pe = (!MIX || stage == 0) ? src[o] : cvt<double2>(src32[o]);
      He = reinterpret_cast<const S*>(I->H)[o];
      const S* Dp = reinterpret_cast<const S*>(I->D);
      // components of the field that are zero for the whole run are not read
#pragma unroll
      for (int x = 0; x < 3; x++)
        if ((fmask >> x) & 1) De[x] = Dp[(size_t)x * NT * nk + o];
      if (MIX) {
#pragma unroll
        for (int x = 0; x < 3; x++)
          if ((fmask >> x) & 1) We[x] = reinterpret_cast<const S*>(I->W)[(size_t)x * NT * nk + o];
        if (i == j) Hii = I->Hdiag[(size_t)i * nk + k];
      }
      if (stage > 0) p1v = I->P1[o];
      if (stage == 1 || stage == 2) p0v = I->P0[o];
      if (s.on) {
        // k-gradient: sum_b (w_b E_pump . b) rho_e(k + b) (headers/RungeKutta.h:258-276)
        // over the b whose coefficient is not identically zero, gathers four at a
        // time, summed in b order (mixed: of the deviation; the rho_eq part is in W)
        constexpr int GB = 4;
        for (int b0 = 0; b0 < nsel; b0 += GB) {
          C pn[GB];
#pragma unroll
          for (int q = 0; q < GB; q++) {
            const int kb = s.nb[b0 + q < nsel ? b0 + q : 0][kl];
            pn[q] = (b0 + q >= nsel) ? xmk<C>(0, 0)
                    : (!MIX || stage == 0) ? cvt<C>(src[(size_t)e * nk + kb])
                                           : cvt<C>(src32[(size_t)e * nk + kb]);
          }
#pragma unroll
          for (int q = 0; q < GB; q++) {
            if (b0 + q >= nsel) break;
            G = xadd(G, xscale(pn[q], (R)s.G[b0 + q]));
          }
        }
      }
    }
    // set-up of the next tile of this block, published by the barrier below
    const int tn = t + gridDim.x;
    if (tn < ntiles) {
      tl = v.tiles[tn];
      it = v.it[parity][tl.inst];
      tile_setup(sn, v, tl, it, stage);
    }
    if (valid) {
      constexpr int RS = Rows<N, KT>::RS;
      const int oij = i * RS + j * KT + kl, oji = j * RS + i * KT + kl;
      const C pc = cvt<C>(Pe);
      s.P[oij] = pc;
      s.P[oji] = xconj(pc);
      // H~ = H + E^w . D, w = probe when exactly one index is a core band; the
      // lower entry is conj(H) + E^w . D (D symmetric)
      const int w = (i < nch) != (j < nch);
      C hu = cvt<C>(He), hl = xconj(cvt<C>(He));
#pragma unroll
      for (int x = 0; x < 3; x++) {
        const C d = cvt<C>(De[x]);
        hu = xadd(hu, xscale(d, (R)s.E[w][x]));
        hl = xadd(hl, xscale(d, (R)s.E[w][x]));
      }
      if (MIX) {
        if (i == j) {
          // the band energies enter in FP64: their FP32 rounding would be the same
          // at every k and turn into a coherent phase drift
          double ed = Hii;
#pragma unroll
          for (int x = 0; x < 3; x++) ed += (double)De[x].x * s.E[0][x];
          s.Ed[i * KT + kl] = ed;
          hu = hl = xmk<C>(0, 0);
        }
        // field-driven equilibrium terms, linear in E: -i[E.D, rho_eq] + k-gradient of rho_eq
#pragma unroll
        for (int x = 0; x < 3; x++) G = xadd(G, xscale(cvt<C>(We[x]), (R)s.E[0][x]));
      }
      s.H[oij] = hu;
      s.H[oji] = hl;
    }
    __syncthreads();
    if (valid) {
      // -i[H~, rho]_ij in the reference's transposed convention
      // (headers/RungeKutta.h:158-208): beta = sum_l H~_jl P_il - conj(H~_il P_jl);
      // on the diagonal this is 2i Im sum_l H~_il P_il, the reference's Pv_ii.
      // Mixed: P = rho - rho_eq, H~ without its diagonal (added below in FP64);
      // [H, rho_eq] vanishes for the ground-state projector and the E-linear
      // rho_eq terms come precomputed (W), so every FP32 rounding is relative to
      // the driven part instead of the O(1) background.
      constexpr int RS = Rows<N, KT>::RS;
      const C* Hi = s.H + i * RS + kl;
      const C* Hj = s.H + j * RS + kl;
      const C* Pi = s.P + i * RS + kl;
      const C* Pj = s.P + j * RS + kl;
      CommAcc<C> acc;
#pragma unroll
      for (int l = 0; l < N; l++) acc.add(l & 1, Hj[l * KT], Pi[l * KT], Hi[l * KT], Pj[l * KT]);
      const C beta = acc.sum();
      C vv = xmi(beta);
      if (!MIX && i < nch && j >= nch) vv = xadd(vv, xmi(xscale(cvt<C>(Pe), (R)(-I->wx2))));
      vv = xadd(vv, G);
      double2 d = cvt<double2>(vv);
      if constexpr (MIX) {
        // diagonal part of [H~, rho - rho_eq]: (H~_jj - H~_ii) (rho - rho_eq)_ij in FP64
        const double dE = s.Ed[j * KT + kl] - s.Ed[i * KT + kl];
        d = cadd(d, cmi(cscale(Pe, dE)));
      }
      if (i == j) d.y = 0;
      const double dt = I->dt, dt6 = I->dt6, dt3 = I->dt3, dt2 = dt / 2.0;
      if constexpr (MIX) {
        // FP64 accumulation of the deviation; FP32 stage inputs
        float2* Pa32 = reinterpret_cast<float2*>(I->Pa);
        float2* Pb32 = reinterpret_cast<float2*>(I->Pb);
        switch (stage) {
          case 0:
            I->P1[o] = cadd(Pe, cscale(d, dt6));
            Pa32[o] = cvt<float2>(cadd(Pe, cscale(d, dt2)));
            break;
          case 1:
            I->P1[o] = cadd(p1v, cscale(d, dt3));
            Pb32[o] = cvt<float2>(cadd(p0v, cscale(d, dt2)));
            break;
          case 2:
            I->P1[o] = cadd(p1v, cscale(d, dt3));
            Pa32[o] = cvt<float2>(cadd(p0v, cscale(d, dt)));
            break;
          default: {
            // the new deviation, and its FP32 copy that the next stage 0 reads
            const double2 pn = cadd(p1v, cscale(d, dt6));
            I->P0[o] = pn;
            Pb32[o] = cvt<float2>(pn);
            break;
          }
        }
      } else {
        switch (stage) {
          case 0:
            I->P1[o] = cadd(Pe, cscale(d, dt6));
            I->Pa[o] = cadd(Pe, cscale(d, dt2));
            break;
          case 1:
            I->P1[o] = cadd(p1v, cscale(d, dt3));
            I->Pb[o] = cadd(p0v, cscale(d, dt2));
            break;
          case 2:
            I->P1[o] = cadd(p1v, cscale(d, dt3));
            I->Pa[o] = cadd(p0v, cscale(d, dt));
            break;
          default:
            I->P0[o] = cadd(p1v, cscale(d, dt6));
            break;
        }
      }
    }
  }
}

// Equilibrium terms of the mixed-precision deviation form, linear in the
// field: W_x = -i [D_x, rho_eq] (transposed convention, as the commutator above)
// + sum_b w_b b_x rho_eq(k + b). Thread per (k, element); FP64 from the stored D.
template <class S>
__global__ void k_weq(const Inst* __restrict__ insts, int slot) {
  const Inst* I = insts + slot;
  const int n = I->n, nk = I->nk, nt = I->ntri;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = blockIdx.y;
  if (k >= nk) return;
  int i = 0, r = e;
  while (r >= n - i) {
    r -= n - i;
    i++;
  }
  const int j = i + r;
  auto up = [&](int a, int b) { return a * n - (a * (a - 1)) / 2 + (b - a); };
  auto Q = [&](int a, int b) -> double2 {
    return a <= b ? I->Peq[(size_t)up(a, b) * nk + k] : cconj(I->Peq[(size_t)up(b, a) * nk + k]);
  };
  const S* D = reinterpret_cast<const S*>(I->D);
  auto Dx = [&](int x, int a, int b) -> double2 {
    const S v = D[((size_t)x * nt + (a <= b ? up(a, b) : up(b, a))) * nk + k];
    return make_double2((double)v.x, (double)v.y);
  };
  S* W = reinterpret_cast<S*>(const_cast<void*>(I->W));
  const int i1 = k / I->n2, i2 = k - (k / I->n2) * I->n2;
  for (int x = 0; x < 3; x++) {
    double2 beta = cz();
    for (int l = 0; l < n; l++) beta = cadd(beta, csub(cmul(Dx(x, j, l), Q(i, l)), cconj(cmul(Dx(x, i, l), Q(j, l)))));
    double2 w = cmi(beta);
    for (int b = 0; b < I->nnb; b++) {
      int kb;
      if (I->lattice) {
        int j1 = i1 + I->off[b][0], j2 = i2 + I->off[b][1];
        j1 += j1 < 0 ? I->n1 : (j1 >= I->n1 ? -I->n1 : 0);
        j2 += j2 < 0 ? I->n2 : (j2 >= I->n2 ? -I->n2 : 0);
        kb = j1 * I->n2 + j2;
      } else {
        kb = I->nbr[(size_t)b * nk + k];
      }
      w = cadd(w, cscale(I->Peq[(size_t)e * nk + kb], I->wb[b] * I->bvec[b][x]));
    }
    W[((size_t)x * nt + e) * nk + k] = cvt<S>(w);
  }
}

// ------------------------------------------------------------------ dispatch
template <int N, int KT, bool MIX, int OCC>
cudaError_t stage_n(const View& v, int stage, int parity, int grid, cudaStream_t s) {
  k_bstage<N, KT, MIX, OCC><<<grid, pad32(KT * TriB<N>::NT), 0, s>>>(v, stage, parity);
  return cudaGetLastError();
}

template <int N, int KT, bool MIX, int OCC>
int stage_grid_n() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bstage<N, KT, MIX, OCC>, pad32(KT * TriB<N>::NT), 0);
  return sms * (per > 0 ? per : 1);
}

#define EDUS_BATCH_CLASSES(X) X(2, 16) X(2, 32) X(3, 16) X(3, 32) X(4, 16) X(5, 16) X(8, 4) X(8, 8) X(16, 2)

}  // namespace

bool class_supported(int N, int kt) {
#define X(n, k) \
  if (N == n && kt == k) return true;
  EDUS_BATCH_CLASSES(X)
#undef X
  return false;
}

cudaError_t launch_stage(int N, int kt, int occ, bool mixed, const View& v, int stage, int parity, int grid, cudaStream_t s) {
#define X(n, k)                                                                                       \
  if (N == n && kt == k) {                                                                            \
    if (occ == 0)                                                                                     \
      return mixed ? stage_n<n, k, true, 0>(v, stage, parity, grid, s) : stage_n<n, k, false, 0>(v, stage, parity, grid, s); \
    return mixed ? stage_n<n, k, true, 1>(v, stage, parity, grid, s) : stage_n<n, k, false, 1>(v, stage, parity, grid, s);   \
  }
  EDUS_BATCH_CLASSES(X)
#undef X
  return cudaErrorInvalidValue;
}

int stage_grid(int N, int kt, int occ, bool mixed) {
#define X(n, k)                                                                                   \
  if (N == n && kt == k) {                                                                        \
    if (occ == 0) return mixed ? stage_grid_n<n, k, true, 0>() : stage_grid_n<n, k, false, 0>(); \
    return mixed ? stage_grid_n<n, k, true, 1>() : stage_grid_n<n, k, false, 1>();               \
  }
  EDUS_BATCH_CLASSES(X)
#undef X
  return 0;
}


cudaError_t launch_weq(const Inst* insts, int slot, int ntri, int nk, cudaStream_t s) {
  k_weq<float2><<<dim3((nk + 127) / 128, ntri), 128, 0, s>>>(insts, slot);
  return cudaGetLastError();
}

}  // namespace batch
}  // namespace edus
