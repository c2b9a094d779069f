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
// Row r of a shared matrix starts at r * RS(N, KT): one entry of padding per
// row keeps the rows of a warp's elements on different banks.
template <int N, int KT>
struct Rows {
  static constexpr int RS = N * KT + 1;
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
  const int nk = I->nk, nnb = I->nnb;
  const FieldRow* fr = I->field + it;
  const double* Es = stage == 0 ? fr->Et : (stage == 3 ? fr[1].Et : fr->Eh);
  if (tid < nnb) {
    const int b = tid;
    s.G[b] = I->wb[b] * (Es[0] * I->bvec[b][0] + Es[1] * I->bvec[b][1] + Es[2] * I->bvec[b][2]);
  }
  if (tid == 0) {
    for (int q = 0; q < 6; q++) s.E[q / 3][q % 3] = Es[q];
    s.on = (it == 0) || field_on(fr->Et);
  }
  for (int q = tid; q < nnb * KT; q += blockDim.x) {
    const int b = q / KT, kq = tl.k0 + q % KT;
    s.nb[b][q % KT] = kq < nk ? neighbour(I, kq, b) : 0;
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
    const int nk = I->nk, nch = I->nch, nnb = I->nnb;
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
#pragma unroll
      for (int x = 0; x < 3; x++) De[x] = Dp[(size_t)x * NT * nk + o];
      if (MIX) {
#pragma unroll
        for (int x = 0; x < 3; x++) We[x] = reinterpret_cast<const S*>(I->W)[(size_t)x * NT * nk + o];
        if (i == j) Hii = I->Hdiag[(size_t)i * nk + k];
      }
      if (stage > 0) p1v = I->P1[o];
      if (stage == 1 || stage == 2) p0v = I->P0[o];
      if (s.on) {
        // k-gradient: sum_b (w_b E_pump . b) rho_e(k + b) (headers/RungeKutta.h:258-276),
        // gathers four at a time, summed in b order (mixed: of the deviation; the
        // rho_eq part is in W)
        constexpr int GB = 4;
        for (int b0 = 0; b0 < nnb; b0 += GB) {
          C pn[GB];
#pragma unroll
          for (int q = 0; q < GB; q++) {
            const int kb = s.nb[b0 + q < nnb ? b0 + q : 0][kl];
            pn[q] = (b0 + q >= nnb) ? xmk<C>(0, 0)
                    : (!MIX || stage == 0) ? cvt<C>(src[(size_t)e * nk + kb])
                                           : cvt<C>(src32[(size_t)e * nk + kb]);
          }
#pragma unroll
          for (int q = 0; q < GB; q++) {
            if (b0 + q >= nnb) break;
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
      C beta = xmk<C>(0, 0);
#pragma unroll
      for (int l = 0; l < N; l++) {
        const C x = xmul(Hj[l * KT], Pi[l * KT]);
        const C y = xmul(Hi[l * KT], Pj[l * KT]);
        beta = xadd(beta, xsub(x, xconj(y)));
      }
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
      const double dt = I->dt, dt6 = dt / 6.0, dt3 = dt / 3.0, dt2 = dt / 2.0;
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
          default:
            I->P0[o] = cadd(p1v, cscale(d, dt6));
            break;
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

// ------------------------------------------------------------------ observables
struct Part {
  double pop[kMaxBands];
  double2 J1[3], J2[3], TA[3];
  double pmax, pmin;
};
__device__ __forceinline__ void part_zero(Part& p) {
  for (int c = 0; c < kMaxBands; c++) p.pop[c] = 0;
  for (int x = 0; x < 3; x++) p.J1[x] = p.J2[x] = p.TA[x] = cz();
  p.pmax = 0;
  p.pmin = 1.0;
}
__device__ __forceinline__ void part_add(Part& d, const Part& o, int n) {
  for (int c = 0; c < n; c++) d.pop[c] += o.pop[c];
  for (int x = 0; x < 3; x++) {
    d.J1[x] = cadd(d.J1[x], o.J1[x]);
    d.J2[x] = cadd(d.J2[x], o.J2[x]);
    d.TA[x] = cadd(d.TA[x], o.TA[x]);
  }
  d.pmax = fmax(d.pmax, o.pmax);
  d.pmin = fmin(d.pmin, o.pmin);
}

__device__ __forceinline__ double warp_sum(double x) {
  for (int s = 16; s > 0; s >>= 1) x += __shfl_xor_sync(0xffffffffu, x, s);
  return x;
}

constexpr int kRedVals = kMaxBands + 20;

// Sums (max / min for pmax / pmin) one Part per thread over the block into
// out, in a fixed order: warp butterflies, then warps in index order.
template <int N, int NW>
__device__ __forceinline__ void block_reduce(Part& my, Part& out, double (*sW)[kRedVals]) {
  const int lane = threadIdx.x % 32, w = threadIdx.x / 32;
  double vals[N + 20];
  for (int c = 0; c < N; c++) vals[c] = my.pop[c];
  for (int x = 0; x < 3; x++) {
    vals[N + 6 * x + 0] = my.J1[x].x;
    vals[N + 6 * x + 1] = my.J1[x].y;
    vals[N + 6 * x + 2] = my.J2[x].x;
    vals[N + 6 * x + 3] = my.J2[x].y;
    vals[N + 6 * x + 4] = my.TA[x].x;
    vals[N + 6 * x + 5] = my.TA[x].y;
  }
  for (int q = 0; q < N + 18; q++) vals[q] = warp_sum(vals[q]);
  double pmax = my.pmax, pmin = my.pmin;
  for (int s = 16; s > 0; s >>= 1) {
    pmax = fmax(pmax, __shfl_xor_sync(0xffffffffu, pmax, s));
    pmin = fmin(pmin, __shfl_xor_sync(0xffffffffu, pmin, s));
  }
  vals[N + 18] = pmax;
  vals[N + 19] = pmin;
  if (lane == 0)
    for (int q = 0; q < N + 20; q++) sW[w][q] = vals[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    part_zero(out);
    for (int ww = 0; ww < NW; ww++) {
      for (int c = 0; c < N; c++) out.pop[c] += sW[ww][c];
      for (int x = 0; x < 3; x++) {
        out.J1[x] = cadd(out.J1[x], cmk(sW[ww][N + 6 * x], sW[ww][N + 6 * x + 1]));
        out.J2[x] = cadd(out.J2[x], cmk(sW[ww][N + 6 * x + 2], sW[ww][N + 6 * x + 3]));
        out.TA[x] = cadd(out.TA[x], cmk(sW[ww][N + 6 * x + 4], sW[ww][N + 6 * x + 5]));
      }
      out.pmax = fmax(out.pmax, sW[ww][N + 18]);
      out.pmin = fmin(out.pmin, sW[ww][N + 19]);
    }
  }
  __syncthreads();
}

// Observables at one output instant (headers/Observables_MPI.h:217-484,559-598,
// 668-775) of every instance due at this tick; the tile's k points are taken
// KO at a time. Also advances the step counter of every instance of the class.
template <int N, int KO, bool MIX>
__global__ void __launch_bounds__(pad32(KO* TriB<N>::NT)) k_bobs(View v, int parity, int kt) {
  constexpr int NT = TriB<N>::NT;
  constexpr int NTHR = pad32(KO * NT);
  constexpr int NW = NTHR / 32;
  using S = typename Types<MIX>::S;
  __shared__ double2 sP[NT][KO];
  __shared__ double2 sH[NT][KO];
  __shared__ double2 sD[3][NT][KO];
  __shared__ double2 sU[N * N][KO];
  __shared__ double sW[NW][kRedVals];
  __shared__ Part sT;
  __shared__ bool sLast;
  const int tid = threadIdx.x;
  const int kl = tid % KO, e = tid / KO;
  const bool lane_ok = e < NT;
  int i = 0, j = 0;
  if (lane_ok) TriB<N>::ij(e, i, j);
  const int ntiles = *v.ntiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = v.tiles[t];
    const int it = v.it[parity][tl.inst];
    const Inst* I = v.insts + tl.inst;
    const int itfi = I->itfi;
    if (tl.t_in == 0 && tid == 0) v.it[parity ^ 1][tl.inst] = it <= itfi ? it + 1 : it;
    if (it < 0 || it > itfi || it % I->res != 0) continue;
    const int nk = I->nk, nch = I->nch;
    const S* H = reinterpret_cast<const S*>(I->H);
    const S* D = reinterpret_cast<const S*>(I->D);
    const S* GE = reinterpret_cast<const S*>(I->GE);
    const S* U = reinterpret_cast<const S*>(I->U);
    Part my;
    part_zero(my);
    const int kend = min(tl.k0 + kt, nk);
    for (int k0 = tl.k0; k0 < kend; k0 += KO) {
      const int k = k0 + kl;
      const bool valid = lane_ok && k < kend;
      if (lane_ok) {
        const size_t o = (size_t)e * nk + k;
        sP[e][kl] = valid ? (MIX ? cadd(I->P0[o], I->Peq[o]) : I->P0[o]) : cz();
        sH[e][kl] = valid ? cvt<double2>(H[o]) : cz();
        for (int x = 0; x < 3; x++) sD[x][e][kl] = valid ? cvt<double2>(D[(size_t)x * NT * nk + o]) : cz();
      }
      for (int q = tid; q < N * N * KO; q += NTHR) {
        const int u = q / KO, kq = k0 + q % KO;
        sU[u][q % KO] = kq < kend ? cvt<double2>(U[(size_t)u * nk + kq]) : cz();
      }
      __syncthreads();
      if (valid) {
        auto Pf = [&](int r, int c) -> double2 { return (r <= c) ? sP[TriB<N>::idx(r, c)][kl] : cconj(sP[TriB<N>::idx(c, r)][kl]); };
        auto Hf = [&](int r, int c) -> double2 { return (r <= c) ? sH[TriB<N>::idx(r, c)][kl] : cconj(sH[TriB<N>::idx(c, r)][kl]); };
        auto Df = [&](int x, int r, int c) -> double2 {
          return r <= c ? sD[x][TriB<N>::idx(r, c)][kl] : sD[x][TriB<N>::idx(c, r)][kl];
        };
        const double2 pe = sP[e][kl];
        if (I->want_current) {
          const size_t o = (size_t)e * nk + k;
          for (int x = 0; x < 3; x++) {
            const double2 ge = cvt<double2>(GE[(size_t)x * NT * nk + o]);
            my.J1[x] = cadd(my.J1[x], cmul(pe, ge));
            if (i != j) my.J1[x] = cadd(my.J1[x], cmul(cconj(pe), cconj(ge)));
          }
          // J2: sum_l P_ab H_al conj(D_bl) for (a, b) = (i, j) and, off the diagonal, (j, i)
          for (int pass = 0; pass < (i == j ? 1 : 2); pass++) {
            const int a = pass ? j : i, b = pass ? i : j;
            const double2 pab = pass ? cconj(pe) : pe;
            for (int l = 0; l < N; l++) {
              const double2 ph = cmul(pab, Hf(a, l));
              for (int x = 0; x < 3; x++) my.J2[x] = cadd(my.J2[x], cmulc(ph, Df(x, b, l)));
            }
          }
        }
        if (I->want_tabs && i < nch && j >= nch)
          for (int x = 0; x < 3; x++) my.TA[x] = csub(my.TA[x], cmul(cscale(sD[x][e][kl], 2.), pe));
        if (e < N) {
          // population of band c = e in the model eigenbasis: sum_ij conj(U_ci) P_ij U_cj
          const int c = e;
          double2 acc = cz();
          for (int ii = 0; ii < N; ii++) {
            double2 m = cz();
            for (int jj = 0; jj < N; jj++) m = cadd(m, cmul(Pf(ii, jj), sU[c * N + jj][kl]));
            acc = cadd(acc, cmul(cconj(sU[c * N + ii][kl]), m));
          }
          const double Pk = acc.x;
          my.pop[c] += Pk;
          if (c < I->nbands) {
            my.pmax = fmax(my.pmax, fabs(1. - Pk));
            my.pmin = fmin(my.pmin, 1. - Pk);
          } else {
            my.pmax = fmax(my.pmax, fabs(Pk));
            my.pmin = fmin(my.pmin, Pk);
          }
        }
      }
      __syncthreads();
    }
    block_reduce<N, NW>(my, sT, sW);
    if (tid == 0) {
      reinterpret_cast<Part*>(I->part)[tl.t_in] = sT;
      __threadfence();
      sLast = atomicAdd(I->done, 1u) == (unsigned)(I->ntiles - 1);
    }
    __syncthreads();
    if (sLast) {
      // last tile of the instance to finish: fixed-order reduction over its tiles
      __threadfence();
      const Part* part = reinterpret_cast<const Part*>(I->part);
      Part acc;
      part_zero(acc);
      for (int q = tid; q < I->ntiles; q += NTHR) {
        // written by other blocks of this launch: read past L1
        Part pq;
        const double* src = reinterpret_cast<const double*>(part + q);
        double* dst = reinterpret_cast<double*>(&pq);
        for (int w = 0; w < (int)(sizeof(Part) / sizeof(double)); w++) dst[w] = __ldcg(src + w);
        part_add(acc, pq, N);
      }
      block_reduce<N, NW>(acc, sT, sW);
      if (tid == 0) {
        edus_obs rec;
        memset(&rec, 0, sizeof(rec));
        rec.t = I->field[it].t;
        if (it > 0)
          for (int x = 0; x < 3; x++) {
            rec.EF_pump[x] = I->field[it].Et[x];
            rec.EF_probe[x] = I->field[it].Et[3 + x];
          }
        rec.dt = I->dt;
        const double inv = 1. / nk;
        double trace = -(double)I->nbands, ncd = 0;
        for (int c = 0; c < N; c++) {
          double val = sT.pop[c] * inv;
          trace += val;
          if (c < I->nbands) val = 1.0 - val;
          rec.pop[c] = val;
          if (val > ncd) ncd = val;
        }
        for (int x = 0; x < 3; x++) {
          rec.J1[2 * x] = sT.J1[x].x * I->scaleJ;
          rec.J1[2 * x + 1] = sT.J1[x].y * I->scaleJ;
          rec.J2[x] = -2. * (sT.J2[x].y * I->scaleJ);
          rec.tabs[2 * x] = sT.TA[x].x * I->scaleTA * inv;
          rec.tabs[2 * x + 1] = sT.TA[x].y * I->scaleTA * inv;
        }
        rec.trace_dev = trace;
        rec.p_cond_max = sT.pmax;
        rec.p_min = sT.pmin;
        rec.n_cond = ncd;
        I->log[it / I->res] = rec;
        *I->done = 0u;
      }
    }
    __syncthreads();
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

// observable sub-tile length per band count
template <int N>
struct ObsKO {
  static constexpr int v = N <= 2 ? 32 : (N <= 3 ? 16 : (N <= 4 ? 8 : (N <= 8 ? 4 : 1)));
};

template <int N, bool MIX>
cudaError_t obs_n(const View& v, int parity, int kt, int grid, cudaStream_t s) {
  constexpr int KO = ObsKO<N>::v;
  k_bobs<N, KO, MIX><<<grid, pad32(KO * TriB<N>::NT), 0, s>>>(v, parity, kt);
  return cudaGetLastError();
}

template <int N, bool MIX>
int obs_grid_n() {
  constexpr int KO = ObsKO<N>::v;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bobs<N, KO, MIX>, pad32(KO * TriB<N>::NT), 0);
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

cudaError_t launch_obs(int N, int kt, bool mixed, const View& v, int parity, int grid, cudaStream_t s) {
  switch (N) {
    case 2: return mixed ? obs_n<2, true>(v, parity, kt, grid, s) : obs_n<2, false>(v, parity, kt, grid, s);
    case 3: return mixed ? obs_n<3, true>(v, parity, kt, grid, s) : obs_n<3, false>(v, parity, kt, grid, s);
    case 4: return mixed ? obs_n<4, true>(v, parity, kt, grid, s) : obs_n<4, false>(v, parity, kt, grid, s);
    case 5: return mixed ? obs_n<5, true>(v, parity, kt, grid, s) : obs_n<5, false>(v, parity, kt, grid, s);
    case 8: return mixed ? obs_n<8, true>(v, parity, kt, grid, s) : obs_n<8, false>(v, parity, kt, grid, s);
    case 16: return mixed ? obs_n<16, true>(v, parity, kt, grid, s) : obs_n<16, false>(v, parity, kt, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

int obs_grid(int N, int kt, bool mixed) {
  (void)kt;
  switch (N) {
    case 2: return mixed ? obs_grid_n<2, true>() : obs_grid_n<2, false>();
    case 3: return mixed ? obs_grid_n<3, true>() : obs_grid_n<3, false>();
    case 4: return mixed ? obs_grid_n<4, true>() : obs_grid_n<4, false>();
    case 5: return mixed ? obs_grid_n<5, true>() : obs_grid_n<5, false>();
    case 8: return mixed ? obs_grid_n<8, true>() : obs_grid_n<8, false>();
    case 16: return mixed ? obs_grid_n<16, true>() : obs_grid_n<16, false>();
    default: return 0;
  }
}

size_t obs_part_bytes() { return sizeof(Part); }

cudaError_t launch_weq(const Inst* insts, int slot, int ntri, int nk, cudaStream_t s) {
  k_weq<float2><<<dim3((nk + 127) / 128, ntri), 128, 0, s>>>(insts, slot);
  return cudaGetLastError();
}

}  // namespace batch
}  // namespace edus
