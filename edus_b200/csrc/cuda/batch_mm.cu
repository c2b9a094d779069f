// batch_mm.cu — RK4 stage kernel of the batch for larger band counts (n = 8, 16)
// in matrix-product form.
//
// The commutator of headers/RungeKutta.h:158-208 in the reference's transposed
// convention is beta_ij = sum_l H~_jl P_il - conj(H~_il P_jl) = C_ij - conj(C_ji)
// with C = P H~^T. Per tile of KT k points:
//   (A) element items (k, i <= j): loads, k-gradient gathers and H~ into
//       shared memory;
//   (B) every thread accumulates a BR x BC block of C for one k point in
//       registers: 1 / BR + 1 / BC shared loads per complex multiply-add,
//       against 2 for the element-parallel form;
//   (C) element items: beta from C, RWA, k-gradient, RK4 stage update.
// Same arithmetic as the FP64 k_bstage (batch_kernels.cu). FP64 only: a
// mixed-precision batch runs the element-parallel or the staged forms.
#include "batch.cuh"

namespace edus {
namespace batch {
namespace {

template <int N>
struct TriM {
  static constexpr int NT = N * (N + 1) / 2;
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

template <class C>
__device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <class To, class From>
__device__ __forceinline__ To cv(From a) { return mk<To>((decltype(To::x))a.x, (decltype(To::x))a.y); }

// shape of one instantiation
template <int N>
struct MM {
  using C = double2;
  static constexpr int BR = 2;                // rows of C per thread
  static constexpr int BC = 4;                // columns of C per thread
  static constexpr int TPK = (N / BR) * (N / BC);  // threads per k point
};

template <int N, int KT>
struct MMLayout {
  using C = typename MM<N>::C;
  static constexpr int RS = N * KT + 1;     // padded row of a shared matrix
  static constexpr int MAT = N * RS;        // one full matrix, all KT k points
  static constexpr int NT = TriM<N>::NT;
  static constexpr size_t bytes() {
    return sizeof(C) * (size_t)MAT * 3      // P, H, C
           + sizeof(C) * (size_t)NT * KT;   // k-gradient term per element
  }
};

struct Setup {
  double E[2][3];
  double G[kBatchMaxNb];  // w_b (E_pump . b)
  int on, active;
};

__device__ __forceinline__ bool field_nonzero(const double* E) {
  double s = 0;
  for (int q = 0; q < 6; q++) s += E[q] * E[q];
  return sqrt(s) > 1e-20;
}

__device__ __forceinline__ int nb_of(const Inst* I, int k, int b) {
  if (!I->lattice) return I->nbr[(size_t)b * I->nk + k];
  const int i1 = k / I->n2, i2 = k - i1 * I->n2;
  int j1 = i1 + I->off[b][0], j2 = i2 + I->off[b][1];
  j1 += j1 < 0 ? I->n1 : (j1 >= I->n1 ? -I->n1 : 0);
  j2 += j2 < 0 ? I->n2 : (j2 >= I->n2 ? -I->n2 : 0);
  return j1 * I->n2 + j2;
}

template <int N, int KT>
__global__ void __launch_bounds__(KT* MM<N>::TPK) k_bstage_mm(View v, int stage, int parity) {
  using L = MMLayout<N, KT>;
  using C = typename MM<N>::C;
  using S = C;
  using R = decltype(C::x);
  constexpr int NT = L::NT, RS = L::RS, MAT = L::MAT;
  constexpr int BR = MM<N>::BR, BC = MM<N>::BC;
  constexpr int NTHR = KT * MM<N>::TPK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sP = reinterpret_cast<C*>(smem_raw);
  C* sH = sP + MAT;
  C* sC = sH + MAT;
  C* sG = sC + MAT;  // [NT][KT]
  __shared__ Setup su[2];
  __shared__ int snb[2][kBatchMaxNb][KT];
  const int tid = threadIdx.x;
  const int ntiles = *v.ntiles;
  if ((int)blockIdx.x >= ntiles) return;  // uniform over the block

  auto setup = [&](int slot, const Tile& tl, int it) {
    const Inst* I = v.insts + tl.inst;
    const bool active = it >= 0 && it <= I->itfi;
    if (tid == 0) su[slot].active = active;
    if (!active) return;
    const FieldRow* fr = I->field + it;
    const double* Es = stage == 0 ? fr->Et : (stage == 3 ? fr[1].Et : fr->Eh);
    const int nsel = I->nsel, nk = I->nk;
    if (tid < nsel) {
      const int b = I->bsel[tid];
      su[slot].G[tid] = I->wb[b] * (Es[0] * I->bvec[b][0] + Es[1] * I->bvec[b][1] + Es[2] * I->bvec[b][2]);
    }
    if (tid == 0) {
      for (int q = 0; q < 6; q++) su[slot].E[q / 3][q % 3] = Es[q];
      su[slot].on = (it == 0) || field_nonzero(fr->Et);
    }
    for (int q = tid; q < nsel * KT; q += NTHR) {
      const int c = q / KT, kq = tl.k0 + q % KT;
      snb[slot][c][q % KT] = kq < nk ? nb_of(I, kq, I->bsel[c]) : 0;
    }
  };

  int buf = 0;
  Tile tl = v.tiles[blockIdx.x];
  int it = v.it[parity][tl.inst];
  setup(0, tl, it);
  __syncthreads();
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int cur = buf;
    buf ^= 1;
    const Inst* I = v.insts + tl.inst;
    const bool active = su[cur].active;
    const int nk = I->nk, nch = I->nch, nsel = I->nsel, fmask = I->fmask, k0 = tl.k0;
    const double2* src = stage == 0 ? I->P0 : (stage == 2 ? I->Pb : I->Pa);
    // ---- (A) element items
    if (active) {
      const S* Hg = reinterpret_cast<const S*>(I->H);
      const S* Dg = reinterpret_cast<const S*>(I->D);
      for (int q = tid; q < NT * KT; q += NTHR) {
        const int kl = q % KT, e = q / KT, k = k0 + kl;
        int i, j;
        TriM<N>::ij(e, i, j);
        const int oij = i * RS + j * KT + kl, oji = j * RS + i * KT + kl;
        if (k >= nk) {
          sP[oij] = sP[oji] = sH[oij] = sH[oji] = mk<C>(0, 0);
          sG[e * KT + kl] = mk<C>(0, 0);
          continue;
        }
        const size_t o = (size_t)e * nk + k;
        const double2 Pe = src[o];
        const S He = Hg[o];
        S De[3];
#pragma unroll
        for (int x = 0; x < 3; x++) De[x] = ((fmask >> x) & 1) ? Dg[(size_t)x * NT * nk + o] : mk<S>(0, 0);
        C G = mk<C>(0, 0);
        if (su[cur].on) {
          const double2* row = src + (size_t)e * nk;
          constexpr int GB = 4;
          for (int b0 = 0; b0 < nsel; b0 += GB) {
            double2 pn[GB];
#pragma unroll
            for (int u = 0; u < GB; u++) pn[u] = (b0 + u < nsel) ? row[snb[cur][b0 + u][kl]] : make_double2(0., 0.);
#pragma unroll
            for (int u = 0; u < GB; u++) {
              if (b0 + u >= nsel) break;
              const C pq = cv<C>(pn[u]);
              const R c = (R)su[cur].G[b0 + u];
              G = mk<C>(G.x + pq.x * c, G.y + pq.y * c);
            }
          }
        }
        sG[e * KT + kl] = G;
        const int w = (i < nch) != (j < nch);
        C hu = cv<C>(He), hl = mk<C>(hu.x, -hu.y);
#pragma unroll
        for (int x = 0; x < 3; x++) {
          const C d = cv<C>(De[x]);
          const R ex = (R)su[cur].E[w][x];
          hu = mk<C>(hu.x + d.x * ex, hu.y + d.y * ex);
          hl = mk<C>(hl.x + d.x * ex, hl.y + d.y * ex);
        }
        const C pc = cv<C>(Pe);
        sP[oij] = pc;
        sP[oji] = mk<C>(pc.x, -pc.y);
        sH[oij] = hu;
        sH[oji] = hl;
      }
    }
    // set-up of the next tile, published by the barrier below
    const int tn = t + gridDim.x;
    if (tn < ntiles) {
      tl = v.tiles[tn];
      it = v.it[parity][tl.inst];
      setup(buf, tl, it);
    }
    __syncthreads();
    // ---- (B) C = P H~^T, BR x BC per thread
    if (active) {
      const int kl = tid % KT, blk = tid / KT;
      const int i0 = (blk / (N / BC)) * BR, j0 = (blk % (N / BC)) * BC;
      C acc[BR][BC];
#pragma unroll
      for (int r = 0; r < BR; r++)
#pragma unroll
        for (int c = 0; c < BC; c++) acc[r][c] = mk<C>(0, 0);
      auto product = [&](const C* A, const C* B) {
#pragma unroll 4
        for (int l = 0; l < N; l++) {
          C a[BR], b[BC];
#pragma unroll
          for (int r = 0; r < BR; r++) a[r] = A[(i0 + r) * RS + l * KT + kl];
#pragma unroll
          for (int c = 0; c < BC; c++) b[c] = B[(j0 + c) * RS + l * KT + kl];
#pragma unroll
          for (int r = 0; r < BR; r++)
#pragma unroll
            for (int c = 0; c < BC; c++) {
              acc[r][c].x += a[r].x * b[c].x - a[r].y * b[c].y;
              acc[r][c].y += a[r].x * b[c].y + a[r].y * b[c].x;
            }
        }
      };
      product(sP, sH);
#pragma unroll
      for (int r = 0; r < BR; r++)
#pragma unroll
        for (int c = 0; c < BC; c++) sC[(i0 + r) * RS + (j0 + c) * KT + kl] = acc[r][c];
    }
    __syncthreads();
    // ---- (C) element items: beta_ij = C_ij - conj(C_ji), then the stage update
    if (active) {
      const double dt = I->dt, dt6 = I->dt6, dt3 = I->dt3, dt2 = dt / 2.0;
      for (int q = tid; q < NT * KT; q += NTHR) {
        const int kl = q % KT, e = q / KT, k = k0 + kl;
        if (k >= nk) continue;
        int i, j;
        TriM<N>::ij(e, i, j);
        const size_t o = (size_t)e * nk + k;
        double2 p1v = make_double2(0., 0.), p0v = make_double2(0., 0.);
        if (stage > 0) p1v = I->P1[o];
        if (stage == 1 || stage == 2) p0v = I->P0[o];
        const double2 Pe = src[o];
        const C cij = sC[i * RS + j * KT + kl], cji = sC[j * RS + i * KT + kl];
        C beta = mk<C>(cij.x - cji.x, cij.y + cji.y);
        C vv = mk<C>(beta.y, -beta.x);  // -i beta
        if (i < nch && j >= nch) {
          const R wx2 = (R)I->wx2;
          const C pcv = cv<C>(Pe);
          vv = mk<C>(vv.x - pcv.y * wx2, vv.y + pcv.x * wx2);  // -i (P * -wx2)
        }
        const C G = sG[e * KT + kl];
        vv = mk<C>(vv.x + G.x, vv.y + G.y);
        double2 d = cv<double2>(vv);
        if (i == j) d.y = 0;
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
    __syncthreads();  // phase (A) of the next tile rewrites the shared matrices
  }
}

template <int N, int KT>
cudaError_t mm_launch(const View& v, int stage, int parity, int grid, cudaStream_t s) {
  const size_t smem = MMLayout<N, KT>::bytes();
  static bool attr = false;  // per instantiation, per process
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_bstage_mm<N, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_bstage_mm<N, KT><<<grid, KT * MM<N>::TPK, smem, s>>>(v, stage, parity);
  return cudaGetLastError();
}

template <int N, int KT>
int mm_grid() {
  const size_t smem = MMLayout<N, KT>::bytes();
  cudaFuncSetAttribute(k_bstage_mm<N, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bstage_mm<N, KT>, KT * MM<N>::TPK, smem);
  return sms * (per > 0 ? per : 1);
}

}  // namespace

// Matrix-product stage kernel for the classes (8, 8), (8, 16), (16, 2), (16, 4), (16, 8).
bool mm_supported(int N, int kt) {
  return (N == 8 && (kt == 8 || kt == 16)) || (N == 16 && (kt == 2 || kt == 4 || kt == 8));
}

cudaError_t launch_stage_mm(int N, int kt, bool mixed, const View& v, int stage, int parity, int grid, cudaStream_t s) {
  if (mixed) return cudaErrorInvalidValue;  // FP64 only
#define MMX(n, k) \
  if (N == n && kt == k) return mm_launch<n, k>(v, stage, parity, grid, s);
  MMX(8, 8) MMX(8, 16) MMX(16, 2) MMX(16, 4) MMX(16, 8)
#undef MMX
  return cudaErrorInvalidValue;
}

int stage_grid_mm(int N, int kt, bool mixed) {
  if (mixed) return 0;  // FP64 only
#define MMX(n, k) \
  if (N == n && kt == k) return mm_grid<n, k>();
  MMX(8, 8) MMX(8, 16) MMX(16, 2) MMX(16, 4) MMX(16, 8)
#undef MMX
  return 0;
}

}  // namespace batch
}  // namespace edus
