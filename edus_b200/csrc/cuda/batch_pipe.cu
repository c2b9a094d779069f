// batch_pipe.cu — mixed-precision RK4 stage kernel of the batch engine with
// asynchronous staging (register profile 3).
//
// Same arithmetic as k_bstage<N, KT, mixed> (batch_kernels.cu), element by
// element and in the same order, so both forms give the same numbers; the
// difference is how the operands reach the SM:
//
//  * each persistent block owns a contiguous run of the class's tile table,
//    so consecutive tiles almost always belong to one instance. The
//    instance's pointers, grid, stencil and stage field live in a small
//    shared-memory record (ring of 3) that warp 0 refreshes only when the
//    instance changes, one tile ahead;
//  * every thread copies the operands of its own element for the NEXT tile
//    (stage input, rho - rho_eq, RK4 accumulator, H, the field components in
//    use of D and W, the FP64 band energy, the stencil gathers rho(k + b))
//    into its own shared-memory slots with cp.async right after the tile's
//    barrier, then evaluates the commutator of the current tile while the
//    copies are in flight. One wait_group and one barrier per tile.
//
// The staging slots for D, W and the stencil gathers are sized at launch for
// the most field components and stencil vectors in use among the class's
// instances. Eligible instances: lattice stencils (the host falls back to
// k_bstage otherwise).
#include "batch.cuh"

namespace edus {
namespace batch {
namespace {

template <int N>
struct TriP {
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

constexpr int pipe_pad32(int x) { return (x + 31) / 32 * 32; }

__device__ __forceinline__ float2 fmk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fadd(float2 a, float2 b) { return fmk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fscale(float2 a, float s) { return fmk(a.x * s, a.y * s); }
__device__ __forceinline__ float2 fconj(float2 a) { return fmk(a.x, -a.y); }
__device__ __forceinline__ float2 fmi(float2 a) { return fmk(a.y, -a.x); }
__device__ __forceinline__ float2 to_f(double2 a) { return fmk((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One instance for one stage launch. Fields that are read together sit in
// 16-byte groups and are read with one vector load (a broadcast: one shared
// memory wavefront per warp).
struct alignas(16) PipeMeta {
  int active, nk, on, nsel;      // group a
  int nch, n1, n2, ncomp;        // group b
  const double2* P0;             // rho - rho_eq (FP64); stage 3 writes the new one
  const float2* src;             // FP32 stage input: stage 0 Pb (copy of P0), 1 Pa, 2 Pb, 3 Pa
  double2* P1;
  const float2* H;
  const double* Hdiag;
  float2* dst;                   // FP32 stage input written: stage 0 Pa, 1 Pb, 2 Pa, 3 Pb
  const float2* DW[3][2];        // (D_x, W_x) of the field components in use
  double E[3][2];                // (pump, probe / 2) of the components in use
  float Ef[3][4];                // the same in FP32 (pump, probe / 2, -, -) as the commutator uses them
  int off[kBatchMaxNb][2];       // lattice steps of the stencil vectors in use
  int delta[kBatchMaxNb];        // d1 n2 + d2: k + b on an interior tile
  float G[kBatchMaxNb];          // their w_b (E_pump . b), in FP32 as the commutator uses it
  double dt, dt6, dt3;           // the step, dt / 6, dt / 3 (the instance's host-side divisions)
  int inst, pad;
};

template <class V, class T>
__device__ __forceinline__ V ldv(const T* p) { return *reinterpret_cast<const V*>(p); }

template <int N, int KT>
struct PipeRows {
  static constexpr int RS = N * KT + ((N % 2) ? 0 : KT);  // as k_bstage (mixed)
  static constexpr int SIZE = N * RS;
};

// Dynamic shared memory of one block, carved at run time: per-thread staging
// slots (struct of arrays, slot = thread; sD, sW and sG sized for the field
// components and stencil vectors of the class), the double-buffered exchange
// matrices and the ring of instance records.
template <int N, int KT>
struct PipeCarve {
  static constexpr int NT = TriP<N>::NT;
  static constexpr int NTHR = pipe_pad32(KT * NT);
  double2 *sP0, *sP1;
  double* sHii;
  float2 *sPin, *sH, *sD, *sW, *sG;  // sD, sW: [ncomp][NTHR]; sG: [nsel][NTHR]
  float2 *xP, *xH;                    // [2][SIZE]
  float2* xC;                         // blocked commutator only: C = P H~^T [SIZE]
  double* xEd;                        // [2][N * KT]
  PipeMeta* meta;                     // [3]
  static __host__ __device__ size_t bytes(int nsel, int ncomp, int cb) {
    return (size_t)NTHR * (16 + 16 + 8 + 8 + 8 + 16 * ncomp + 8 * nsel) + (4 + (cb ? 1 : 0)) * PipeRows<N, KT>::SIZE * sizeof(float2) +
           2 * N * KT * sizeof(double) + 3 * sizeof(PipeMeta);
  }
  __device__ PipeCarve(unsigned char* base, int nsel, int ncomp, int cb) {
    unsigned char* p = base;
    auto take = [&](size_t b) {
      unsigned char* r = p;
      p += b;
      return r;
    };
    sP0 = (double2*)take(NTHR * 16);
    sP1 = (double2*)take(NTHR * 16);
    sHii = (double*)take(NTHR * 8);
    sPin = (float2*)take(NTHR * 8);
    sH = (float2*)take(NTHR * 8);
    sD = (float2*)take((size_t)NTHR * 8 * ncomp);
    sW = (float2*)take((size_t)NTHR * 8 * ncomp);
    sG = (float2*)take((size_t)NTHR * 8 * nsel);
    xP = (float2*)take(2 * PipeRows<N, KT>::SIZE * sizeof(float2));
    xH = (float2*)take(2 * PipeRows<N, KT>::SIZE * sizeof(float2));
    xC = (float2*)take(cb ? PipeRows<N, KT>::SIZE * sizeof(float2) : 0);
    xEd = (double*)take(2 * N * KT * sizeof(double));
    meta = (PipeMeta*)take(3 * sizeof(PipeMeta));
  }
};

__device__ __forceinline__ bool pipe_field_on(const double* E) {
  double s = 0;
  for (int q = 0; q < 6; q++) s += E[q] * E[q];
  return sqrt(s) > 1e-20;
}

// Instance record for this stage, written by the 32 lanes of one warp.
template <int N, int STAGE>
__device__ __forceinline__ void pipe_meta(PipeMeta& M, const View& v, int inst, int parity, int lane) {
  constexpr int NT = TriP<N>::NT;
  const Inst* I = v.insts + inst;
  const int it = (parity ? v.it[1] : v.it[0])[inst];
  const bool active = it >= 0 && it <= I->itfi;
  if (lane == 0) {
    M.inst = inst;
    M.active = active;
  }
  if (!active) return;
  const int nk = I->nk, fmask = I->fmask;
  const FieldRow* fr = I->field + it;
  const double* Es = STAGE == 0 ? fr->Et : (STAGE == 3 ? fr[1].Et : fr->Eh);
  float2* Pa32 = reinterpret_cast<float2*>(I->Pa);
  float2* Pb32 = reinterpret_cast<float2*>(I->Pb);
  if (lane == 0) {
    M.P0 = I->P0;
    M.src = (STAGE == 1 || STAGE == 3) ? Pa32 : Pb32;
    M.dst = (STAGE == 0 || STAGE == 2) ? Pa32 : Pb32;
    M.H = reinterpret_cast<const float2*>(I->H);
    M.Hdiag = I->Hdiag;
    M.P1 = I->P1;
    M.on = (it == 0) || pipe_field_on(fr->Et);
    M.nk = nk;
    M.nch = I->nch;
    M.n1 = I->n1;
    M.n2 = I->n2;
    M.nsel = I->nsel;
    M.dt = I->dt;
    M.dt6 = I->dt6;
    M.dt3 = I->dt3;
    M.ncomp = (fmask & 1) + ((fmask >> 1) & 1) + ((fmask >> 2) & 1);
  }
  if (lane >= 24 && lane < 27) {
    // component c = lane - 24: the c-th set bit of the field mask
    const int c = lane - 24;
    int x = -1, seen = 0;
    for (int q = 0; q < 3 && x < 0; q++)
      if ((fmask >> q) & 1) {
        if (seen == c) x = q;
        seen++;
      }
    if (x >= 0) {
      const size_t plane = (size_t)NT * nk;
      M.DW[c][0] = reinterpret_cast<const float2*>(I->D) + x * plane;
      M.DW[c][1] = reinterpret_cast<const float2*>(I->W) + x * plane;
      M.E[c][0] = Es[x];
      M.E[c][1] = Es[3 + x];
      M.Ef[c][0] = (float)Es[x];
      M.Ef[c][1] = (float)Es[3 + x];
    }
  }
  if (lane < I->nsel) {
    const int b = I->bsel[lane];
    M.G[lane] = (float)(I->wb[b] * (Es[0] * I->bvec[b][0] + Es[1] * I->bvec[b][1] + Es[2] * I->bvec[b][2]));
    M.off[lane][0] = I->off[b][0];
    M.off[lane][1] = I->off[b][1];
    M.delta[lane] = I->off[b][0] * I->n2 + I->off[b][1];
  }
}

// Copies of this thread's operands of tile k0 (element e, k = k0 + kl).
template <int N, int KT, int STAGE>
__device__ __forceinline__ void pipe_issue(const PipeCarve<N, KT>& S, const PipeMeta& M, int k0, bool interior, int tid, int kl,
                                           int e, int i, int j) {
  constexpr int NTHR = PipeCarve<N, KT>::NTHR;
  const int4 a = ldv<int4>(&M.active);  // active, nk, on, nsel
  const int k = k0 + kl, nk = a.y;
  if (!a.x || e >= TriP<N>::NT || k >= nk) return;
  const int o = e * nk + k;
  const ulonglong2 p01 = ldv<ulonglong2>(&M.P0);  // P0, src
  const ulonglong2 p23 = ldv<ulonglong2>(&M.P1);  // P1, H
  const double2* P0 = (const double2*)p01.x;
  const float2* src = (const float2*)p01.y;
  if (STAGE <= 2) cp_async16(&S.sP0[tid], P0 + o);
  if (STAGE >= 1) {
    cp_async8(&S.sPin[tid], src + o);
    cp_async16(&S.sP1[tid], (const double2*)p23.x + o);
  }
  cp_async8(&S.sH[tid], (const float2*)p23.y + o);
  const int4 b = ldv<int4>(&M.nch);  // nch, n1, n2, ncomp
  for (int c = 0; c < b.w; c++) {
    const ulonglong2 dw = ldv<ulonglong2>(&M.DW[c][0]);
    cp_async8(&S.sD[c * NTHR + tid], (const float2*)dw.x + o);
    cp_async8(&S.sW[c * NTHR + tid], (const float2*)dw.y + o);
  }
  if (i == j) cp_async8(&S.sHii[tid], M.Hdiag + i * nk + k);
  if (a.z && interior) {
    const float2* at = src + o;
    for (int c = 0; c < a.w; c += 4) {
      const int4 d = ldv<int4>(&M.delta[c]);
      cp_async8(&S.sG[c * NTHR + tid], at + d.x);
      if (c + 1 < a.w) cp_async8(&S.sG[(c + 1) * NTHR + tid], at + d.y);
      if (c + 2 < a.w) cp_async8(&S.sG[(c + 2) * NTHR + tid], at + d.z);
      if (c + 3 < a.w) cp_async8(&S.sG[(c + 3) * NTHR + tid], at + d.w);
    }
  } else if (a.z) {
    const int n1 = b.y, n2 = b.z;
    const int i1 = k / n2, i2 = k - i1 * n2;
    const float2* row = src + e * nk;
    for (int c = 0; c < a.w; c += 2) {
      const int4 d = ldv<int4>(&M.off[c][0]);  // steps of c and c + 1
#pragma unroll
      for (int h = 0; h < 2; h++) {
        if (c + h >= a.w) break;
        int j1 = i1 + (h ? d.z : d.x), j2 = i2 + (h ? d.w : d.y);
        j1 += j1 < 0 ? n1 : (j1 >= n1 ? -n1 : 0);
        j2 += j2 < 0 ? n2 : (j2 >= n2 ? -n2 : 0);
        cp_async8(&S.sG[(c + h) * NTHR + tid], row + j1 * n2 + j2);
      }
    }
  }
}

// Register blocks of the blocked commutator (C = P H~^T, BR x BC entries of C
// per thread and k point): CB 1, 2 x 2 (for 16 bands measured 5 % faster than
// 4 x 2: more threads share the phase); CB 2, 2 x 1 (twice the threads again,
// about all of the block's). Every entry of C is the same sum over l in l
// order in every blocking.
template <int N, int CB>
struct CBlk {
  static constexpr int BR = 2, BC = CB == 2 ? 1 : 2;
  static constexpr int NB = (N / BR) * (N / BC);
};

template <int N, int KT, int STAGE, int CB>
__global__ void __launch_bounds__(pipe_pad32(KT* TriP<N>::NT), (1152 / pipe_pad32(KT * TriP<N>::NT)) > 0 ? 1152 / pipe_pad32(KT * TriP<N>::NT) : 1)
    k_bpipe(View v, int parity, int nsel_max, int ncomp_max) {
  constexpr int NT = TriP<N>::NT;
  constexpr int RS = PipeRows<N, KT>::RS;
  constexpr int SIZE = PipeRows<N, KT>::SIZE;
  constexpr int NTHR = PipeCarve<N, KT>::NTHR;
  extern __shared__ __align__(16) unsigned char pipe_smem[];
  const PipeCarve<N, KT> S(pipe_smem, nsel_max, ncomp_max, CB);
  const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
  const int kl = tid % KT, e = tid / KT;
  const bool lane_ok = e < NT;
  int i = 0, j = 0;
  if (lane_ok) TriP<N>::ij(e, i, j);
  const int ntiles = *v.ntiles;
  const int t0 = (int)((long long)blockIdx.x * ntiles / gridDim.x);
  const int t1 = (int)((long long)(blockIdx.x + 1) * ntiles / gridDim.x);
  if (t0 >= t1) return;  // uniform over the block

  Tile cur = v.tiles[t0];
  int ms = 0;
  if (warp == 0) pipe_meta<N, STAGE>(S.meta[0], v, cur.inst, parity, lane);
  __syncthreads();
  pipe_issue<N, KT, STAGE>(S, S.meta[0], cur.k0, cur.interior, tid, kl, e, i, j);
  cp_async_commit();
  Tile nxt = t0 + 1 < t1 ? v.tiles[t0 + 1] : cur;

  for (int t = t0; t < t1; t++) {
    const PipeMeta& M = S.meta[ms];
    const int buf = t & 1;
    float2* xP = S.xP + buf * SIZE;
    float2* xH = S.xH + buf * SIZE;
    double* xEd = S.xEd + buf * N * KT;
    const int4 a = ldv<int4>(&M.active);  // active, nk, on, nsel
    const bool valid = a.x && lane_ok && cur.k0 + kl < a.y;
    cp_async_wait_all();
    // ---- this tile's operands: exchange rows, gradient and field terms
    double2 Pe = cz(), p1v = cz(), p0v = cz();
    float2 G = fmk(0.f, 0.f);
    if (valid) {
      // stages 1-3: the FP32 stage input feeds the exchange rows as it is
      const float2 pin = S.sPin[tid];
      Pe = STAGE == 0 ? S.sP0[tid] : to_d(pin);
      if (STAGE >= 1) p1v = S.sP1[tid];
      if (STAGE == 1 || STAGE == 2) p0v = S.sP0[tid];
      if (a.z)
        for (int c = 0; c < a.w; c += 4) {
          const float4 g = ldv<float4>(&M.G[c]);
          G = fadd(G, fscale(S.sG[c * NTHR + tid], g.x));
          if (c + 1 < a.w) G = fadd(G, fscale(S.sG[(c + 1) * NTHR + tid], g.y));
          if (c + 2 < a.w) G = fadd(G, fscale(S.sG[(c + 2) * NTHR + tid], g.z));
          if (c + 3 < a.w) G = fadd(G, fscale(S.sG[(c + 3) * NTHR + tid], g.w));
        }
      const int4 b = ldv<int4>(&M.nch);  // nch, n1, n2, ncomp
      const int oij = i * RS + j * KT + kl, oji = j * RS + i * KT + kl;
      const float2 pc = STAGE == 0 ? to_f(Pe) : pin;
      xP[oij] = pc;
      xP[oji] = fconj(pc);
      const int w = (i < b.x) != (j < b.x);
      const float2 h0 = S.sH[tid];
      float2 hu = h0, hl = fconj(h0);
      double ed = i == j ? S.sHii[tid] : 0.;
      for (int c = 0; c < b.w; c++) {
        const float2 ef = ldv<float2>(&M.Ef[c][0]);  // pump, probe / 2
        const float2 d = S.sD[c * NTHR + tid];
        const float ew = w ? ef.y : ef.x;
        hu = fadd(hu, fscale(d, ew));
        hl = fadd(hl, fscale(d, ew));
        if (i == j) ed += (double)d.x * M.E[c][0];
      }
      if (i == j) {
        xEd[i * KT + kl] = ed;
        hu = hl = fmk(0.f, 0.f);
      }
      for (int c = 0; c < b.w; c++) G = fadd(G, fscale(S.sW[c * NTHR + tid], M.Ef[c][0]));
      xH[oij] = hu;
      xH[oji] = hl;
    }
    // ---- record of the next tile when its instance differs (warp 0, one tile ahead)
    const bool more = t + 1 < t1;
    const bool newrun = more && nxt.inst != cur.inst;
    const int msn = newrun ? (ms == 2 ? 0 : ms + 1) : ms;
    if (newrun && warp == 0) pipe_meta<N, STAGE>(S.meta[msn], v, nxt.inst, parity, lane);
    __syncthreads();
    // ---- copies of the next tile, in flight during this tile's commutator
    if (more) {
      pipe_issue<N, KT, STAGE>(S, S.meta[msn], nxt.k0, nxt.interior, tid, kl, e, i, j);
      cp_async_commit();
    }
    const Tile after = t + 2 < t1 ? v.tiles[t + 2] : nxt;
    if (CB) {
      // C = P H~^T in register blocks: C_rc = sum_l P_rl H~_cl (rows of the
      // exchange matrices), BR x BC entries per thread, then beta_ij = C_ij -
      // conj(C_ji) below. Block (rb, cb) holds rows rb + x N/BR and columns
      // cb + y N/BC, so the blocks of one warp read consecutive rows (the
      // padded row stride puts them on different banks).
      constexpr int BR = CBlk<N, CB>::BR, BC = CBlk<N, CB>::BC, NBC = N / BC, NBR = N / BR;
      static_assert(KT * CBlk<N, CB>::NB <= NTHR, "every block of C needs a thread");
      if (a.x && tid < KT * CBlk<N, CB>::NB) {
        const int kc = tid % KT, blk = tid / KT;
        const int r0 = blk / NBC, c0 = blk % NBC;
        float2 acc[BR][BC];
#pragma unroll
        for (int x = 0; x < BR; x++)
#pragma unroll
          for (int y = 0; y < BC; y++) acc[x][y] = fmk(0.f, 0.f);
#pragma unroll
        for (int l = 0; l < N; l++) {
          float2 pr[BR], hc[BC];
#pragma unroll
          for (int x = 0; x < BR; x++) pr[x] = xP[(r0 + x * NBR) * RS + l * KT + kc];
#pragma unroll
          for (int y = 0; y < BC; y++) hc[y] = xH[(c0 + y * NBC) * RS + l * KT + kc];
#pragma unroll
          for (int x = 0; x < BR; x++)
#pragma unroll
            for (int y = 0; y < BC; y++) {
              acc[x][y].x = fmaf(pr[x].x, hc[y].x, acc[x][y].x);
              acc[x][y].x = fmaf(-pr[x].y, hc[y].y, acc[x][y].x);
              acc[x][y].y = fmaf(pr[x].x, hc[y].y, acc[x][y].y);
              acc[x][y].y = fmaf(pr[x].y, hc[y].x, acc[x][y].y);
            }
        }
#pragma unroll
        for (int x = 0; x < BR; x++)
#pragma unroll
          for (int y = 0; y < BC; y++) S.xC[(r0 + x * NBR) * RS + (c0 + y * NBC) * KT + kc] = acc[x][y];
      }
      __syncthreads();
    }
    if (valid) {
      // -i[H~, rho - rho_eq] in the reference's transposed convention
      // (headers/RungeKutta.h:158-208), as k_bstage
      const float2* Hi = xH + i * RS + kl;
      const float2* Hj = xH + j * RS + kl;
      const float2* Pi = xP + i * RS + kl;
      const float2* Pj = xP + j * RS + kl;
      // sum_l H~_jl P_il - conj(H~_il P_jl) in eight partial sums, as k_bstage
      float ax[2] = {0.f, 0.f}, ay[2] = {0.f, 0.f}, bx[2] = {0.f, 0.f}, by[2] = {0.f, 0.f};
#pragma unroll
      for (int l = 0; l < (CB ? 0 : N); l++) {
        const int q = l & 1;
        const float2 hj = Hj[l * KT], pi = Pi[l * KT], hi = Hi[l * KT], pj = Pj[l * KT];
        ax[q] = fmaf(hj.x, pi.x, ax[q]);
        ax[q] = fmaf(-hj.y, pi.y, ax[q]);
        ay[q] = fmaf(hj.x, pi.y, ay[q]);
        ay[q] = fmaf(hj.y, pi.x, ay[q]);
        bx[q] = fmaf(hi.x, pj.x, bx[q]);
        bx[q] = fmaf(-hi.y, pj.y, bx[q]);
        by[q] = fmaf(hi.x, pj.y, by[q]);
        by[q] = fmaf(hi.y, pj.x, by[q]);
      }
      float2 beta = fmk((ax[0] + ax[1]) - (bx[0] + bx[1]), (ay[0] + ay[1]) + (by[0] + by[1]));
      if (CB) {
        const float2 cij = S.xC[i * RS + j * KT + kl], cji = S.xC[j * RS + i * KT + kl];
        beta = fmk(cij.x - cji.x, cij.y + cji.y);
      }
      float2 vv = fmi(beta);
      vv = fadd(vv, G);
      double2 d = to_d(vv);
      const double dE = xEd[j * KT + kl] - xEd[i * KT + kl];
      d = cadd(d, cmi(cscale(Pe, dE)));
      if (i == j) d.y = 0;
      const double dt = M.dt, dt6 = M.dt6, dt3 = M.dt3, dt2 = dt / 2.0;
      const int o = e * a.y + cur.k0 + kl;
      const ulonglong2 pw = ldv<ulonglong2>(&M.Hdiag);  // Hdiag, dst
      float2* dst = (float2*)pw.y;
      if (STAGE == 0) {
        M.P1[o] = cadd(Pe, cscale(d, dt6));
        dst[o] = to_f(cadd(Pe, cscale(d, dt2)));
      } else if (STAGE == 1) {
        M.P1[o] = cadd(p1v, cscale(d, dt3));
        dst[o] = to_f(cadd(p0v, cscale(d, dt2)));
      } else if (STAGE == 2) {
        M.P1[o] = cadd(p1v, cscale(d, dt3));
        dst[o] = to_f(cadd(p0v, cscale(d, dt)));
      } else {
        const double2 pn = cadd(p1v, cscale(d, dt6));
        const_cast<double2*>(M.P0)[o] = pn;
        dst[o] = to_f(pn);
      }
    }
    cur = nxt;
    nxt = after;
    ms = msn;
  }
  cp_async_wait_all();
}

// (the dynamic shared-memory limit of the four kernels is raised by
// stage_grid_pipe on the batch's device before the first launch)
template <int N, int KT, int STAGE, int CB>
cudaError_t pipe_launch(const View& v, int parity, int nsel, int ncomp, int grid, cudaStream_t s) {
  constexpr int NTHR = PipeCarve<N, KT>::NTHR;
  k_bpipe<N, KT, STAGE, CB><<<grid, NTHR, PipeCarve<N, KT>::bytes(nsel, ncomp, CB), s>>>(v, parity, nsel, ncomp);
  return cudaGetLastError();
}

template <int N, int KT, int CB>
cudaError_t pipe_stage(const View& v, int stage, int parity, int nsel, int ncomp, int grid, cudaStream_t s) {
  switch (stage) {
    case 0: return pipe_launch<N, KT, 0, CB>(v, parity, nsel, ncomp, grid, s);
    case 1: return pipe_launch<N, KT, 1, CB>(v, parity, nsel, ncomp, grid, s);
    case 2: return pipe_launch<N, KT, 2, CB>(v, parity, nsel, ncomp, grid, s);
    default: return pipe_launch<N, KT, 3, CB>(v, parity, nsel, ncomp, grid, s);
  }
}

template <int N, int KT, int CB>
int pipe_grid_n(int nsel, int ncomp) {
  constexpr int NTHR = PipeCarve<N, KT>::NTHR;
  const size_t smem = PipeCarve<N, KT>::bytes(nsel, ncomp, CB);
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(k_bpipe<N, KT, 0, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_bpipe<N, KT, 1, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_bpipe<N, KT, 2, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_bpipe<N, KT, 3, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bpipe<N, KT, 0, CB>, NTHR, smem) != cudaSuccess) return 0;
  return sms * per;
}

#define EDUS_PIPE_CLASSES(X) X(2, 32) X(3, 32) X(4, 16) X(5, 16) X(8, 8) X(16, 2)
// classes with the blocked commutator (register profiles 4 and 5)
#define EDUS_PIPE_CB_CLASSES(X) X(8, 8) X(8, 16) X(16, 2) X(16, 4)

}  // namespace

bool pipe_supported(int N, int kt, int cb) {
  if (cb < 0 || cb > 2) return false;
#define X(n, k) \
  if (N == n && kt == k) return true;
  if (cb) {
    EDUS_PIPE_CB_CLASSES(X)
  } else {
    EDUS_PIPE_CLASSES(X)
  }
#undef X
  return false;
}

cudaError_t launch_stage_pipe(int N, int kt, int cb, const View& v, int stage, int parity, int nsel, int ncomp, int grid,
                              cudaStream_t s) {
#define X(n, k) \
  if (N == n && kt == k) return pipe_stage<n, k, 0>(v, stage, parity, nsel, ncomp, grid, s);
#define Y(n, k) \
  if (N == n && kt == k) return pipe_stage<n, k, 1>(v, stage, parity, nsel, ncomp, grid, s);
#define Z(n, k) \
  if (N == n && kt == k) return pipe_stage<n, k, 2>(v, stage, parity, nsel, ncomp, grid, s);
  if (cb == 2) {
    EDUS_PIPE_CB_CLASSES(Z)
  } else if (cb) {
    EDUS_PIPE_CB_CLASSES(Y)
  } else {
    EDUS_PIPE_CLASSES(X)
  }
#undef X
#undef Y
#undef Z
  return cudaErrorInvalidValue;
}

int stage_grid_pipe(int N, int kt, int cb, int nsel, int ncomp) {
#define X(n, k) \
  if (N == n && kt == k) return pipe_grid_n<n, k, 0>(nsel, ncomp);
#define Y(n, k) \
  if (N == n && kt == k) return pipe_grid_n<n, k, 1>(nsel, ncomp);
#define Z(n, k) \
  if (N == n && kt == k) return pipe_grid_n<n, k, 2>(nsel, ncomp);
  if (cb == 2) {
    EDUS_PIPE_CB_CLASSES(Z)
  } else if (cb) {
    EDUS_PIPE_CB_CLASSES(Y)
  } else {
    EDUS_PIPE_CLASSES(X)
  }
#undef X
#undef Y
#undef Z
  return 0;
}

}  // namespace batch
}  // namespace edus
