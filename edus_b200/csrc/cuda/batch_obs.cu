// batch_obs.cu — observables of the batch engine at the output instants of
// its instances (headers/Observables_MPI.h:217-484,559-598,668-775), and the
// step-counter advance of every instance of a class.
//
// Per launch (one per time step and class): the step counters of the class's
// instances advance (one thread per instance, from the class's instance
// table); every block then finds the instances due at this step (it %
// it_resolution == 0) from the same table and walks only their tiles. A tile
// unit of work is ObsUnit<N> consecutive k points of one instance, taken KO
// k points at a time with one thread per (k point, full-matrix entry (b, l)):
//   J1_x = sum_e P_e dH/dk^x_e (+ the mirrored lower element),
//   J2_x = sum_{b,l} conj(D^x_bl) Q_bl with Q = P^T H (Q_bl = sum_a P_ab H_al,
//          formed once for the three components),
//   pop_b += Re conj(U_bl) sum_j P_lj U_bj (band b, row l of U^+ P U),
// in FP64. Each unit writes one partial; the last unit of an instance to
// finish reduces its partials in unit order, so an instance's record depends
// only on its own k points.
#include <type_traits>

#include "batch.cuh"

namespace edus {
namespace batch {
namespace {

constexpr int opad32(int x) { return (x + 31) / 32 * 32; }

template <int N>
__device__ __forceinline__ int tri_up(int i, int j) { return i * N - (i * (i - 1)) / 2 + (j - i); }

template <class To, class From>
__device__ __forceinline__ To ocvt(From a) {
  To r;
  r.x = a.x;
  r.y = a.y;
  return r;
}

// Tile partials are stored field-major: part[f][tile], f = 0..kPartF-1:
// populations 0..kMaxBands-1, then for x = 0..2 (J1 re, J1 im, J2 re, J2 im,
// TA re, TA im, polarisation re, im), then max |P - P_eq| and min P.
constexpr int kAccF = 26;                 // fields after the populations
constexpr int kPartF = kMaxBands + kAccF;
constexpr int kFJ = kMaxBands;            // first current field

__device__ __forceinline__ double warp_sum(double x) {
  for (int s = 16; s > 0; s >>= 1) x += __shfl_xor_sync(0xffffffffu, x, s);
  return x;
}
__device__ __forceinline__ double warp_max(double x) {
  for (int s = 16; s > 0; s >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, s));
  return x;
}
__device__ __forceinline__ double warp_min(double x) {
  for (int s = 16; s > 0; s >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, s));
  return x;
}

// What one thread accumulates over the k points of a tile.
struct Acc {
  double pop;                 // thread (k, c), c < N: band c
  double2 J1[3], J2[3], TA[3], PL[3];
  double pmax, pmin;
};

// Value v (0 .. N+25) of a thread's accumulator in the flat field order; pop
// values sit at their band c = q.
template <int N>
__device__ __forceinline__ double acc_val(const Acc& a, int v, int q) {
  if (v < N) return q == v ? a.pop : 0.;
  const int r = v - N;
  if (r < 24) {
    const int x = r / 8, m = r % 8;
    const double2 z = m < 2 ? a.J1[x] : (m < 4 ? a.J2[x] : (m < 6 ? a.TA[x] : a.PL[x]));
    return (m & 1) ? z.y : z.x;
  }
  return r == 24 ? a.pmax : a.pmin;
}
template <int N>
__host__ __device__ constexpr int field_of(int v) { return v < N ? v : kFJ + (v - N); }

// Block reduction of the accumulators into the tile's partial, in a fixed
// order (warp butterflies, then warps in index order); field f of the tile
// goes to part[f * stride + t].
template <int N, int NW>
__device__ __forceinline__ void tile_reduce(const Acc& a, int q, double (*sW)[N + kAccF], double* part, size_t stride, int t) {
  const int lane = threadIdx.x % 32, w = threadIdx.x / 32;
#pragma unroll
  for (int v = 0; v < N + kAccF; v++) {
    const double x = acc_val<N>(a, v, q);
    const double r = v == N + 24 ? warp_max(x) : (v == N + 25 ? warp_min(x) : warp_sum(x));
    if (lane == 0) sW[w][v] = r;
  }
  __syncthreads();
  const int v = threadIdx.x;
  if (v < N + kAccF) {
    double r = v == N + 25 ? 1.0 : 0.;
    for (int ww = 0; ww < NW; ww++) {
      const double y = sW[ww][v];
      r = v == N + 24 ? fmax(r, y) : (v == N + 25 ? fmin(r, y) : r + y);
    }
    part[(size_t)field_of<N>(v) * stride + t] = r;
  }
}

// k points per sub-tile (one thread per k point and full-matrix entry)
template <int N>
struct ObsK {
  static constexpr int v = N <= 2 ? 32 : (N <= 4 ? 16 : (N <= 5 ? 8 : (N <= 8 ? 4 : 1)));
};
// k points per unit (one partial each)
template <int N>
struct ObsUnit {
  static constexpr int v = N >= 16 ? 64 : 128;
};

template <int N, bool MIX>
__global__ void __launch_bounds__(opad32(ObsK<N>::v* N* N), 3) k_bobs(View v, int parity) {
  constexpr int KO = ObsK<N>::v;
  constexpr int NN = N * N, NT = N * (N + 1) / 2;
  constexpr int NTHR = opad32(KO * NN), NW = NTHR / 32;
  using S = typename std::conditional<MIX, float2, double2>::type;
  __shared__ double2 sP[NN][KO];
  __shared__ double2 sH[NN][KO];
  __shared__ double2 sD[3][NN][KO];
  __shared__ double2 sU[NN][KO];
  __shared__ double sTerm[NN][KO];  // population terms
  __shared__ double sW[NW][N + kAccF];
  __shared__ double sT[N + kAccF];  // the instance's totals (last tile)
  __shared__ int sScan[NTHR];
  __shared__ bool sLast;
  extern __shared__ int sPre[];  // [ninst + 1] first due tile of each instance
  const int tid = threadIdx.x;
  const int kl = tid % KO, q = tid / KO;
  const bool lane_ok = q < NN;
  const int b = lane_ok ? q / N : 0, l = lane_ok ? q % N : 0;
  const int* itp = parity ? v.it[1] : v.it[0];
  int* itn = parity ? v.it[0] : v.it[1];
  const int nci = *v.ninst;
  // step counters (it[parity] is only read in this launch)
  for (int x = blockIdx.x * NTHR + tid; x < nci; x += gridDim.x * NTHR) {
    const ClassInst c = v.cinst[x];
    const int it = itp[c.slot];
    itn[c.slot] = it <= c.itfi ? it + 1 : it;
  }
  // tiles due at this step: exclusive prefix sums over the instance table
  auto due = [&](int x) {
    const ClassInst c = v.cinst[x];
    const int it = itp[c.slot];
    return (it >= 0 && it <= c.itfi && it % c.res == 0) ? c.nunits : 0;
  };
  const int per = (nci + NTHR - 1) / NTHR;
  const int c0 = min(tid * per, nci), c1 = min(c0 + per, nci);
  int mine = 0;
  for (int x = c0; x < c1; x++) mine += due(x);
  sScan[tid] = mine;
  __syncthreads();
  for (int off = 1; off < NTHR; off <<= 1) {
    const int add = tid >= off ? sScan[tid - off] : 0;
    __syncthreads();
    sScan[tid] += add;
    __syncthreads();
  }
  int run = sScan[tid] - mine;
  for (int x = c0; x < c1; x++) {
    sPre[x] = run;
    run += due(x);
  }
  if (tid == NTHR - 1) sPre[nci] = sScan[NTHR - 1];
  __syncthreads();
  const int total = sPre[nci];

  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    // instance of due tile w: the last x with sPre[x] <= w (instances without
    // due tiles have sPre[x] == sPre[x + 1])
    int lo = 0, hi = nci - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (sPre[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const ClassInst ci = v.cinst[lo];
    const int u_in = w - sPre[lo];  // unit of the instance
    const int slot = ci.slot;
    const Inst* I = v.insts + slot;
    const int it = itp[slot];
    const int nk = I->nk, nch = I->nch;
    const S* H = reinterpret_cast<const S*>(I->H);
    const S* D = reinterpret_cast<const S*>(I->D);
    const S* GE = reinterpret_cast<const S*>(I->GE);
    const S* U = reinterpret_cast<const S*>(I->U);
    const bool cur = I->want_current, tabs = I->want_tabs;
    Acc my;
    my.pop = 0.;
    for (int x = 0; x < 3; x++) my.J1[x] = my.J2[x] = my.TA[x] = my.PL[x] = cz();
    my.pmax = 0.;
    my.pmin = 1.;
    constexpr int UK = ObsUnit<N>::v;
    const int k0t = u_in * UK, kend = min(k0t + UK, nk);
    for (int k0 = k0t; k0 < kend; k0 += KO) {
      const int k = k0 + kl;
      const bool valid = lane_ok && k < kend;
      if (lane_ok) {
        double2 p = cz(), h = cz(), u = cz(), d[3] = {cz(), cz(), cz()};
        if (valid) {
          const bool lower = b > l;
          const int e = lower ? tri_up<N>(l, b) : tri_up<N>(b, l);
          const size_t o = (size_t)e * nk + k;
          p = MIX ? cadd(I->P0[o], I->Peq[o]) : I->P0[o];
          h = ocvt<double2>(H[o]);
          if (lower) {
            p = cconj(p);
            h = cconj(h);
          }
          for (int x = 0; x < 3; x++) d[x] = ocvt<double2>(D[(size_t)x * NT * nk + o]);  // symmetric
          u = ocvt<double2>(U[(size_t)q * nk + k]);
        }
        sP[q][kl] = p;
        sH[q][kl] = h;
        for (int x = 0; x < 3; x++) sD[x][q][kl] = d[x];
        sU[q][kl] = u;
      }
      __syncthreads();
      if (valid) {
        if (b <= l) {
          const int e = tri_up<N>(b, l);
          const double2 pe = sP[q][kl];
          if (cur) {
            const size_t o = (size_t)e * nk + k;
            for (int x = 0; x < 3; x++) {
              const double2 ge = ocvt<double2>(GE[(size_t)x * NT * nk + o]);
              my.J1[x] = cadd(my.J1[x], cmul(pe, ge));
              if (b != l) my.J1[x] = cadd(my.J1[x], cmul(cconj(pe), cconj(ge)));
            }
          }
          if (tabs && b < nch && l >= nch)
            for (int x = 0; x < 3; x++) my.TA[x] = csub(my.TA[x], cmul(cscale(sD[x][q][kl], 2.), pe));
        }
        // polarisation: Tr(D_x rho) = sum_bl D^x_bl P_bl (P_bl = rho_lb), this thread's entry
        for (int x = 0; x < 3; x++) my.PL[x] = cadd(my.PL[x], cmul(sD[x][q][kl], sP[q][kl]));
        if (cur) {
          // Q_bl = sum_a P_ab H_al; J2_x += Q_bl conj(D^x_bl)
          double2 Q = cz();
#pragma unroll
          for (int a = 0; a < N; a++) Q = cadd(Q, cmul(sP[a * N + b][kl], sH[a * N + l][kl]));
          for (int x = 0; x < 3; x++) my.J2[x] = cadd(my.J2[x], cmulc(Q, sD[x][q][kl]));
        }
        {
          // population of band b in the model eigenbasis, sum_l conj(U_bl) sum_j P_lj U_bj:
          // this thread's term l (summed over l below, in l order)
          double2 m = cz();
#pragma unroll
          for (int jj = 0; jj < N; jj++) m = cadd(m, cmul(sP[l * N + jj][kl], sU[b * N + jj][kl]));
          sTerm[q][kl] = cmul(cconj(sU[q][kl]), m).x;
        }
      }
      __syncthreads();
      if (valid && l == 0) {
        double Pk = 0.;
        for (int ll = 0; ll < N; ll++) Pk += sTerm[b * N + ll][kl];
        my.pop += Pk;
        if (b < I->nbands) {
          my.pmax = fmax(my.pmax, fabs(1. - Pk));
          my.pmin = fmin(my.pmin, 1. - Pk);
        } else {
          my.pmax = fmax(my.pmax, fabs(Pk));
          my.pmin = fmin(my.pmin, Pk);
        }
      }
    }
    double* part = reinterpret_cast<double*>(I->part);
    const size_t stride = (size_t)I->ntiles;  // the partials are sized per tile, at least one per unit
    const int nunits = ci.nunits;
    tile_reduce<N, NW>(my, b, sW, part, stride, u_in);
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      sLast = atomicAdd(I->done, 1u) == (unsigned)(nunits - 1);
    }
    __syncthreads();
    if (sLast) {
      // last tile of the instance to finish: every field summed over the tiles
      // in a fixed order (lane-strided sums, then a warp butterfly); partials of
      // other blocks are read past L1
      __threadfence();
      const int lane = tid % 32, wid = tid / 32;
      for (int v = wid; v < N + kAccF; v += NW) {
        const double* row = part + (size_t)field_of<N>(v) * stride;
        double r = v == N + 25 ? 1.0 : 0.;
        for (int x = lane; x < nunits; x += 32) {
          const double y = __ldcg(row + x);
          r = v == N + 24 ? fmax(r, y) : (v == N + 25 ? fmin(r, y) : r + y);
        }
        r = v == N + 24 ? warp_max(r) : (v == N + 25 ? warp_min(r) : warp_sum(r));
        if (lane == 0) sT[v] = r;
      }
      __syncthreads();
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
          double val = sT[c] * inv;
          trace += val;
          if (c < I->nbands) val = 1.0 - val;
          rec.pop[c] = val;
          if (val > ncd) ncd = val;
        }
        for (int x = 0; x < 3; x++) {
          const double* f = sT + N + 8 * x;  // J1 re, im, J2 re, im, TA re, im, polarisation re, im
          rec.J1[2 * x] = f[0] * I->scaleJ;
          rec.J1[2 * x + 1] = f[1] * I->scaleJ;
          rec.J2[x] = -2. * (f[3] * I->scaleJ);
          rec.tabs[2 * x] = f[4] * I->scaleTA * inv;
          rec.tabs[2 * x + 1] = f[5] * I->scaleTA * inv;
          rec.pol[2 * x] = f[6] * inv;
          rec.pol[2 * x + 1] = f[7] * inv;
        }
        rec.trace_dev = trace;
        rec.p_cond_max = sT[N + 24];
        rec.p_min = sT[N + 25];
        rec.n_cond = ncd;
        I->log[it / I->res] = rec;
        *I->done = 0u;
      }
    }
    __syncthreads();
  }
}

template <int N, bool MIX>
cudaError_t obs_n(const View& v, int parity, int kt, int max_inst, int grid, cudaStream_t s) {
  constexpr int NTHR = opad32(ObsK<N>::v * N * N);
  (void)kt;
  k_bobs<N, MIX><<<grid, NTHR, (size_t)(max_inst + 1) * sizeof(int), s>>>(v, parity);
  return cudaGetLastError();
}

template <int N, bool MIX>
int obs_grid_n(int max_inst) {
  constexpr int NTHR = opad32(ObsK<N>::v * N * N);
  const size_t smem = (size_t)(max_inst + 1) * sizeof(int);
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(k_bobs<N, MIX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bobs<N, MIX>, NTHR, smem) != cudaSuccess) return 0;
  return sms * per;
}

}  // namespace

cudaError_t launch_obs(int N, int kt, bool mixed, const View& v, int parity, int max_inst, int grid, cudaStream_t s) {
  switch (N) {
#define X(n) \
  case n: return mixed ? obs_n<n, true>(v, parity, kt, max_inst, grid, s) : obs_n<n, false>(v, parity, kt, max_inst, grid, s);
    X(2) X(3) X(4) X(5) X(8) X(16)
#undef X
    default: return cudaErrorInvalidValue;
  }
}

int obs_grid(int N, bool mixed, int max_inst) {
  switch (N) {
#define X(n) \
  case n: return mixed ? obs_grid_n<n, true>(max_inst) : obs_grid_n<n, false>(max_inst);
    X(2) X(3) X(4) X(5) X(8) X(16)
#undef X
    default: return 0;
  }
}

size_t obs_part_bytes() { return kPartF * sizeof(double); }

int obs_unit(int N) {
  switch (N) {
#define X(n) \
  case n: return ObsUnit<n>::v;
    X(2) X(3) X(4) X(5) X(8) X(16)
#undef X
    default: return 0;
  }
}

}  // namespace batch
}  // namespace edus
