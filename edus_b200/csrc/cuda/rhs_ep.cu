// rhs_ep.cu — element-parallel FP64 RHS + stage update (sm_100a).
//
// One thread per (k point, upper-triangle element e = (i, j)); a block holds
// KT k points x NT elements. Each thread loads its own rho_e, H_e, D_e planes
// (coalesced over k), adds its Coulomb mean-field element and its k-gradient
// element, publishes rho and H~ through shared memory, then evaluates its
// commutator element -i[H~ + E.D, rho]_ij (headers/RungeKutta.h:158-212), RWA
// (:209), dissipation (:219-254), hermitizes (:283-294) and applies the
// integrator's stage update (headers/RungeKutta.h:301-355,
// Source_Main/Linear_Multistep_ODE_solvers.cpp:82-94,
// Source_Main/Taylor_DE_solver_deriv_Polynom.cpp:142-177). Compared with a
// thread per k this gives NT times the parallelism for the small grids of the
// reference's workloads, where one solve has only 10^3-10^4 k points.
#include "dev.cuh"
#include "dyn.cuh"
#include "kernels.hpp"

namespace edus {

template <int N>
struct TriEP {
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

// DYN: the stage scalars come from the adaptive step's device copy (a.dyn);
// a separate instantiation so the constant-step kernel keeps its registers.
template <int N, int KT, bool DYN>
__global__ void __launch_bounds__(KT* TriEP<N>::NT) k_rhs_ep(DevTables tb, const DevConsts* __restrict__ cst, StageArgs a) {
  constexpr int NT = TriEP<N>::NT;
  __shared__ double2 sP[NT][KT];
  __shared__ double2 sHu[NT][KT];  // H~_ij, i <= j
  __shared__ double2 sHl[NT][KT];  // H~_ji, i <= j (D is symmetric, H Hermitian)
  extern __shared__ double2 dyn[];  // Coulomb row tables: h rows [nrows][2][ncut][NT], trig [2][ncut][KT]
  const int kl = threadIdx.x, e = threadIdx.y;
  const int k0 = blockIdx.x * KT;
  const int k = k0 + kl;
  const int nk = tb.nk;
  const bool valid = k < nk;
  const int nch = tb.nch;
  int i, j;
  TriEP<N>::ij(e, i, j);
  __shared__ unsigned long long bar;
  const bool staged = tb.h && a.stage_rows > 0;
  if (staged) {
    // the k2 trig values do not depend on the previous kernel: gathered before
    // the wait; the inverse-transform rows this block touches (written by the
    // previous kernel) then arrive by one bulk copy while the threads load
    // their own planes
    const int n2 = tb.n2, nc = tb.ncut;
    const int tid = threadIdx.y * KT + threadIdx.x, nthr = KT * NT;
    double* ts = reinterpret_cast<double*>(dyn + a.stage_rows * 2 * nc * NT);
#pragma unroll 4
    for (int t = tid; t < 2 * nc * KT; t += nthr) {
      const int q = t % KT, cm = t / KT, cs = cm / nc, m = cm - cs * nc;
      const int kk = min(k0 + q, nk - 1);
      const int i2 = kk - (kk / n2) * n2;
      ts[t] = __ldg((cs == 0 ? tb.t2c : tb.t2s) + m * n2 + i2);
    }
    pdl_wait();
    if (DYN && !a.dyn->active) return;  // the adaptive run has ended (uniform over the grid)
    if (tid == 0) {
      const int r0 = k0 / n2;
      const int r1 = (min(k0 + KT, nk) - 1) / n2;
      const uint32_t hbytes = (uint32_t)((r1 - r0 + 1) * 2 * nc * NT * sizeof(double2));
      mbar_init(&bar, 1);
      mbar_expect_tx(&bar, hbytes);
      bulk_g2s(dyn, tb.h + (size_t)r0 * 2 * nc * NT, hbytes, &bar);
    }
  } else {
    pdl_wait();
    if (DYN && !a.dyn->active) return;
  }
  // stage scalars: kernel arguments, or the adaptive step's device copy
  const DynStep* dy = DYN ? a.dyn : nullptr;
  double ef0[3], ef1[3];  // pump, probe
#pragma unroll
  for (int x = 0; x < 3; x++) {
    ef0[x] = dy ? dy->EF[a.dyn_field][0][x] : a.EF[0][x];
    ef1[x] = dy ? dy->EF[a.dyn_field][1][x] : a.EF[1][x];
  }
  const int e_non0 = dy ? dy->e_non0 : a.e_non0;
  const double c1 = dy ? dy->c[a.dyn_stage][0] : a.c1;
  const double c2 = dy ? dy->c[a.dyn_stage][1] : a.c2;
  const double dtv = dy ? dy->dt : a.dt;
  const double pcn = dy ? (*dy->pcmax + *dy->ncond) : a.pcond_plus_ncond;
  double2 Pe = cz(), He = cz(), G = cz();
  double2 De[3] = {cz(), cz(), cz()};
  if (valid) {
    Pe = a.src[(size_t)e * nk + k];
    He = tb.H[(size_t)e * nk + k];
#pragma unroll
    for (int x = 0; x < 3; x++) De[x] = tb.D[(size_t)(x * NT + e) * nk + k];
  }
  if (staged) {
    __syncthreads();  // trig table + barrier init visible to all threads
    mbar_wait(&bar, 0, tb.err);
  }
  if (valid) {
    if (tb.h && a.xw) {
      // diagonal basis: the term of k_coulomb_xw (screened, rotated back)
      double2 X = a.xw[(size_t)e * nk + k];
      if (i == j) {
        X.y = 0.;
        double eh = 0.;
#pragma unroll
        for (int jj = 0; jj < N; jj++) eh += tb.fdiag[jj].x * cst->VH[i * N + jj];
        eh -= cst->EH0[i];
        He = cadd(He, X);
        He.x += eh;
      } else {
        He = cadd(He, X);
      }
      if (a.hr_out) a.hr_out[(size_t)e * nk + k] = He;
    } else if (tb.h) {
      // X_e(k) = conj(-sum_n hc(i1,n,e) cos(2 pi n k2) + hs(i1,n,e) sin(2 pi n k2))
      const int n2 = tb.n2;
      const int i1 = k / n2, i2 = k - i1 * n2;
      const int nc = tb.ncut;
      double yx = 0., yy = 0.;
      if (a.stage_rows > 0) {
        const double2* hrow = dyn + (size_t)(i1 - k0 / n2) * 2 * nc * NT + e;
        const double* ts = reinterpret_cast<const double*>(dyn + a.stage_rows * 2 * nc * NT);
#pragma unroll 4
        for (int m = 0; m < nc; m++) {
          const double cn = ts[m * KT + kl], sn = ts[(nc + m) * KT + kl];
          const double2 c = hrow[(size_t)m * NT], s = hrow[(size_t)(nc + m) * NT];
          yx += c.x * cn + s.x * sn;
          yy += c.y * cn + s.y * sn;
        }
      } else {
        const double2* hrow = tb.h + (size_t)i1 * 2 * nc * NT + e;
#pragma unroll 4
        for (int m = 0; m < nc; m++) {
          const double cn = tb.t2c[m * n2 + i2], sn = tb.t2s[m * n2 + i2];
          const double2 c = hrow[(size_t)m * NT], s = hrow[(size_t)(nc + m) * NT];
          yx += c.x * cn + s.x * sn;
          yy += c.y * cn + s.y * sn;
        }
      }
      double2 X = cmk(-yx, yy);
      if (*tb.ncond > 1e-20) {
        const double2 dP = csub(Pe, tb.PW0[(size_t)e * nk + k]);
        X = csub(X, cmul(cst->screen[e], cconj(dP)));
      }
      if (i == j) {
        X.y = 0.;
        double eh = 0.;
#pragma unroll
        for (int jj = 0; jj < N; jj++) eh += tb.fdiag[jj].x * cst->VH[i * N + jj];
        eh -= cst->EH0[i];
        He = cadd(He, X);
        He.x += eh;
      } else {
        He = cadd(He, X);
      }
      if (a.hr_out) a.hr_out[(size_t)e * nk + k] = He;
    }
    if (e_non0) {
      // sum_b (w_b E_pump . b) rho_e(k + b)
#pragma unroll 6
      for (int b = 0; b < tb.nnb; b++) {
        const int kb = tb.nbr[(size_t)b * nk + k];
        const double2 pn = a.src[(size_t)e * nk + kb];
        const double f0 = cst->wb[b] * ef0[0] * cst->bvec[b][0];
        const double f1 = cst->wb[b] * ef0[1] * cst->bvec[b][1];
        const double f2 = cst->wb[b] * ef0[2] * cst->bvec[b][2];
        G = cadd(G, cscale(pn, f0));
        G = cadd(G, cscale(pn, f1));
        G = cadd(G, cscale(pn, f2));
      }
    }
  }
  {
    // H~ = H + E^w . D with w = probe when exactly one of (i, j) is a core band
    // (headers/RungeKutta.h:158-208); the lower entry uses conj(H) and the same D
    // (symmetric dipoles) or conj(D) (Hermitian dipoles)
    const int w = (i < nch) != (j < nch);
    double2 hu = He, hl = cconj(He);
    const bool herm = tb.herm_dip != 0;
#pragma unroll
    for (int x = 0; x < 3; x++) {
      const double f = w ? ef1[x] : ef0[x];
      hu = cadd(hu, cscale(De[x], f));
      hl = cadd(hl, cscale(herm ? cconj(De[x]) : De[x], f));
    }
    sP[e][kl] = Pe;
    sHu[e][kl] = hu;
    sHl[e][kl] = hl;
  }
  __syncthreads();

  double dpmax = 0.;
  if (valid) {
    auto Pf = [&](int r, int c) -> double2 {
      return (r <= c) ? sP[TriEP<N>::idx(r, c)][kl] : cconj(sP[TriEP<N>::idx(c, r)][kl]);
    };
    auto HF = [&](int r, int c) -> double2 {
      return (r <= c) ? sHu[TriEP<N>::idx(r, c)][kl] : sHl[TriEP<N>::idx(c, r)][kl];
    };
    double2 v;
    if (i == j) {
      double2 beta = cz();
#pragma unroll
      for (int l = 0; l < N; l++) beta = cadd(beta, cmul(HF(i, l), Pf(i, l)));
      v = cmk(2. * beta.y, 0.);
    } else {
      double2 beta = cz();
#pragma unroll
      for (int l = 0; l < N; l++) {
        const double2 x = cmul(HF(j, l), Pf(i, l));
        const double2 y = cmul(HF(i, l), Pf(j, l));
        beta = cadd(beta, csub(x, cconj(y)));
      }
      v = cmi(beta);
      if (i < nch && j >= nch) v = cadd(v, cmi(cscale(Pe, -a.wx2)));
    }
    if (tb.n_diss > 0) {
      const double2* U = tb.U;
      auto Ug = [&](int r, int c) -> double2 { return U[(size_t)(r * N + c) * nk + k]; };
      for (int t = 0; t < tb.n_diss; t++) {
        const int ii = cst->diss_i[t], jj = cst->diss_j[t];
        double2 m = cz();
        for (int p = 0; p < N; p++)
          for (int q = 0; q < N; q++) m = cadd(m, cmul(cmulc(Ug(jj, q), Ug(ii, p)), Pf(p, q)));
        const double2 f = cscale(cmulc(cconj(Ug(jj, j)), Ug(i, ii)), cst->T[ii * N + jj]);
        v = csub(v, cmul(f, m));
      }
      double2 tii = cz();
      for (int q = 0; q < tb.nbands; q++) tii = cadd(tii, cscale(cmulc(Ug(q, i), Ug(q, j)), cst->T[q * N + q]));
      v = cadd(v, tii);
    }
    v = cadd(v, G);
    if (i == j) v.y = 0.;
    const size_t o = (size_t)e * nk + k;
    switch (a.op) {
      case OP_PV:
        a.dst[o] = v;
        break;
      case OP_RK_FIRST: {
        if (a.ring) a.ring[(size_t)a.ring_idx[0] * NT * nk + o] = v;
        const double2 b0 = a.base[o];
        a.acc[o] = cadd(b0, cscale(v, c1));
        a.dst[o] = cadd(b0, cscale(v, c2));
      } break;
      case OP_RK_MID: {
        const double2 b0 = a.base[o];
        a.acc[o] = cadd(a.acc[o], cscale(v, c1));
        a.dst[o] = cadd(b0, cscale(v, c2));
      } break;
      case OP_RK_LAST: {
        const double2 nv = cadd(a.acc[o], cscale(v, c1));
        if (a.maxdp && i == j) {
          const double2 old = a.dst[o];
          dpmax = 2 * hypot(old.x - nv.x, old.y - nv.y) / (pcn + hypot(nv.x, nv.y) + 1.0e-7);
        }
        a.dst[o] = nv;
      } break;
      case OP_AB: {
        a.ring[(size_t)a.ring_idx[0] * NT * nk + o] = v;
        double2 d = cz();
        for (int s = 0; s < a.order; s++) {
          const double2 f = (s == 0) ? v : a.ring[(size_t)a.ring_idx[s] * NT * nk + o];
          d = cadd(d, cscale(f, a.coef[s]));
        }
        a.dst[o] = cadd(Pe, cscale(d, dtv));
      } break;
      case OP_TAYLOR: {
        const int TO = a.order, m = TO - 1;
        a.ring[(size_t)a.ring_idx[0] * NT * nk + o] = v;
        double2 dP[kMaxOrder];
        for (int q = 0; q < m; q++) dP[q] = csub(v, a.ring[(size_t)a.ring_idx[q + 1] * NT * nk + o]);
        double2 d = cscale(v, dtv);
        for (int r = 1; r < TO; r++) {
          double2 al = cz();
          for (int q = 0; q < m; q++) al = cadd(al, cscale(dP[q], dy ? dy->tinv[(r - 1) * m + q] : a.tinv[(r - 1) * m + q]));
          const double2 inc = cscale(al, dy ? dy->tpow[r] : a.tpow[r]);
          d = cadd(d, cmk(inc.x / (double)(r + 1), inc.y / (double)(r + 1)));
        }
        const double2 nv = cadd(Pe, d);
        if (a.maxdp && i == j)
          dpmax = 2 * hypot(Pe.x - nv.x, Pe.y - nv.y) / (pcn + hypot(nv.x, nv.y) + 1.0e-7);
        a.dst[o] = nv;
      } break;
    }
  }
  if (a.maxdp) {
    for (int s = 16; s > 0; s >>= 1) dpmax = fmax(dpmax, __shfl_xor_sync(0xffffffffu, dpmax, s));
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0) atomicMax(a.maxdp, (unsigned long long)__double_as_longlong(dpmax));
  }
}

template <int N, int KT>
static cudaError_t launch_ep(const DevTables& tb, const DevConsts* cst, const StageArgs& a, cudaStream_t s) {
  constexpr int NT = TriEP<N>::NT;
  static_assert((KT * NT) % 32 == 0 || KT * NT < 32, "block must be whole warps for the shuffle reduction");
  dim3 block(KT, NT);
  StageArgs b = a;
  size_t dyn = 0;
  b.stage_rows = 0;
  if (tb.h && !a.xw) {
    // rows of the k grid one block of KT consecutive k points can touch
    const int rows = (tb.n2 + KT - 2) / tb.n2 + 1;
    const size_t bytes = sizeof(double2) * ((size_t)rows * 2 * tb.ncut * NT + tb.ncut * KT);
    const size_t static_bytes = sizeof(double2) * 3 * NT * KT;
    if (bytes + static_bytes <= 48 * 1024) {
      b.stage_rows = rows;
      dyn = bytes;
    }
  }
  if (a.dyn) return launch_pdl(k_rhs_ep<N, KT, true>, dim3((tb.nk + KT - 1) / KT), block, dyn, s, tb, cst, b);
  return launch_pdl(k_rhs_ep<N, KT, false>, dim3((tb.nk + KT - 1) / KT), block, dyn, s, tb, cst, b);
}

cudaError_t launch_rhs(const DevTables& tb, const DevConsts* cst, const StageArgs& a, cudaStream_t s) {
  switch (tb.n) {
    case 1: return launch_ep<1, 32>(tb, cst, a, s);
    case 2: return launch_ep<2, 32>(tb, cst, a, s);
    case 3: return launch_ep<3, 32>(tb, cst, a, s);
    case 4: return launch_ep<4, 32>(tb, cst, a, s);
    case 5: return launch_ep<5, 32>(tb, cst, a, s);
    case 8: return launch_ep<8, 16>(tb, cst, a, s);
    case 16: return launch_ep<16, 4>(tb, cst, a, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace edus
