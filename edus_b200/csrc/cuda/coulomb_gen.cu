// coulomb_gen.cu — the Coulomb coefficient generator on the GPU
// (Source_Main/Fourier_Coulomb.cpp:95-500 with headers/Coulomb.h:60-235 and
// headers/integrationWeight.h:5-76).
//
// The reference fits the screened lattice-summed interaction
//   W_ij(q) = sum_G V(|q + G|) exp(i (q + G) . (tau_i - tau_j))
// on the Brillouin zone by a Fourier series in the crystal coordinates
// (qx, qy) of q, the coefficients being Simpson integrals over an N x N grid
// (N = 4999) with a G sum of every reciprocal vector inside G_distance
// (502 657 vectors for the shipped hBN files): 1.25e13 potential evaluations,
// CPU-days there. Here:
//   1. one thread per grid point q sums the G list in the reference's order
//      (G tiles staged through shared memory, shared by the block's q points);
//      V is evaluated with the reference's operation order and correctly
//      rounded sqrt / division, and exp(i (q+G).tau) is taken as
//      exp(i q.tau) exp(i G.tau) with the G phases tabulated once;
//   2. the coefficients A, B, C, D of mode (m, n) are separable sums over the
//      grid, sum_x w_x trig_m(x) [sum_y w_y trig_n(y) W(x, y)]: one pass over
//      the rows, then one over the columns;
//   3. Hartree term: the G sum at q = 0 with V = 0 wherever G0 + G1 < 1e-16
//      (Fourier_Coulomb.cpp:166-214);
//   4. screening constant: on the finer grid (N = 39999) the points with
//      |q| < max(qTF, 0.02) get the unscreened W minus the fitted series,
//      times 1 / N^2 (Fourier_Coulomb.cpp:369-470).
// Files: Output/Coulomb/{A,B,C,D}_coeff<label>.txt, V_Hartree_<label>.txt,
// Screen_const_<label>.txt with label G_num<G>_Ncut<Ncut><labelInput>, in the
// reference's formats, so Read_Coulomb_from_files reads them back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../host/problem.hpp"
#include "dev.cuh"

namespace edus {
namespace cgen {

constexpr int kMaxPairs = 6;     // off-diagonal band pairs (up to 4 bands)
constexpr int kGTile = 256;      // G vectors staged per shared-memory tile
constexpr int kWThreads = 128;   // q points per block

struct Geo {
  double M[3][3];  // crystal -> Cartesian (Coordinate::setcrys)
  int o110;        // sample in xy ("110") instead of yz ("011")
};

struct VPar {
  double qTF, eps_area, r0;
  int rk;       // Rytova-Keldysh form
  int hartree;  // V = 0 where G0 + G1 < 1e-16 (the q = 0 Hartree pass)
};

// Coordinate::setcrys (headers/Coordinate.h:133-150) for crys = (0, c1, c2)
// ("011") or (c1, c2, 0) ("110"), accumulated in the reference's order
// without contraction.
__device__ __forceinline__ void cart_of(const Geo& g, double c1, double c2, double* x) {
  const double a = g.o110 ? c1 : 0.0, b = g.o110 ? c2 : c1, c = g.o110 ? 0.0 : c2;
#pragma unroll
  for (int i = 0; i < 3; i++) x[i] = __dadd_rn(__dadd_rn(__dmul_rn(g.M[i][0], a), __dmul_rn(g.M[i][1], b)), __dmul_rn(g.M[i][2], c));
}

// Coloumb_THh_F (headers/Coulomb.h:60-83) at |k|^2 = q_mod.
__device__ __forceinline__ double coul_v(double q_mod, const VPar& v) {
  const double num = 2 * M_PI;
  const double s1 = __dsqrt_rn(__dadd_rn(q_mod, __dmul_rn(v.qTF, v.qTF)));
  double den = __dmul_rn(v.eps_area, s1);
  if (v.rk) den = __dmul_rn(den, __dadd_rn(__dmul_rn(__dsqrt_rn(q_mod), v.r0), 1.0));
  return __ddiv_rn(num, den);
}

// W at a list of q points (or the N x N grid): out[0][iq] = sum_G V (the
// diagonal), out[1 + p][iq] = exp(i q.tau_p) sum_G V exp(i G.tau_p).
template <int NP>
__global__ void __launch_bounds__(kWThreads) k_wq(Geo g, VPar v, const double* __restrict__ qgrid, int nsum,
                                                  const double2* __restrict__ qlist, long long nq,
                                                  const double2* __restrict__ gcrys, const double2* __restrict__ gph, int ng,
                                                  const double* __restrict__ tau, double2* __restrict__ out) {
  __shared__ double2 sG[kGTile];
  __shared__ double2 sP[kGTile * (NP > 0 ? NP : 1)];
  const long long iq = (long long)blockIdx.x * kWThreads + threadIdx.x;
  const bool act = iq < nq;
  double qx = 0, qy = 0;
  if (act) {
    if (qlist) {
      qx = qlist[iq].x;
      qy = qlist[iq].y;
    } else {
      qx = qgrid[iq / nsum];
      qy = qgrid[iq % nsum];
    }
  }
  double w0 = 0;
  double2 wp[NP > 0 ? NP : 1];
#pragma unroll
  for (int p = 0; p < NP; p++) wp[p] = make_double2(0, 0);
  for (int g0 = 0; g0 < ng; g0 += kGTile) {
    const int nt = min(kGTile, ng - g0);
    __syncthreads();
    for (int t = threadIdx.x; t < nt; t += kWThreads) {
      sG[t] = gcrys[g0 + t];
#pragma unroll
      for (int p = 0; p < NP; p++) sP[t * NP + p] = gph[(size_t)(g0 + t) * NP + p];
    }
    __syncthreads();
    if (act) {
      for (int t = 0; t < nt; t++) {
        const double2 G = sG[t];
        double V;
        if (v.hartree && __dadd_rn(G.x, G.y) < 1e-16) {
          V = 0.0;
        } else {
          double x[3];
          cart_of(g, __dadd_rn(qx, G.x), __dadd_rn(qy, G.y), x);
          const double q_mod = __dadd_rn(__dadd_rn(__dmul_rn(x[0], x[0]), __dmul_rn(x[1], x[1])), __dmul_rn(x[2], x[2]));
          V = coul_v(q_mod, v);
        }
        w0 = __dadd_rn(w0, V);
#pragma unroll
        for (int p = 0; p < NP; p++) {
          const double2 e = sP[t * NP + p];
          wp[p].x = __dadd_rn(wp[p].x, __dmul_rn(V, e.x));
          wp[p].y = __dadd_rn(wp[p].y, __dmul_rn(V, e.y));
        }
      }
    }
  }
  if (!act) return;
  out[iq] = make_double2(w0, 0.0);
  if (NP > 0) {
    double xq[3];
    cart_of(g, qx, qy, xq);
#pragma unroll
    for (int p = 0; p < NP; p++) {
      // phi = k.cart . (tau_i - tau_j), summed in the reference's order
      double phi = 0.0;
#pragma unroll
      for (int c = 0; c < 3; c++) phi = __dadd_rn(phi, __dmul_rn(xq[c], tau[p * 3 + c]));
      double s, co;
      sincos(phi, &s, &co);
      out[(size_t)(1 + p) * nq + iq] = make_double2(co * wp[p].x - s * wp[p].y, co * wp[p].y + s * wp[p].x);
    }
  }
}

// Row pass of the mode sums: T[p][x][t] = sum_y w_y trig_t(y) W_p(x, y),
// trig_t = cos(2 pi n q) for t = 2n, sin for t = 2n + 1.
__global__ void k_rows(const double2* __restrict__ W, int nsum, int np1, const double* __restrict__ sp,
                       const double* __restrict__ trig, int nt, double2* __restrict__ T) {
  const int x = blockIdx.x, p = blockIdx.y, t = threadIdx.x;
  if (t >= nt || p >= np1 || x >= nsum) return;
  const double2* row = W + ((size_t)p * nsum + x) * nsum;
  const double* tr = trig + (size_t)t * nsum;
  double2 acc = make_double2(0, 0);
  for (int y = 0; y < nsum; y++) {
    const double c = sp[y] * tr[y];
    acc.x = fma(c, row[y].x, acc.x);
    acc.y = fma(c, row[y].y, acc.y);
  }
  T[((size_t)p * nsum + x) * nt + t] = acc;
}

// Column pass: S[p][m][t][cs] = sum_x 4 w_x trig_(2m+cs)(x) T[p][x][t].
__global__ void k_cols(const double2* __restrict__ T, int nsum, int np1, int ncut, const double* __restrict__ sp,
                       const double* __restrict__ trig, double2* __restrict__ S) {
  const int nt = 2 * ncut;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = np1 * ncut * nt * 2;
  if (id >= total) return;
  const int cs = id % 2, t = (id / 2) % nt, m = (id / (2 * nt)) % ncut, p = id / (2 * nt * ncut);
  const double* tr = trig + (size_t)(2 * m + cs) * nsum;
  double2 acc = make_double2(0, 0);
  for (int x = 0; x < nsum; x++) {
    const double c = 4.0 * sp[x] * tr[x];
    const double2 v = T[((size_t)p * nsum + x) * nt + t];
    acc.x = fma(c, v.x, acc.x);
    acc.y = fma(c, v.y, acc.y);
  }
  S[id] = acc;
}

// Screening constant terms: per candidate point, (W0_ij - series_ij(q)) / N^2
// for every (i <= j) of the n x n table (headers/Coulomb.h:245-267 for the
// series; the diagonal of W0 is W0_00). Up to 4 bands: 10 (i <= j) entries.
__global__ void k_screen_terms(const double2* __restrict__ W0, long long nq, const double2* __restrict__ qlist, int n,
                               int ncut, const double2* __restrict__ A, const double2* __restrict__ B,
                               const double2* __restrict__ C, const double2* __restrict__ D, double dk2,
                               double2* __restrict__ terms) {
  constexpr int kMaxTri = 10;
  const long long iq = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= nq || n > 4) return;
  const double kx = qlist[iq].x, ky = qlist[iq].y;
  const int n2 = n * n;
  double2 vf[kMaxTri];
  for (int t = 0; t < kMaxTri; t++) vf[t] = make_double2(0, 0);
  for (int m = 0; m < ncut; m++) {
    double sm, cm;
    sincos(2 * M_PI * m * kx, &sm, &cm);
    for (int nn = 0; nn < ncut; nn++) {
      double sn, cn;
      sincos(2 * M_PI * nn * ky, &sn, &cn);
      const double fa = cm * cn, fb = cm * sn, fc = sm * cn, fd = sm * sn;
      const size_t row = (size_t)(nn + ncut * m) * n2;
      int t = 0;
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic; jc < n; jc++, t++) {
          const size_t ix = row + ic * n + jc;
          const double2 a = A[ix], b = B[ix], c = C[ix], d = D[ix];
          vf[t].x += a.x * fa + b.x * fb + c.x * fc + d.x * fd;
          vf[t].y += a.y * fa + b.y * fb + c.y * fc + d.y * fd;
        }
    }
  }
  int p = 0, t = 0;
  for (int ic = 0; ic < n; ic++)
    for (int jc = ic; jc < n; jc++, t++) {
      const double2 wv = ic == jc ? W0[iq] : W0[(size_t)(1 + p) * nq + iq];
      if (ic != jc) p++;
      terms[(size_t)(ic * n + jc) * nq + iq] = make_double2((wv.x - vf[t].x) * dk2, (wv.y - vf[t].y) * dk2);
    }
}

// Fixed-order sum of each column of terms [ncol][nq] (one block per column).
__global__ void k_colsum(const double2* __restrict__ terms, long long nq, double2* __restrict__ out) {
  __shared__ double2 red[256];
  const int col = blockIdx.x;
  double2 acc = make_double2(0, 0);
  for (long long i = threadIdx.x; i < nq; i += blockDim.x) {
    const double2 v = terms[(size_t)col * nq + i];
    acc.x += v.x;
    acc.y += v.y;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      red[threadIdx.x].x += red[threadIdx.x + s].x;
      red[threadIdx.x].y += red[threadIdx.x + s].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[col] = red[0];
}

template <int NP>
cudaError_t launch_wq_np(const Geo& g, const VPar& v, const double* qgrid, int nsum, const double2* qlist, long long nq,
                         const double2* gcrys, const double2* gph, int ng, const double* tau, double2* out, cudaStream_t s) {
  const long long blocks = (nq + kWThreads - 1) / kWThreads;
  if (blocks <= 0) return cudaSuccess;
  k_wq<NP><<<(unsigned)blocks, kWThreads, 0, s>>>(g, v, qgrid, nsum, qlist, nq, gcrys, gph, ng, tau, out);
  return cudaGetLastError();
}

cudaError_t launch_wq(int np, const Geo& g, const VPar& v, const double* qgrid, int nsum, const double2* qlist, long long nq,
                      const double2* gcrys, const double2* gph, int ng, const double* tau, double2* out, cudaStream_t s) {
  switch (np) {
    case 0: return launch_wq_np<0>(g, v, qgrid, nsum, qlist, nq, gcrys, gph, ng, tau, out, s);
    case 1: return launch_wq_np<1>(g, v, qgrid, nsum, qlist, nq, gcrys, gph, ng, tau, out, s);
    case 3: return launch_wq_np<3>(g, v, qgrid, nsum, qlist, nq, gcrys, gph, ng, tau, out, s);
    case 6: return launch_wq_np<6>(g, v, qgrid, nsum, qlist, nq, gcrys, gph, ng, tau, out, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace cgen
}  // namespace edus

// ----------------------------------------------------------------- host driver

namespace edus {
namespace cgen {
namespace {

struct DevBuf {
  std::vector<void*> p;
  ~DevBuf() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  int get(T** out, size_t count) {
    void* v = nullptr;
    if (cudaMalloc(&v, sizeof(T) * (count ? count : 1)) != cudaSuccess)
      return fail(EDUS_ENOMEM, "Coulomb generator: cudaMalloc of %zu bytes", sizeof(T) * count);
    p.push_back(v);
    *out = (T*)v;
    return 0;
  }
};

#define GCK(x)                                                                           \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) return fail(EDUS_ECUDA, "Coulomb generator: %s", cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int up(T* d, const std::vector<T>& h, cudaStream_t s) {
  GCK(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
  return 0;
}

// Coordinate::setcrys on the host, as the reference accumulates it.
void host_cart(const Problem& P, const double* c, double* x) {
  for (int i = 0; i < 3; i++) {
    x[i] = 0.;
    for (int j = 0; j < 3; j++) x[i] += P.M[i][j] * c[j];
  }
}

// 1D Simpson grid (headers/integrationWeight.h:5-15), border 0.5.
void simpson(int N, std::vector<double>& q, std::vector<double>& sp) {
  q.resize(N);
  sp.resize(N);
  const double h = 2 * 0.5 / (N - 1);
  for (int i = 0; i < N; i++) q[i] = -0.5 + i * h;
  const double hs = (3 * (N - 1));
  sp[0] = 1 / hs;
  for (int i = 1; i < N; i += 2) sp[i] = 4.0 / hs;
  for (int i = 2; i < N; i += 2) sp[i] = 2.0 / hs;
  sp[N - 1] = 1 / hs;
}

}  // namespace
}  // namespace cgen
}  // namespace edus

using namespace edus;
using namespace edus::cgen;

extern "C" {

int edus_coulomb_gen_options_default(edus_coulomb_gen_options* o) {
  if (!o) return fail(EDUS_EINVAL, "null argument");
  o->device = 0;
  o->n_sum = 4999;
  o->n_sum_screen = 39999;
  return 0;
}

int edus_coulomb_generate(const edus_params* pin, const char* workdir, const edus_coulomb_gen_options* opt, char* label_out,
                          int32_t label_cap, int32_t* g_num_out) {
  if (!pin || !workdir) return fail(EDUS_EINVAL, "null argument");
  edus_coulomb_gen_options o;
  if (opt)
    o = *opt;
  else
    edus_coulomb_gen_options_default(&o);
  if (o.n_sum < 3 || o.n_sum % 2 == 0 || o.n_sum_screen < 3 || o.n_sum_screen % 2 == 0)
    return fail(EDUS_EINVAL, "Simpson grids need an odd number of points >= 3 (%d, %d)", o.n_sum, o.n_sum_screen);
  const int ncut = pin->ncut;
  if (ncut < 1 || ncut > 64) return fail(EDUS_EINVAL, "Ncut %d out of range", ncut);
  // the model and lattice of the run, without the Coulomb tables it is to produce
  edus_params q = *pin;
  q.coulomb = 0;
  Problem P;
  int rc = build_problem(q, workdir, P);
  if (rc) return rc;
  const int n = P.ncv, n2 = n * n;
  const int np = n * (n - 1) / 2;
  if (np > kMaxPairs || (np != 0 && np != 1 && np != 3 && np != 6))
    return fail(EDUS_EUNSUPPORTED, "Coulomb generator: %d bands (up to 4)", n);
  const bool o110 = q.sample_110 != 0;
  // Displacement_orb: real diagonal dipoles at one k point (Fourier_Coulomb.cpp:41-67)
  std::vector<double> disp((size_t)n * 3);
  {
    double kc[3] = {0.0, 0.3, 0.1};
    if (o110) {
      kc[0] = 0.3;
      kc[1] = 0.1;
      kc[2] = 0.0;
    }
    std::vector<cd> H(n2), U(n2), D((size_t)n2 * 3);
    if ((rc = model_hud(P, kc, H.data(), U.data(), D.data()))) return rc;
    for (int ic = 0; ic < n; ic++)
      for (int x = 0; x < 3; x++) disp[ic * 3 + x] = D[((size_t)ic * n + ic) * 3 + x].real();
  }
  std::vector<double> tau((size_t)np * 3);
  {
    int p = 0;
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic + 1; jc < n; jc++, p++)
        for (int x = 0; x < 3; x++) tau[p * 3 + x] = disp[ic * 3 + x] - disp[jc * 3 + x];
  }
  const double det_b = o110 ? std::fabs(q.b[0][0] * q.b[1][1] - q.b[0][1] * q.b[1][0])
                            : std::fabs(q.b[1][1] * q.b[2][2] - q.b[1][2] * q.b[2][1]);
  VPar vp{};
  vp.qTF = q.qTF;
  vp.eps_area = q.epsilon_static * P.det_a;
  vp.r0 = q.r0;
  vp.rk = q.rytova_keldysh;
  const double gdist = q.G_distance * std::sqrt(det_b);
  // G list and the phases exp(i G.tau_p) (Fourier_Coulomb.cpp:113-136; Coulomb.h:128-142)
  std::vector<double2> gl;
  std::vector<double2> gph;
  {
    const int bord = (int)(std::sqrt(9999.0 * 9999.0) / 2);
    for (int ix = -bord; ix <= bord; ix++)
      for (int iy = -bord; iy <= bord; iy++) {
        double c[3] = {0.0, (double)ix, (double)iy}, x[3];
        if (o110) {
          c[0] = ix;
          c[1] = iy;
          c[2] = 0.0;
        }
        host_cart(P, c, x);
        if (std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) < gdist) {
          gl.push_back(make_double2(ix, iy));
          for (int p = 0; p < np; p++) {
            double phi = 0.0;
            for (int k = 0; k < 3; k++) phi += x[k] * tau[p * 3 + k];
            gph.push_back(make_double2(std::cos(phi), std::sin(phi)));
          }
        }
      }
  }
  const int ng = (int)gl.size();
  if (g_num_out) *g_num_out = ng;
  Geo geo{};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) geo.M[i][j] = P.M[i][j];
  geo.o110 = o110;

  GCK(cudaSetDevice(o.device));
  cudaStream_t s = nullptr;
  GCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};
  DevBuf db;
  double2 *d_g = nullptr, *d_ph = nullptr;
  double* d_tau = nullptr;
  if ((rc = db.get(&d_g, ng)) || (rc = db.get(&d_ph, (size_t)ng * np)) || (rc = db.get(&d_tau, tau.size()))) return rc;
  if ((rc = up(d_g, gl, s)) || (np && (rc = up(d_ph, gph, s))) || (np && (rc = up(d_tau, tau, s)))) return rc;

  // ---- Hartree table: W at q = 0 with V = 0 where G0 + G1 < 1e-16
  std::vector<double> VH((size_t)n2);
  {
    double2 *d_q = nullptr, *d_w = nullptr;
    if ((rc = db.get(&d_q, 1)) || (rc = db.get(&d_w, (size_t)(np + 1)))) return rc;
    std::vector<double2> q0(1, make_double2(0.0, 0.0));
    if ((rc = up(d_q, q0, s))) return rc;
    VPar vh = vp;
    vh.hartree = 1;
    GCK(launch_wq(np, geo, vh, nullptr, 0, d_q, 1, d_g, d_ph, ng, d_tau, d_w, s));
    std::vector<double2> w(np + 1);
    GCK(cudaMemcpyAsync(w.data(), d_w, sizeof(double2) * w.size(), cudaMemcpyDeviceToHost, s));
    GCK(cudaStreamSynchronize(s));
    std::vector<cd> V((size_t)n2, 0.0);
    V[0] = cd(w[0].x, w[0].y);
    int p = 0;
    for (int ic = 0; ic < n; ic++)
      for (int jc = ic + 1; jc < n; jc++, p++) V[ic * n + jc] = cd(w[1 + p].x, w[1 + p].y);
    for (int ic = 0; ic < n; ic++) {
      if (ic > 0) V[ic * n + ic] = V[0];
      for (int jc = ic; jc < n; jc++) {
        V[jc * n + ic] = V[ic * n + jc].real();
        V[ic * n + jc] = V[jc * n + ic];
      }
    }
    for (int i = 0; i < n2; i++) VH[i] = V[i].real();
  }

  // ---- W on the N x N Simpson grid, then the separable mode sums
  const int N = o.n_sum, nt = 2 * ncut;
  std::vector<double> qg, sp;
  simpson(N, qg, sp);
  std::vector<double> trig((size_t)nt * N);
  for (int nn = 0; nn < ncut; nn++)
    for (int y = 0; y < N; y++) {
      const double a = 2 * M_PI * nn * qg[y];
      trig[(size_t)(2 * nn) * N + y] = std::cos(a);
      trig[(size_t)(2 * nn + 1) * N + y] = std::sin(a);
    }
  const long long nq = (long long)N * N;
  double *d_qg = nullptr, *d_sp = nullptr, *d_trig = nullptr;
  double2 *d_W = nullptr, *d_T = nullptr, *d_S = nullptr;
  const size_t nS = (size_t)(np + 1) * ncut * nt * 2;
  if ((rc = db.get(&d_qg, N)) || (rc = db.get(&d_sp, N)) || (rc = db.get(&d_trig, trig.size())) ||
      (rc = db.get(&d_W, (size_t)(np + 1) * nq)) || (rc = db.get(&d_T, (size_t)(np + 1) * N * nt)) || (rc = db.get(&d_S, nS)))
    return rc;
  if ((rc = up(d_qg, qg, s)) || (rc = up(d_sp, sp, s)) || (rc = up(d_trig, trig, s))) return rc;
  GCK(launch_wq(np, geo, vp, d_qg, N, nullptr, nq, d_g, d_ph, ng, d_tau, d_W, s));
  k_rows<<<dim3(N, np + 1), (nt + 31) / 32 * 32, 0, s>>>(d_W, N, np + 1, d_sp, d_trig, nt, d_T);
  GCK(cudaGetLastError());
  k_cols<<<(unsigned)((nS + 127) / 128), 128, 0, s>>>(d_T, N, np + 1, ncut, d_sp, d_trig, d_S);
  GCK(cudaGetLastError());
  std::vector<double2> S(nS);
  GCK(cudaMemcpyAsync(S.data(), d_S, sizeof(double2) * nS, cudaMemcpyDeviceToHost, s));
  GCK(cudaStreamSynchronize(s));
  // coefficients [mm][il] (Fourier_Coulomb.cpp:254-265; Coulomb.h:163-233)
  const size_t nc = (size_t)ncut * ncut * n2;
  std::vector<double2> cA(nc, make_double2(0, 0)), cB(nc, make_double2(0, 0)), cC(nc, make_double2(0, 0)),
      cD(nc, make_double2(0, 0));
  auto Sat = [&](int p, int m, int t, int cs) { return S[(((size_t)p * ncut + m) * nt + t) * 2 + cs]; };
  for (int m = 0; m < ncut; m++)
    for (int nn = 0; nn < ncut; nn++) {
      const size_t mm = (size_t)m * ncut + nn;
      const double fac = (m == 0 && nn == 0) ? 0.25 : ((m == 0 || nn == 0) ? 0.5 : 1.0);
      cA[mm * n2].x = fac * Sat(0, m, 2 * nn, 0).x;
      cD[mm * n2].x = fac * Sat(0, m, 2 * nn + 1, 1).x;
      int p = 0;
      for (int ic = 0; ic < n; ic++)
        for (int jc = ic + 1; jc < n; jc++, p++) {
          const size_t il = mm * n2 + ic * n + jc;
          cA[il].x = fac * Sat(1 + p, m, 2 * nn, 0).x;
          cB[il].y = fac * Sat(1 + p, m, 2 * nn + 1, 0).y;
          cC[il].y = fac * Sat(1 + p, m, 2 * nn, 1).y;
          cD[il].x = fac * Sat(1 + p, m, 2 * nn + 1, 1).x;
        }
    }

  // ---- screening constant on the fine grid, points with |q| < max(qTF, 0.02)
  std::vector<double2> screen((size_t)n2, make_double2(0, 0));
  {
    const int N2 = o.n_sum_screen;
    const double h2 = 2 * 0.5 / (N2 - 1), dk2 = 1. / ((double)N2 * N2);
    const double q_peak = q.qTF < 0.02 ? 0.02 : q.qTF;
    auto q_mod_at = [&](double qx, double qy) {
      double c[3] = {0.0, qx, qy}, x[3];
      if (o110) {
        c[0] = qx;
        c[1] = qy;
        c[2] = 0.0;
      }
      host_cart(P, c, x);
      return x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    };
    auto inside = [&](double qm) { return qm < q_peak * q_peak && qm > std::pow(10, -17); };
    // per row, the interval of qy in the ellipse |q(qx, qy)| < q_peak, widened
    // by two points each side and then tested point by point as the reference
    // tests every point
    std::vector<double2> cand;
    for (int ix = 0; ix < N2; ix++) {
      const double qx = -0.5 + ix * h2;
      const double f0 = q_mod_at(qx, 0.0), f1 = q_mod_at(qx, 1.0), fm = q_mod_at(qx, -1.0);
      const double a = 0.5 * (f1 + fm) - f0, b = 0.5 * (f1 - fm), c = f0 - q_peak * q_peak;
      if (a <= 0) continue;
      const double disc = b * b - 4 * a * c;
      const double vtx = -b / (2 * a);
      double lo, hi;
      if (disc < 0) {
        if (c - b * b / (4 * a) > 1e-12 * q_peak * q_peak) continue;
        lo = hi = vtx;
      } else {
        lo = (-b - std::sqrt(disc)) / (2 * a);
        hi = (-b + std::sqrt(disc)) / (2 * a);
      }
      const long long i0 = std::max<long long>(0, (long long)std::floor((lo + 0.5) / h2) - 2);
      const long long i1 = std::min<long long>(N2 - 1, (long long)std::ceil((hi + 0.5) / h2) + 2);
      for (long long iy = i0; iy <= i1; iy++) {
        const double qy = -0.5 + iy * h2;
        if (inside(q_mod_at(qx, qy))) cand.push_back(make_double2(qx, qy));
      }
    }
    const long long nc2 = (long long)cand.size();
    if (nc2 > 0) {
      double2 *d_c = nullptr, *d_W0 = nullptr, *d_terms = nullptr, *d_sum = nullptr;
      double2 *dA = nullptr, *dB = nullptr, *dC = nullptr, *dD = nullptr;
      if ((rc = db.get(&d_c, nc2)) || (rc = db.get(&d_W0, (size_t)(np + 1) * nc2)) ||
          (rc = db.get(&d_terms, (size_t)n2 * nc2)) || (rc = db.get(&d_sum, n2)) || (rc = db.get(&dA, nc)) ||
          (rc = db.get(&dB, nc)) || (rc = db.get(&dC, nc)) || (rc = db.get(&dD, nc)))
        return rc;
      if ((rc = up(d_c, cand, s)) || (rc = up(dA, cA, s)) || (rc = up(dB, cB, s)) || (rc = up(dC, cC, s)) || (rc = up(dD, cD, s)))
        return rc;
      GCK(cudaMemsetAsync(d_terms, 0, sizeof(double2) * n2 * nc2, s));
      VPar v0 = vp;
      v0.qTF = 0.0;
      GCK(launch_wq(np, geo, v0, nullptr, 0, d_c, nc2, d_g, d_ph, ng, d_tau, d_W0, s));
      k_screen_terms<<<(unsigned)((nc2 + 127) / 128), 128, 0, s>>>(d_W0, nc2, d_c, n, ncut, dA, dB, dC, dD, dk2, d_terms);
      GCK(cudaGetLastError());
      k_colsum<<<n2, 256, 0, s>>>(d_terms, nc2, d_sum);
      GCK(cudaGetLastError());
      GCK(cudaMemcpyAsync(screen.data(), d_sum, sizeof(double2) * n2, cudaMemcpyDeviceToHost, s));
      GCK(cudaStreamSynchronize(s));
    }
  }

  // ---- files (Fourier_Coulomb.cpp:145-153, 196-208, 337-366, 476-484)
  std::ostringstream lb;
  lb << "G_num" << ng << "_Ncut" << ncut << q.coulomb_label;
  const std::string label = lb.str();
  if (label_out && label_cap > 0) snprintf(label_out, (size_t)label_cap, "%s", label.c_str());
  const std::string od = std::string(workdir) + "/Output", cdir = od + "/Coulomb";
  mkdir(od.c_str(), 0755);
  mkdir(cdir.c_str(), 0755);
  {
    std::ofstream f(cdir + "/V_Hartree_" + label + ".txt");
    if (!f) return fail(EDUS_EIO, "cannot write into %s", cdir.c_str());
    for (int ic = 0; ic < n; ic++) {
      for (int jc = 0; jc < n; jc++) f << std::setprecision(20) << VH[ic * n + jc] << "    ";
      f << std::endl;
    }
  }
  const char* nm[4] = {"A", "B", "C", "D"};
  const std::vector<double2>* cs4[4] = {&cA, &cB, &cC, &cD};
  for (int k = 0; k < 4; k++) {
    std::ofstream f(cdir + "/" + nm[k] + "_coeff" + label + ".txt");
    if (!f) return fail(EDUS_EIO, "cannot write into %s", cdir.c_str());
    for (int mm = 0; mm < ncut * ncut; mm++) {
      for (int il = 0; il < n2; il++) {
        const double2 v = (*cs4[k])[(size_t)mm * n2 + il];
        f << std::setprecision(20) << std::scientific << v.x << "    " << v.y << "    ";
      }
      f << std::endl;
    }
  }
  {
    std::ofstream f(cdir + "/Screen_const_" + label + ".txt");
    if (!f) return fail(EDUS_EIO, "cannot write into %s", cdir.c_str());
    for (int il = 0; il < n2; il++) f << std::setprecision(20) << screen[il].x << " " << screen[il].y << std::endl;
  }
  return 0;
}

}  // extern "C"
