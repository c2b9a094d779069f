// batch.cu — host side of the batched engine: instance admission and release,
// per-class tile tables, chunked CUDA-graph replay (C ABI edus_batch_*).
//
// The time loop of each instance is the reference's constant-dt loop
// (Source_Main/const_dt_evolution.cpp:1-54) with the RK4 step of
// Source_Main/RungeKutta.cpp; instances share only the GPU. Device memory of
// an instance comes from a stream-ordered pool owned by the batch, so admission
// and release never synchronise the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "ctx_hooks.hpp"
#include "cuda/batch.cuh"
#include "cuda/model_build.hpp"
#include "cuda/tc_contract.hpp"
#include "host/problem.hpp"

namespace edus {
namespace batch {
namespace {

#define BCK(x)                                                                            \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) return fail(EDUS_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int default_tile(int n) {
  switch (n) {
    case 2: return 32;
    case 3: return 32;
    case 4: return 16;
    case 5: return 16;
    case 8: return 8;
    case 16: return 2;
  }
  return 0;
}

struct Slot {
  int status = EDUS_INST_FREE;
  int n = 0, kt = 0, nk = 0, ntri = 0, itfi = 0, res = 1, nlog = 0, ntiles = 0;
  int64_t tag = 0;
  int64_t bytes = 0;
  long long tick_admit = 0;
  std::vector<void*> mem;
  Inst inst{};
  // an instance with the Coulomb mean field: a single-solve context whose
  // whole loop runs as one graph on the context's stream (FP64)
  edus_ctx* sub = nullptr;
};

struct ClassTab {
  int n = 0, kt = 0, occ = 0;  // occ: requested register profile / kernel form
  int form = -1;               // form in use (profile 3 falls back to 0 when an instance does not fit it)
  int psel = 0, pcomp = 0;     // profile 3: most stencil vectors / field components in use per instance
  std::vector<Tile> tiles;
  Tile* d_tiles = nullptr;
  size_t cap = 0;
  int* d_ntiles = nullptr;         // [0] tiles, [1] instances of the class
  std::vector<ClassInst> insts;    // instance table (observable kernel)
  ClassInst* d_cinst = nullptr;    // capacity: the batch's max_instances
  int sgrid = 0, ogrid = 0;
  bool dirty = false;
};

struct Layout {
  size_t state, H, D, GE, U, nbr, field, log, part;
  size_t eq;     // initial state kept for the mixed-precision deviation form
  size_t hdiag;  // FP64 band energies of the mixed-precision commutator
  size_t w;      // E-linear rho_eq terms of the mixed-precision deviation form
  size_t total() const { return 4 * state + eq + hdiag + w + H + D + GE + U + nbr + field + log + part + 256; }
};

}  // namespace
}  // namespace batch
}  // namespace edus

using namespace edus;
using namespace edus::batch;

struct edus_batch {
  edus_batch_options opt{};
  bool mixed = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<Slot> slots;
  Inst* d_insts = nullptr;
  int* d_it[2] = {nullptr, nullptr};
  int* d_err = nullptr;  // device error word of bounded waits
  std::map<int, ClassTab> classes;
  long long tick = 0;
  int64_t bytes_used = 0, budget = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::string graph_key;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double device_ms = 0, kpoint_steps = 0;
  long long launches = 0;
  long long h2d_bytes = 0, d2h_bytes = 0;
};

namespace {

// Precision of a class of band count n. A mixed-precision batch runs classes
// of 4 bands and more in mixed precision and the 2- and 3-band classes in
// FP64: their stage is dominated by the finite-difference k-gradient, whose
// terms cancel to ~1/N of their size, so FP32 stage inputs leave a relative
// error of ~N x 6e-8 in it (J1 error 1.1e-6 measured on a 144 x 144 hBN
// sweep instance), while FP64 costs these classes little (their kernels are
// latency-bound). The autotuner's options for mixed batches give these
// classes their FP64 tuning (edus_b200/autotune.py, MIXED_MIN_BANDS).
constexpr int kMixedMinBands = 4;
bool cmix(const edus_batch* b, int n) { return b->mixed && n >= kMixedMinBands; }

int tile_len(const edus_batch* b, int n) {
  int kt = (n >= 0 && n <= EDUS_MAX_BANDS) ? b->opt.tile_k[n] : 0;
  return kt > 0 ? kt : default_tile(n);
}

Layout layout_of(const edus_batch* b, const Problem& P, int kt) {
  const size_t n = P.ncv, nk = P.nk, nt = n * (n + 1) / 2;
  const bool mix = cmix(b, (int)n);
  const size_t s = mix ? sizeof(float2) : sizeof(double2);
  Layout L;
  L.state = align256(nt * nk * sizeof(double2));
  L.eq = mix ? L.state : 0;
  L.hdiag = mix ? align256(n * nk * sizeof(double)) : 0;
  L.w = mix ? align256(3 * nt * nk * sizeof(float2)) : 0;
  L.H = align256(nt * nk * s);
  L.D = align256(3 * nt * nk * s);
  L.GE = P.p.current ? align256(3 * nt * nk * s) : 0;
  L.U = align256(n * n * nk * s);
  L.nbr = align256((size_t)P.nnb * nk * sizeof(int));
  L.field = align256((size_t)(P.itfi + 2) * sizeof(FieldRow));
  const int res = std::max(1, P.p.it_resolution);
  L.log = align256((size_t)(P.itfi / res + 1) * sizeof(edus_obs));
  L.part = align256(((nk + kt - 1) / kt) * obs_part_bytes());
  return L;
}

// commutator form of the staged kernel for register profile 3, 4, 5:
// element-parallel, register blocks of C of 2 x 2, of 2 x 1
int pipe_cb(int prof) { return prof == 5 ? 2 : (prof == 4 ? 1 : 0); }

// register profile / kernel form of a band count; the matrix-product form is built for FP64 only
int profile_of(const edus_batch* b, int n) {
  const int p = (n >= 0 && n <= EDUS_MAX_BANDS) ? b->opt.regs_profile[n] : 0;
  if (p == 2 && cmix(b, n)) return 0;
  if (p >= 3 && !cmix(b, n)) return 0;  // asynchronous staging is built for mixed precision
  return p;
}

// Kernel form a class runs: profiles 3 and 4 need every running instance of
// the class on a lattice stencil, otherwise the element-parallel form. Also
// the staging sizes of profiles 3 and 4 (at least one slot each).
int form_of(const edus_batch* b, const ClassTab& c, int& psel, int& pcomp) {
  psel = pcomp = 1;
  if (c.occ < 3 || c.occ > 5) return c.occ;
  if (!pipe_supported(c.n, c.kt, pipe_cb(c.occ))) return 0;
  for (const Slot& s : b->slots) {
    if (s.status != EDUS_INST_RUNNING || s.n != c.n) continue;
    const Inst& I = s.inst;
    if (!I.lattice) return 0;
    psel = std::max(psel, I.nsel);
    pcomp = std::max(pcomp, ((I.fmask >> 0) & 1) + ((I.fmask >> 1) & 1) + ((I.fmask >> 2) & 1));
  }
  return c.occ;
}

int grid_of(const edus_batch* b, const ClassTab& c) {
  switch (c.form) {
    case 2: return stage_grid_mm(c.n, c.kt, cmix(b, c.n));
    case 3:
    case 4:
    case 5: return stage_grid_pipe(c.n, c.kt, pipe_cb(c.form), c.psel, c.pcomp);
    default: return stage_grid(c.n, c.kt, c.form ? 1 : 0, cmix(b, c.n));
  }
}

int check_problem(const edus_batch* b, const Problem& P) {
  const int n = P.ncv;
  if (P.p.mode == EDUS_MODE_CRYSTAL)
    return fail(EDUS_EUNSUPPORTED, "batch: Crystal models keep Hermitian dipoles, which the batch kernels (one symmetric dipole "
                                   "plane per band pair) do not run; single-solve contexts run them");
  if (P.p.coulomb) {
    // runs as a single-solve context inside the batch (every solver at constant dt, FP64)
    if (P.p.dynamical_dt) return fail(EDUS_EUNSUPPORTED, "batch: a Coulomb instance integrates at constant dt");
    if (P.model_deferred) return fail(EDUS_EUNSUPPORTED, "batch: a Coulomb instance needs host-built model tables");
    return 0;
  }
  const int prof = profile_of(b, n), kt = tile_len(b, n);
  // the staged forms also run tile lengths the element-parallel form is not built for
  // (their instances must then be on a lattice stencil, checked at admission)
  const bool ok = prof == 2 ? mm_supported(n, kt) : (class_supported(n, kt) || (prof >= 3 && pipe_supported(n, kt, pipe_cb(prof))));
  if (!ok)
    return fail(EDUS_EUNSUPPORTED, "batch: %d bands with %d k points per tile (profile %d) is not built", n, tile_len(b, n),
                profile_of(b, n));
  if (cmix(b, n) && P.nch > 0)
    return fail(EDUS_EUNSUPPORTED,
                "batch: mixed precision needs a problem without core bands (edus_problem_drop_decoupled_core, or FP64)");
  if (!P.diss_i.empty()) return fail(EDUS_EUNSUPPORTED, "batch: dissipation runs only in single-solve contexts");
  if (P.p.solver != EDUS_SOLVER_RK4 || P.p.dynamical_dt)
    return fail(EDUS_EUNSUPPORTED, "batch: instances integrate with RK4 at constant dt");
  if (P.nnb > kBatchMaxNb) return fail(EDUS_EUNSUPPORTED, "batch: %d stencil neighbours (max %d)", P.nnb, kBatchMaxNb);
  return 0;
}

template <class T>
T mkc(const cd& v);
template <>
double2 mkc<double2>(const cd& v) { return make_double2(v.real(), v.imag()); }
template <>
float2 mkc<float2>(const cd& v) { return make_float2((float)v.real(), (float)v.imag()); }

// reference layout [k][n][n](x comps) -> upper-triangle planes [x][e][k]
template <class T>
void planes(const cd* src, int nk, int n, int comps, std::vector<T>& dst) {
  const int nt = n * (n + 1) / 2;
  dst.resize((size_t)comps * nt * nk);
  for (int k = 0; k < nk; k++)
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++)
        for (int x = 0; x < comps; x++)
          dst[((size_t)x * nt + tri_index(i, j, n)) * nk + k] = mkc<T>(src[(((size_t)k * n + i) * n + j) * comps + x]);
}

template <class T>
int put(edus_batch* b, void* d, const std::vector<T>& h) {
  BCK(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, b->stream));
  b->h2d_bytes += (long long)(sizeof(T) * h.size());
  return 0;
}

template <class T>
int upload_model(edus_batch* b, const Problem& P, const Inst& I) {
  const int n = P.ncv, nk = P.nk;
  std::vector<T> pl;
  int rc;
  planes<T>(P.H.data(), nk, n, 1, pl);
  if ((rc = put(b, (void*)I.H, pl))) return rc;
  planes<T>(P.D.data(), nk, n, 3, pl);
  if ((rc = put(b, (void*)I.D, pl))) return rc;
  if (I.GE) {
    planes<T>(P.GE.data(), nk, n, 3, pl);
    if ((rc = put(b, (void*)I.GE, pl))) return rc;
  }
  pl.resize((size_t)n * n * nk);
  for (int k = 0; k < nk; k++)
    for (int e = 0; e < n * n; e++) pl[(size_t)e * nk + k] = mkc<T>(P.U[(size_t)k * n * n + e]);
  if ((rc = put(b, (void*)I.U, pl))) return rc;
  if (I.Hdiag) {
    std::vector<double> hd((size_t)n * nk);
    for (int k = 0; k < nk; k++)
      for (int i = 0; i < n; i++) hd[(size_t)i * nk + k] = P.H[((size_t)k * n + i) * n + i].real();
    if ((rc = put(b, (void*)I.Hdiag, hd))) return rc;
  }
  return 0;
}

// Field components and stencil vectors that contribute for the whole run. A
// component that is zero in every field-table row (pump and probe, at t and
// t + dt/2) adds E_x D_x = 0 and E_x W_x = 0 exactly; a stencil vector
// orthogonal to every pump component in use has a gradient coefficient
// w_b (E_pump . b) that is exactly 0. A shell weight below 1e-12 of the
// largest is least-squares noise of the weight fit (headers/CalculateWeigths.h:
// the diagonal shell of a square grid comes out near 1e-21 against 1e3) and
// its terms lie below the FP64 resolution of the sum. The stage kernels skip
// all of these; the remaining terms are summed in the same order.
//
// fp32_terms (classes whose commutator runs in FP32): a stencil vector whose
// coefficient bound |w_b| |b restricted to the pump components| is at most
// 1e-12 of the largest is skipped too. Such vectors are in-plane steps whose
// pump-direction component is rounding residue of the grid-vector differences
// (7.4e-17 against 1.4e-2 on a 98 x 98 square grid with a z-polarised pump):
// their terms are 1e-12 or less of the largest term, four orders below the
// FP32 rounding of the sum, and kept they would double the staging slots of
// every instance of the class (one such instance sets the class's slot count).
void select_terms(const Problem& P, const std::vector<FieldRow>& fr, Inst& I, bool fp32_terms) {
  int fmask = 0, pmask = 0;
  for (const FieldRow& r : fr)
    for (int x = 0; x < 3; x++) {
      if (r.Et[x] != 0. || r.Eh[x] != 0.) pmask |= 1 << x;
      if (r.Et[3 + x] != 0. || r.Eh[3 + x] != 0.) fmask |= 1 << x;
    }
  I.fmask = fmask | pmask;
  I.nsel = 0;
  double wmax = 0., cmax = 0.;
  auto coef = [&](int b) {
    double s = 0.;
    for (int x = 0; x < 3; x++)
      if ((pmask >> x) & 1) s += P.bvec[b * 3 + x] * P.bvec[b * 3 + x];
    return std::fabs(P.shell_w[P.bshell[b]]) * std::sqrt(s);
  };
  for (int b = 0; b < P.nnb; b++) {
    wmax = std::max(wmax, std::fabs(P.shell_w[P.bshell[b]]));
    cmax = std::max(cmax, coef(b));
  }
  for (int b = 0; b < P.nnb; b++) {
    bool on = false;
    for (int x = 0; x < 3; x++) on = on || ((pmask >> x) & 1 && P.bvec[b * 3 + x] != 0.);
    if (fp32_terms && coef(b) <= 1e-12 * cmax) on = false;
    if (on && std::fabs(P.shell_w[P.bshell[b]]) > 1e-12 * wmax) I.bsel[I.nsel++] = b;
  }
}

// A tile is interior when its k points lie in one grid row and every selected
// stencil step stays inside the grid without wrapping: then k + b = k + d1 n2 + d2.
int interior_tile(const Inst& I, int k0, int kt) {
  if (!I.lattice) return 0;
  const int k1 = std::min(k0 + kt, I.nk) - 1;
  const int i1 = k0 / I.n2, i2a = k0 % I.n2, i2b = k1 % I.n2;
  if (k1 / I.n2 != i1) return 0;
  for (int c = 0; c < I.nsel; c++) {
    const int b = I.bsel[c];
    const int j1 = i1 + I.off[b][0];
    if (j1 < 0 || j1 >= I.n1 || i2a + I.off[b][1] < 0 || i2b + I.off[b][1] >= I.n2) return 0;
  }
  return 1;
}

// The k-gradient neighbours of a Monkhorst-Pack grid are fixed lattice steps
// with periodic wrap. Find the step of every b from k = 0 and keep the table
// path unless every k agrees.
void detect_lattice(const Problem& P, Inst& I) {
  const int* Nk = P.p.nk;
  int n1 = 0, n2 = 0;
  if (Nk[0] == 1) {
    n1 = Nk[1];
    n2 = Nk[2];
  } else if (Nk[2] == 1) {
    n1 = Nk[0];
    n2 = Nk[1];
  }
  I.n1 = n1 > 0 ? n1 : 1;
  I.n2 = n2 > 0 ? n2 : P.nk;
  I.lattice = 0;
  if (n1 <= 0 || n2 <= 0 || (size_t)n1 * n2 != (size_t)P.nk || P.nnb > kBatchMaxNb) return;
  for (int b = 0; b < P.nnb; b++) {
    const int kb = P.nbr[b];
    int d1 = kb / n2, d2 = kb % n2;
    if (d1 > n1 / 2) d1 -= n1;
    if (d2 > n2 / 2) d2 -= n2;
    I.off[b][0] = d1;
    I.off[b][1] = d2;
  }
  for (int k = 0; k < P.nk; k++) {
    const int i1 = k / n2, i2 = k % n2;
    for (int b = 0; b < P.nnb; b++) {
      const int j1 = ((i1 + I.off[b][0]) % n1 + n1) % n1, j2 = ((i2 + I.off[b][1]) % n2 + n2) % n2;
      if (P.nbr[(size_t)k * P.nnb + b] != j1 * n2 + j2) return;
    }
  }
  for (int b = 0; b < P.nnb; b++)
    if (I.off[b][0] <= -n1 || I.off[b][0] >= n1 || I.off[b][1] <= -n2 || I.off[b][1] >= n2) return;
  I.lattice = 1;
}

// Mixed precision: H(k), D(k) on the tensor cores (cuda/tc_contract.cu, split
// TF32), band energies in FP64, then the eigensolve and dH/dk on the FP64 matrix
// the dynamics uses.
int build_model_tc(edus_batch* b, const Problem& P, const Inst& I) {
  const int n = P.ncv, nt = n * (n + 1) / 2, nk = P.nk, nr = P.nrpts;
  // H and D on the tensor cores; dH/dk, an observable-only table whose k sums
  // cancel strongly, is the reference's stencil over an FP64 H(k) (CUDA cores)
  const int ncomp = 4;
  const int kp = tc_pad_k(nr), kseg = tc_seg_k(nr), ncols = 2 * ncomp * nt, K = 2 * nr;
  std::vector<uint16_t> Bw((size_t)ncols * kp, 0);
  std::vector<double> col(K);
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) {
      const int e = tri_index(i, j, n);
      for (int comp = 0; comp < ncomp; comp++) {
        const int ce = comp * nt + e;
        for (int part = 0; part < 2; part++) {
          // re column: [Re c ; -Im c], im column: [Im c ; Re c]
          double amax = 0.;
          for (int r = 0; r < nr; r++) {
            const cd c = comp == 0 ? P.HR[((size_t)i * n + j) * nr + r]
                                   : 0.5 * (P.rR[(((size_t)(comp - 1) * n + i) * n + j) * nr + r] +
                                            P.rR[(((size_t)(comp - 1) * n + j) * n + i) * nr + r]);
            col[r] = part == 0 ? c.real() : c.imag();
            col[nr + r] = part == 0 ? -c.imag() : c.real();
            amax = std::max(amax, std::max(std::fabs(col[r]), std::fabs(col[nr + r])));
          }
          // power-of-two scale of the column: every y = value / scale in [-1/2, 1/2), so every
          // slice is at most 128 in magnitude; the phases enter halved, so the stored
          // slices carry 2 scale
          const double scale = amax > 0. ? std::ldexp(1.0, std::ilogb(amax) + 2) : 1.0;
          uint16_t* row = &Bw[(size_t)(2 * ce + part) * kp];
          for (int p = 0; p < kTcPairs; p++)
            for (int q = 0; q < K; q++) row[(size_t)p * kseg + q] = tc_bf16(2.0 * scale * tc_slice(col[q] / scale, tc_pair_b(p)));
        }
      }
    }
  std::vector<double2> hdr((size_t)n * nr);
  for (int i = 0; i < n; i++)
    for (int r = 0; r < nr; r++) hdr[(size_t)i * nr + r] = mkc<double2>(P.HR[((size_t)i * n + i) * nr + r]);
  std::vector<double> gb((size_t)P.nnb * 3);
  for (int bb = 0; bb < P.nnb; bb++)
    for (int x = 0; x < 3; x++) gb[bb * 3 + x] = P.shell_w[P.bshell[bb]] * P.bvec[bb * 3 + x];
  const size_t plane = (size_t)nt * nk;
  const size_t bytes = align256(sizeof(double) * 3 * nk) + align256(sizeof(double) * 3 * nr) + align256(sizeof(uint16_t) * Bw.size()) +
                       align256(sizeof(double2) * hdr.size()) + align256(sizeof(double) * gb.size()) +
                       align256(sizeof(uint16_t) * (size_t)nk * kp) + align256(sizeof(double) * (size_t)nk * ncols) +
                       align256(sizeof(double2) * plane) + align256(sizeof(double2) * n * n * nk) +
                       (I.GE ? align256(sizeof(double2) * plane) + align256(sizeof(double2) * 3 * plane) +
                                   align256(sizeof(double2) * 4 * nt * nr)
                             : 0);
  char* base = nullptr;
  if (cudaMallocAsync((void**)&base, bytes, b->pool, b->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(EDUS_ENOMEM, "batch: tensor-core model build scratch of %zu bytes", bytes);
  }
  char* p = base;
  auto carve = [&](size_t sz) {
    char* r = p;
    p += align256(sz);
    return r;
  };
  double* dk = (double*)carve(sizeof(double) * 3 * nk);
  double* dR = (double*)carve(sizeof(double) * 3 * nr);
  uint16_t* dB = (uint16_t*)carve(sizeof(uint16_t) * Bw.size());
  double2* dh = (double2*)carve(sizeof(double2) * hdr.size());
  double* dg = (double*)carve(sizeof(double) * gb.size());
  int rc;
  if ((rc = put(b, dk, P.kpt)) || (rc = put(b, dR, P.Rvec)) || (rc = put(b, dB, Bw)) || (rc = put(b, dh, hdr)) || (rc = put(b, dg, gb))) {
    cudaFreeAsync(base, b->stream);
    return rc;
  }
  TcArgs t;
  t.n = n;
  t.ntri = nt;
  t.nk = nk;
  t.nr = nr;
  t.kpt = dk;
  t.Rvec = dR;
  t.Bw = dB;
  t.hdiagR = dh;
  t.Aw = (uint16_t*)carve(sizeof(uint16_t) * (size_t)nk * kp);
  t.Cw = (double*)carve(sizeof(double) * (size_t)nk * ncols);
  t.H32 = (float2*)I.H;
  t.D32 = (float2*)I.D;
  t.Hdiag = (double*)I.Hdiag;
  t.Hused = (double2*)carve(sizeof(double2) * plane);
  t.err = b->d_err;
  ModelBuildArgs a;
  memset(&a, 0, sizeof(a));
  a.n = n;
  a.ntri = nt;
  a.nk = nk;
  a.nr = nr;
  a.nnb = P.nnb;
  a.nbands = P.nbands;
  a.nv = P.p.nb[1];
  a.scissor = 0.;
  a.kpt = dk;
  a.Rvec = dR;
  a.nbr = I.nbr;
  a.gb = dg;
  a.H = t.Hused;
  a.U = (double2*)carve(sizeof(double2) * n * n * nk);
  a.GE = nullptr;
  a.P0 = I.P0;
  cudaError_t e = tc_contract(t, b->stream);
  if (e == cudaSuccess) e = finish_wannier_model(a, b->stream);
  if (e == cudaSuccess) e = planes_to_float(a.U, (float2*)I.U, (size_t)n * n * nk, b->stream);
  if (e == cudaSuccess && I.GE) {
    // dH/dk: FP64 H(k) (coefficients: H(R) upper elements) and the stencil
    std::vector<double2> hc((size_t)nt * nr);
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++)
        for (int r = 0; r < nr; r++) hc[(size_t)tri_index(i, j, n) * nr + r] = mkc<double2>(P.HR[((size_t)i * n + j) * nr + r]);
    ModelBuildArgs g = a;
    g.only_h = 1;
    g.H = (double2*)carve(sizeof(double2) * plane);
    g.GE = (double2*)carve(sizeof(double2) * 3 * plane);
    double2* dhc = (double2*)carve(sizeof(double2) * 4 * nt * nr);
    int prc = put(b, dhc, hc);
    if (prc) {
      cudaFreeAsync(base, b->stream);
      return prc;
    }
    g.coef = dhc;
    e = wannier_h_and_gradient(g, b->stream);
    if (e == cudaSuccess) e = planes_to_float(g.GE, (float2*)I.GE, 3 * plane, b->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync((void*)I.Peq, I.P0, sizeof(double2) * plane, cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(I.P0, 0, sizeof(double2) * plane, b->stream);  // deviation = 0
  cudaFreeAsync(base, b->stream);
  if (e != cudaSuccess) return fail(EDUS_ECUDA, "batch: tensor-core model build: %s", cudaGetErrorString(e));
  return 0;
}

// Deferred Wannier model: tabulate H, D, U, dH/dk and the initial state on the
// device (cuda/model_build.cu) straight into the instance's tables; mixed
// precision goes through FP64 scratch and is rounded once.
int build_model_on_device(edus_batch* b, const Problem& P, const Inst& I) {
  const int n = P.ncv, nt = n * (n + 1) / 2, nk = P.nk, nr = P.nrpts;
  std::vector<double2> coef((size_t)4 * nt * nr);
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) {
      const int e = tri_index(i, j, n);
      for (int r = 0; r < nr; r++) {
        coef[(size_t)e * nr + r] = mkc<double2>(P.HR[((size_t)i * n + j) * nr + r]);
        for (int x = 0; x < 3; x++) {
          const cd v = 0.5 * (P.rR[(((size_t)x * n + i) * n + j) * nr + r] + P.rR[(((size_t)x * n + j) * n + i) * nr + r]);
          coef[((size_t)(1 + x) * nt + e) * nr + r] = mkc<double2>(v);
        }
      }
    }
  std::vector<double> gb((size_t)P.nnb * 3);
  for (int bb = 0; bb < P.nnb; bb++)
    for (int x = 0; x < 3; x++) gb[bb * 3 + x] = P.shell_w[P.bshell[bb]] * P.bvec[bb * 3 + x];
  const size_t plane = (size_t)nt * nk;
  // scratch: inputs, and FP64 outputs when the instance stores FP32
  size_t bytes = align256(sizeof(double) * 3 * nk) + align256(sizeof(double) * 3 * nr) + align256(sizeof(double2) * coef.size()) +
                 align256(sizeof(double) * gb.size());
  const bool mix = cmix(b, n);
  if (mix) bytes += align256(sizeof(double2) * plane) * (4 + (I.GE ? 3 : 0)) + align256(sizeof(double2) * n * n * nk);
  char* base = nullptr;
  if (cudaMallocAsync((void**)&base, bytes, b->pool, b->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(EDUS_ENOMEM, "batch: model build scratch of %zu bytes", bytes);
  }
  char* p = base;
  auto carve = [&](size_t sz) {
    char* r = p;
    p += align256(sz);
    return r;
  };
  ModelBuildArgs a;
  memset(&a, 0, sizeof(a));
  a.n = n;
  a.ntri = nt;
  a.nk = nk;
  a.nr = nr;
  a.nnb = P.nnb;
  a.nbands = P.nbands;
  a.nv = P.p.nb[1];
  a.scissor = P.p.conduction_shift;
  double* dk = (double*)carve(sizeof(double) * 3 * nk);
  double* dR = (double*)carve(sizeof(double) * 3 * nr);
  double2* dc = (double2*)carve(sizeof(double2) * coef.size());
  double* dg = (double*)carve(sizeof(double) * gb.size());
  int rc;
  if ((rc = put(b, dk, P.kpt)) || (rc = put(b, dR, P.Rvec)) || (rc = put(b, dc, coef)) || (rc = put(b, dg, gb))) {
    cudaFreeAsync(base, b->stream);
    return rc;
  }
  a.kpt = dk;
  a.Rvec = dR;
  a.coef = dc;
  a.gb = dg;
  a.nbr = I.nbr;
  a.P0 = I.P0;
  if (mix) {
    a.H = (double2*)carve(sizeof(double2) * plane);
    a.D = (double2*)carve(sizeof(double2) * 3 * plane);
    a.U = (double2*)carve(sizeof(double2) * n * n * nk);
    a.GE = I.GE ? (double2*)carve(sizeof(double2) * 3 * plane) : nullptr;
  } else {
    a.H = (double2*)I.H;
    a.D = (double2*)I.D;
    a.U = (double2*)I.U;
    a.GE = (double2*)I.GE;
  }
  cudaError_t e = build_wannier_model(a, b->stream);
  if (e == cudaSuccess && mix) {
    if (e == cudaSuccess) e = planes_diagonal(a.H, (double*)I.Hdiag, n, nk, b->stream);
    if (e == cudaSuccess) e = planes_to_float(a.H, (float2*)I.H, plane, b->stream);
    if (e == cudaSuccess) e = planes_to_float(a.D, (float2*)I.D, 3 * plane, b->stream);
    if (e == cudaSuccess) e = planes_to_float(a.U, (float2*)I.U, (size_t)n * n * nk, b->stream);
    if (e == cudaSuccess && I.GE) e = planes_to_float(a.GE, (float2*)I.GE, 3 * plane, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync((void*)I.Peq, I.P0, sizeof(double2) * plane, cudaMemcpyDeviceToDevice, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(I.P0, 0, sizeof(double2) * plane, b->stream);  // deviation = 0
  }
  cudaFreeAsync(base, b->stream);
  if (e != cudaSuccess) return fail(EDUS_ECUDA, "batch: device model build: %s", cudaGetErrorString(e));
  return 0;
}

void free_slot_mem(edus_batch* b, Slot& s) {
  for (void* p : s.mem) cudaFreeAsync(p, b->stream);
  s.mem.clear();
}

int sync_tiles(edus_batch* b) {
  for (auto& kv : b->classes) {
    ClassTab& c = kv.second;
    if (!c.dirty) continue;
    if (c.tiles.size() > c.cap) {
      size_t cap = std::max<size_t>(1024, c.cap);
      while (cap < c.tiles.size()) cap *= 2;
      Tile* nt = nullptr;
      BCK(cudaMallocAsync((void**)&nt, cap * sizeof(Tile), b->pool, b->stream));
      if (c.d_tiles) cudaFreeAsync(c.d_tiles, b->stream);
      c.d_tiles = nt;
      c.cap = cap;
    }
    if (!c.tiles.empty()) BCK(cudaMemcpyAsync(c.d_tiles, c.tiles.data(), c.tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, b->stream));
    // instance table: the runs of equal slots in the tile table
    c.insts.clear();
    for (size_t t = 0; t < c.tiles.size();) {
      size_t u = t;
      while (u < c.tiles.size() && c.tiles[u].inst == c.tiles[t].inst) u++;
      const Slot& sl = b->slots[c.tiles[t].inst];
      const int uk = obs_unit(c.n);
      c.insts.push_back(ClassInst{c.tiles[t].inst, (sl.nk + uk - 1) / uk, sl.itfi, sl.res});
      t = u;
    }
    if (!c.insts.empty())
      BCK(cudaMemcpyAsync(c.d_cinst, c.insts.data(), c.insts.size() * sizeof(ClassInst), cudaMemcpyHostToDevice, b->stream));
    const int counts[2] = {(int)c.tiles.size(), (int)c.insts.size()};
    BCK(cudaMemcpyAsync(c.d_ntiles, counts, sizeof(counts), cudaMemcpyHostToDevice, b->stream));
    // pageable sources: the copies have left the host buffers before the calls return
    int psel = 1, pcomp = 1;
    const int form = form_of(b, c, psel, pcomp);
    if (form != c.form || psel != c.psel || pcomp != c.pcomp) {
      c.form = form;
      c.psel = psel;
      c.pcomp = pcomp;
      c.sgrid = grid_of(b, c);
      if (c.sgrid <= 0) return fail(EDUS_ECUDA, "batch: no resident block for %d bands (form %d)", c.n, c.form);
    }
    c.dirty = false;
  }
  return 0;
}

std::string graph_key(const edus_batch* b) {
  std::string k;
  for (const auto& kv : b->classes) {
    char buf[96];
    snprintf(buf, sizeof(buf), "%d:%d:%d:%d:%d:%p;", kv.second.n, kv.second.kt, kv.second.form, kv.second.psel, kv.second.pcomp,
             (const void*)kv.second.d_tiles);
    k += buf;
  }
  return k;
}

// CUDA-event pairs around individual launches (edus_batch_profile): pair i
// brackets one launch of kernel kind[i] (0 observables, 1-4 stage 0-3) of class nb[i]
struct LaunchTimer {
  std::vector<cudaEvent_t> ev;
  std::vector<int> nb, kind;
  size_t used = 0;
  ~LaunchTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
  cudaError_t begin(int n, int k, cudaStream_t s) {
    while (ev.size() < 2 * (used + 1)) {
      cudaEvent_t e;
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return r;
      ev.push_back(e);
    }
    if (nb.size() <= used) {
      nb.resize(used + 1);
      kind.resize(used + 1);
    }
    nb[used] = n;
    kind[used] = k;
    return cudaEventRecord(ev[2 * used], s);
  }
  cudaError_t end(cudaStream_t s) { return cudaEventRecord(ev[2 * used++ + 1], s); }
};

int record_chunk(edus_batch* b, LaunchTimer* tm = nullptr) {
  const int S = b->opt.chunk_steps;
  for (int s = 0; s < S; s++) {
    const int parity = s & 1;
    for (auto& kv : b->classes) {
      ClassTab& c = kv.second;
      View v{b->d_insts, {b->d_it[0], b->d_it[1]}, c.d_tiles, c.d_ntiles, c.d_cinst, c.d_ntiles + 1};
      if (tm) BCK(tm->begin(c.n, 0, b->stream));
      BCK(launch_obs(c.n, c.kt, cmix(b, c.n), v, parity, (int)b->slots.size(), c.ogrid, b->stream));
      if (tm) BCK(tm->end(b->stream));
    }
    for (int st = 0; st < 4; st++)
      for (auto& kv : b->classes) {
        ClassTab& c = kv.second;
        View v{b->d_insts, {b->d_it[0], b->d_it[1]}, c.d_tiles, c.d_ntiles, c.d_cinst, c.d_ntiles + 1};
        if (tm) BCK(tm->begin(c.n, 1 + st, b->stream));
        if (c.form >= 3 && c.form <= 5)
          BCK(launch_stage_pipe(c.n, c.kt, pipe_cb(c.form), v, st, parity, c.psel, c.pcomp, c.sgrid, b->stream));
        else if (c.form == 2)
          BCK(launch_stage_mm(c.n, c.kt, cmix(b, c.n), v, st, parity, c.sgrid, b->stream));
        else
          BCK(launch_stage(c.n, c.kt, c.form, cmix(b, c.n), v, st, parity, c.sgrid, b->stream));
        if (tm) BCK(tm->end(b->stream));
      }
  }
  return 0;
}

int run_chunk(edus_batch* b, LaunchTimer* tm = nullptr) {
  int rc = sync_tiles(b);
  if (rc) return rc;
  bool any = false;
  for (auto& kv : b->classes) any = any || kv.second.d_tiles;
  if (!any) return 0;
  const std::string key = graph_key(b);
  BCK(cudaEventRecord(b->e0, b->stream));
  if (tm) {
    if ((rc = record_chunk(b, tm))) return rc;
  } else if (b->opt.use_graphs) {
    if (!b->gexec || key != b->graph_key) {
      if (b->gexec) cudaGraphExecDestroy(b->gexec);
      if (b->graph) cudaGraphDestroy(b->graph);
      b->gexec = nullptr;
      b->graph = nullptr;
      BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      rc = record_chunk(b);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return fail(EDUS_ECUDA, "capture of the batch chunk: %s", cudaGetErrorString(e));
      b->graph = g;
      BCK(cudaGraphInstantiate(&b->gexec, g, 0));
      b->graph_key = key;
    }
    BCK(cudaGraphLaunch(b->gexec, b->stream));
  } else {
    if ((rc = record_chunk(b))) return rc;
  }
  BCK(cudaEventRecord(b->e1, b->stream));
  BCK(cudaEventSynchronize(b->e1));
  int derr = 0;
  BCK(cudaMemcpy(&derr, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (derr) return fail(EDUS_ETIMEOUT, "batch: a bounded device wait ran out (error %d)", derr);
  float ms = 0;
  BCK(cudaEventElapsedTime(&ms, b->e0, b->e1));
  b->device_ms += ms;
  const int S = b->opt.chunk_steps;
  b->launches += (long long)S * 5 * b->classes.size();
  // progress of every running instance over this chunk
  for (size_t q = 0; q < b->slots.size(); q++) {
    Slot& s = b->slots[q];
    if (s.status != EDUS_INST_RUNNING) continue;
    const long long it0 = b->tick - s.tick_admit;
    const long long steps = std::max(0LL, std::min<long long>(S, (long long)s.itfi + 1 - it0));
    b->kpoint_steps += (double)steps * s.nk;
  }
  b->tick += S;
  // retire instances past the end of their time grid
  for (size_t q = 0; q < b->slots.size(); q++) {
    Slot& s = b->slots[q];
    if (s.status == EDUS_INST_RUNNING && b->tick - s.tick_admit > s.itfi) {
      s.status = EDUS_INST_DONE;
      ClassTab& c = b->classes[s.n];
      c.tiles.erase(std::remove_if(c.tiles.begin(), c.tiles.end(), [&](const Tile& t) { return t.inst == (int)q; }), c.tiles.end());
      c.dirty = true;
    }
  }
  return 0;
}

Slot* slot_of(edus_batch* b, int32_t slot) {
  if (!b || slot < 0 || slot >= (int)b->slots.size()) return nullptr;
  return &b->slots[slot];
}

int occupy_slot(edus_batch* b, int q, edus_ctx* ctx, const Problem& P, int64_t tag, int32_t* slot_out);

// An instance with the Coulomb mean field: its own FP64 context, the whole loop
// launched at once on the context's stream (it runs beside the chunk graphs and
// is retired by polling). Its result equals edus_run's on the same problem.
int add_coulomb(edus_batch* b, const edus_problem* pb, int64_t tag, int32_t* slot_out) {
  const Problem& P = pb->P;
  const int64_t est = ctx_footprint_estimate(P);
  if (b->bytes_used + est > b->budget)
    return fail(EDUS_ENOMEM, "batch: %lld bytes do not fit the HBM budget (%lld of %lld used)", (long long)est,
                (long long)b->bytes_used, (long long)b->budget);
  int q = -1;
  for (size_t i = 0; i < b->slots.size(); i++)
    if (b->slots[i].status == EDUS_INST_FREE) {
      q = (int)i;
      break;
    }
  if (q < 0) return fail(EDUS_ENOMEM, "batch: all %zu slots are in use", b->slots.size());
  edus_options o;
  edus_options_default(&o);
  o.device = b->device;
  o.use_graphs = 1;
  edus_ctx* ctx = nullptr;
  int rc = edus_create(pb, &o, &ctx);
  if (rc) return rc;
  const int64_t bytes = (int64_t)ctx_device_bytes(ctx);
  if (b->bytes_used + bytes > b->budget) {
    edus_destroy(ctx);
    return fail(EDUS_ENOMEM, "batch: %lld bytes do not fit the HBM budget", (long long)bytes);
  }
  if ((rc = ctx_start_async(ctx))) {
    edus_destroy(ctx);
    return rc;
  }
  return occupy_slot(b, q, ctx, P, tag, slot_out);
}

// Slot q takes a started Coulomb context.
int occupy_slot(edus_batch* b, int q, edus_ctx* ctx, const Problem& P, int64_t tag, int32_t* slot_out) {
  const int64_t bytes = (int64_t)ctx_device_bytes(ctx);
  Slot s;
  s.n = P.ncv;
  s.nk = P.nk;
  s.ntri = P.ncv * (P.ncv + 1) / 2;
  s.itfi = P.itfi;
  s.res = std::max(1, P.p.it_resolution);
  s.nlog = s.itfi / s.res + 1;
  s.tag = tag;
  s.bytes = bytes;
  s.sub = ctx;
  s.status = EDUS_INST_RUNNING;
  s.tick_admit = b->tick;
  b->bytes_used += bytes;
  b->slots[q] = std::move(s);
  *slot_out = q;
  return 0;
}

}  // namespace

namespace edus {

int batch_adopt_context(edus_batch* b, edus_ctx* ctx, const Problem& P, int64_t tag, int32_t* slot_out) {
  if (!b || !ctx || !slot_out) return fail(EDUS_EINVAL, "null argument");
  for (size_t i = 0; i < b->slots.size(); i++)
    if (b->slots[i].status == EDUS_INST_FREE) return occupy_slot(b, (int)i, ctx, P, tag, slot_out);
  return fail(EDUS_ENOMEM, "batch: all %zu slots are in use", b->slots.size());
}

}  // namespace edus

namespace {
int poll_subs(edus_batch* b, bool wait);
}

namespace edus {

bool batch_has_tiles(const edus_batch* b) {
  for (const auto& kv : b->classes)
    if (!kv.second.tiles.empty()) return true;
  return false;
}

int batch_poll_contexts(edus_batch* b) {
  BCK(cudaSetDevice(b->device));
  return poll_subs(b, false);
}

}  // namespace edus

namespace {

// Retire the Coulomb instances whose run has ended; with wait, block until the
// earliest-admitted running one has ended (the batch has no other work).
int poll_subs(edus_batch* b, bool wait) {
  Slot* first = nullptr;
  for (auto& s : b->slots) {
    if (!s.sub || s.status != EDUS_INST_RUNNING) continue;
    bool done = false;
    int rc = ctx_poll(s.sub, &done);
    if (rc) return rc;
    if (done) {
      s.status = EDUS_INST_DONE;
      b->kpoint_steps += (double)s.nk * (s.itfi + 1);
    } else if (!first || s.tick_admit < first->tick_admit) {
      first = &s;
    }
  }
  if (wait && first) {
    int rc = ctx_wait(first->sub);
    if (rc) return rc;
    first->status = EDUS_INST_DONE;
    b->kpoint_steps += (double)first->nk * (first->itfi + 1);
  }
  return 0;
}

}  // namespace

extern "C" {

int edus_batch_options_default(edus_batch_options* o) {
  if (!o) return fail(EDUS_EINVAL, "null argument");
  memset(o, 0, sizeof(*o));
  o->device = 0;
  o->precision = EDUS_PREC_FP64;
  o->max_instances = 1024;
  o->chunk_steps = 16;
  o->use_graphs = 1;
  o->tc_contraction = 1;
  o->hbm_budget_bytes = 0;
  return 0;
}

int edus_batch_create(const edus_batch_options* o, edus_batch** out) {
  if (!o || !out) return fail(EDUS_EINVAL, "null argument");
  if (o->max_instances <= 0 || o->chunk_steps <= 0 || (o->chunk_steps & 1))
    return fail(EDUS_EINVAL, "batch: max_instances > 0 and an even chunk_steps are required");
  if (o->precision != EDUS_PREC_FP64 && o->precision != EDUS_PREC_MIXED) return fail(EDUS_EINVAL, "batch: unknown precision");
  edus_batch* b = new edus_batch();
  b->opt = *o;
  b->mixed = o->precision == EDUS_PREC_MIXED;
  b->device = o->device;
  auto bail = [&](int rc) {
    edus_batch_destroy(b);
    return rc;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return bail(fail(EDUS_ECUDA, "cannot select device %d", b->device));
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(EDUS_ECUDA, "stream"));
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = b->device;
  if (cudaMemPoolCreate(&b->pool, &props) != cudaSuccess) return bail(fail(EDUS_ECUDA, "memory pool"));
  uint64_t keep = ~0ull;
  cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  b->budget = o->hbm_budget_bytes > 0 ? o->hbm_budget_bytes : (int64_t)(0.9 * (double)fr);
  const int cap = o->max_instances;
  b->slots.resize(cap);
  if (cudaMalloc(&b->d_insts, sizeof(Inst) * cap) != cudaSuccess || cudaMalloc(&b->d_it[0], sizeof(int) * cap) != cudaSuccess ||
      cudaMalloc(&b->d_it[1], sizeof(int) * cap) != cudaSuccess || cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess)
    return bail(fail(EDUS_ENOMEM, "batch tables"));
  cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream);
  cudaMemsetAsync(b->d_insts, 0, sizeof(Inst) * cap, b->stream);
  cudaMemsetAsync(b->d_it[0], 0xff, sizeof(int) * cap, b->stream);
  cudaMemsetAsync(b->d_it[1], 0xff, sizeof(int) * cap, b->stream);
  if (cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) return bail(fail(EDUS_ECUDA, "events"));
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(fail(EDUS_ECUDA, "sync"));
  *out = b;
  return 0;
}

void edus_batch_destroy(edus_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto& s : b->slots) {
    if (s.sub) edus_destroy(s.sub);
    s.sub = nullptr;
    free_slot_mem(b, s);
  }
  for (auto& kv : b->classes) {
    if (kv.second.d_tiles) cudaFreeAsync(kv.second.d_tiles, b->stream);
    if (kv.second.d_ntiles) cudaFree(kv.second.d_ntiles);
    if (kv.second.d_cinst) cudaFree(kv.second.d_cinst);
  }
  if (b->stream) cudaStreamSynchronize(b->stream);
  cudaFree(b->d_insts);
  cudaFree(b->d_it[0]);
  cudaFree(b->d_it[1]);
  cudaFree(b->d_err);
  if (b->pool) cudaMemPoolDestroy(b->pool);
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int edus_batch_footprint(edus_batch* b, const edus_problem* pb, int64_t* bytes) {
  if (!b || !pb || !bytes) return fail(EDUS_EINVAL, "null argument");
  int rc = check_problem(b, pb->P);
  if (rc) return rc;
  *bytes = pb->P.p.coulomb ? ctx_footprint_estimate(pb->P) : (int64_t)layout_of(b, pb->P, tile_len(b, pb->P.ncv)).total();
  return 0;
}

int edus_batch_add(edus_batch* b, const edus_problem* pb, int64_t tag, int32_t* slot_out) {
  if (!b || !pb || !slot_out) return fail(EDUS_EINVAL, "null argument");
  const Problem& P = pb->P;
  int rc = check_problem(b, P);
  if (rc) return rc;
  if (P.p.coulomb) return add_coulomb(b, pb, tag, slot_out);
  const int n = P.ncv, nk = P.nk, nt = n * (n + 1) / 2, kt = tile_len(b, n);
  const Layout L = layout_of(b, P, kt);
  const int64_t bytes = (int64_t)L.total();
  if (b->bytes_used + bytes > b->budget)
    return fail(EDUS_ENOMEM, "batch: %lld bytes do not fit the HBM budget (%lld of %lld used)", (long long)bytes,
                (long long)b->bytes_used, (long long)b->budget);
  int q = -1;
  for (size_t i = 0; i < b->slots.size(); i++)
    if (b->slots[i].status == EDUS_INST_FREE) {
      q = (int)i;
      break;
    }
  if (q < 0) return fail(EDUS_ENOMEM, "batch: all %zu slots are in use", b->slots.size());
  BCK(cudaSetDevice(b->device));
  Slot s;
  s.n = n;
  s.kt = kt;
  s.nk = nk;
  s.ntri = nt;
  s.itfi = P.itfi;
  s.res = std::max(1, P.p.it_resolution);
  s.nlog = s.itfi / s.res + 1;
  s.ntiles = (nk + kt - 1) / kt;
  s.tag = tag;
  s.bytes = bytes;
  // one allocation, carved in the layout order
  char* base = nullptr;
  if (cudaMallocAsync((void**)&base, L.total(), b->pool, b->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(EDUS_ENOMEM, "batch: device allocation of %lld bytes failed", (long long)bytes);
  }
  s.mem.push_back(base);
  char* p = base;
  auto carve = [&](size_t sz) {
    char* r = sz ? p : nullptr;
    p += sz;
    return r;
  };
  Inst& I = s.inst;
  memset(&I, 0, sizeof(I));
  I.n = n;
  I.ntri = nt;
  I.nk = nk;
  I.nnb = P.nnb;
  I.nch = P.nch;
  I.nbands = P.nbands;
  I.itfi = P.itfi;
  I.res = s.res;
  I.want_current = P.p.current;
  I.want_tabs = P.p.tabs && P.nch > 0;
  I.ntiles = s.ntiles;
  I.dt = P.p.dt;
  I.dt6 = P.p.dt / 6.0;
  I.dt3 = P.p.dt / 3.0;
  I.wx2 = P.p.probe.wl;
  I.scaleJ = P.dk[0] * P.dk[1] * P.dk[2] / P.det_a;
  I.scaleTA = std::fabs(P.jac) * P.dk[0] * P.dk[1] * P.dk[2];
  I.P0 = (double2*)carve(L.state);
  I.P1 = (double2*)carve(L.state);
  I.Pa = (double2*)carve(L.state);
  I.Pb = (double2*)carve(L.state);
  I.Peq = (const double2*)carve(L.eq);
  I.Hdiag = (const double*)carve(L.hdiag);
  I.W = carve(L.w);
  I.H = carve(L.H);
  I.D = carve(L.D);
  I.GE = carve(L.GE);
  I.U = carve(L.U);
  I.nbr = (const int*)carve(L.nbr);
  I.field = (const FieldRow*)carve(L.field);
  I.log = (edus_obs*)carve(L.log);
  I.part = carve(L.part);
  I.done = (unsigned int*)carve(256);
  for (int bb = 0; bb < P.nnb; bb++) {
    I.wb[bb] = P.shell_w[P.bshell[bb]];
    for (int x = 0; x < 3; x++) I.bvec[bb][x] = P.bvec[bb * 3 + x];
  }
  detect_lattice(P, I);
  if (!I.lattice && !class_supported(n, kt))
    return fail(EDUS_EUNSUPPORTED, "batch: %d k points per tile needs a lattice stencil for %d bands", kt, n);
  auto undo = [&](int code) {
    free_slot_mem(b, s);
    return code;
  };
  // neighbour table, then model tables and initial state (host-built, or
  // tabulated on the device from H(R), r(R) for a deferred Wannier model)
  {
    std::vector<int> nb((size_t)P.nnb * nk);
    for (int k = 0; k < nk; k++)
      for (int bb = 0; bb < P.nnb; bb++) nb[(size_t)bb * nk + k] = P.nbr[(size_t)k * P.nnb + bb];
    if ((rc = put(b, (void*)I.nbr, nb))) return undo(rc);
  }
  if (P.model_deferred) {
    // (the exact segment sums hold up to 1024-deep segments, 512 R vectors)
    const bool tc = cmix(b, n) && b->opt.tc_contraction && P.p.conduction_shift <= 1e-16 && tc_seg_k(P.nrpts) <= 1024;
    if ((rc = tc ? build_model_tc(b, P, I) : build_model_on_device(b, P, I))) return undo(rc);
  } else {
    rc = cmix(b, n) ? upload_model<float2>(b, P, I) : upload_model<double2>(b, P, I);
    if (rc) return undo(rc);
    std::vector<double2> st;
    planes<double2>(P.P0.data(), nk, n, 1, st);
    if (I.Peq) {
      // mixed precision: the state is the deviation from rho_eq
      if ((rc = put(b, (void*)I.Peq, st))) return undo(rc);
      if (cudaMemsetAsync(I.P0, 0, sizeof(double2) * st.size(), b->stream) != cudaSuccess)
        return undo(fail(EDUS_ECUDA, "batch: clear deviation"));
    } else if ((rc = put(b, I.P0, st))) {
      return undo(rc);
    }
  }
  // mixed precision: Pb starts as the FP32 copy of the deviation P0 = 0 that
  // stage 0 reads (stage 3 refreshes it every step)
  if (cmix(b, n) && cudaMemsetAsync(I.Pb, 0, L.state, b->stream) != cudaSuccess)
    return undo(fail(EDUS_ECUDA, "batch: clear stage input"));
  {
    // field table: the single-solve loop's times (t += dt) and fields
    std::vector<FieldRow> fr((size_t)P.itfi + 2);
    double t = P.t_start;
    for (auto& row : fr) {
      memset(&row, 0, sizeof(row));
      row.t = t;
      double E[2][3];
      field_at(P.p, t, E);
      for (int x = 0; x < 6; x++) row.Et[x] = E[x / 3][x % 3];
      field_at(P.p, t + P.p.dt / 2.0, E);
      for (int x = 0; x < 6; x++) row.Eh[x] = E[x / 3][x % 3];
      t += P.p.dt;
    }
    if ((rc = put(b, (void*)I.field, fr))) return undo(rc);
    select_terms(P, fr, I, cmix(b, n));
  }
  if (cudaMemsetAsync(I.done, 0, sizeof(unsigned int), b->stream) != cudaSuccess ||
      cudaMemcpyAsync(b->d_insts + q, &I, sizeof(Inst), cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
    return undo(fail(EDUS_ECUDA, "batch: upload of the instance descriptor"));
  b->h2d_bytes += (long long)sizeof(Inst);
  if (cmix(b, n) && launch_weq(b->d_insts, q, nt, nk, b->stream) != cudaSuccess)
    return undo(fail(EDUS_ECUDA, "batch: equilibrium terms"));
  const int zero = 0;
  if (cudaMemcpyAsync(b->d_it[b->tick & 1] + q, &zero, sizeof(int), cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
    return undo(fail(EDUS_ECUDA, "batch: clock"));
  // tiles
  ClassTab& c = b->classes[n];
  if (!c.n) {
    c.n = n;
    c.kt = kt;
    c.occ = profile_of(b, n);
    c.form = -1;  // chosen with the tile table, before the next chunk
    c.ogrid = obs_grid(n, cmix(b, n), (int)b->slots.size());
    if (c.ogrid <= 0) return undo(fail(EDUS_ECUDA, "batch: no resident block of the observable kernel for %d bands", n));
    if (cudaMalloc(&c.d_ntiles, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c.d_cinst, b->slots.size() * sizeof(ClassInst)) != cudaSuccess)
      return undo(fail(EDUS_ENOMEM, "tile count"));
  }
  for (int t = 0; t < s.ntiles; t++) c.tiles.push_back(Tile{q, t * kt, t, interior_tile(I, t * kt, kt)});
  c.dirty = true;
  s.status = EDUS_INST_RUNNING;
  s.tick_admit = b->tick;
  b->bytes_used += bytes;
  b->slots[q] = std::move(s);
  *slot_out = q;
  return 0;
}

int edus_batch_advance(edus_batch* b, int32_t nsteps) {
  if (!b || nsteps < 0) return fail(EDUS_EINVAL, "bad argument");
  BCK(cudaSetDevice(b->device));
  const int S = b->opt.chunk_steps;
  bool tiles = false;
  for (auto& kv : b->classes) tiles = tiles || !kv.second.tiles.empty();
  for (int done = 0; done < nsteps; done += S) {
    int rc = run_chunk(b);
    if (rc) return rc;
  }
  // with no tile of any class left, only Coulomb instances run: wait for one
  return poll_subs(b, !tiles && nsteps > 0);
}

int edus_batch_poll(edus_batch* b, int32_t slot, int32_t* status, int32_t* it, int64_t* tag) {
  Slot* s = slot_of(b, slot);
  if (!s) return fail(EDUS_EINVAL, "bad slot");
  if (status) *status = s->status;
  if (it) *it = s->status == EDUS_INST_FREE ? 0
                : (s->sub && s->status == EDUS_INST_DONE) ? s->itfi + 1
                                                          : (int32_t)std::min<long long>(b->tick - s->tick_admit, s->itfi + 1);
  if (tag) *tag = s->tag;
  return 0;
}

int edus_batch_obs_count(edus_batch* b, int32_t slot, int32_t* n) {
  Slot* s = slot_of(b, slot);
  if (!s || !n || s->status == EDUS_INST_FREE) return fail(EDUS_EINVAL, "bad slot");
  if (s->sub) {
    // a Coulomb instance's log is complete when its run has ended
    if (s->status != EDUS_INST_DONE) {
      *n = 0;
      return 0;
    }
    return edus_obs_count(s->sub, n);
  }
  const long long it = std::min<long long>(b->tick - s->tick_admit, s->itfi + 1);
  *n = (int32_t)std::min<long long>(s->nlog, (it + s->res - 1) / s->res);
  return 0;
}

int edus_batch_obs_get(edus_batch* b, int32_t slot, int32_t first, int32_t count, edus_obs* out) {
  Slot* s = slot_of(b, slot);
  if (!s || !out || s->status == EDUS_INST_FREE) return fail(EDUS_EINVAL, "bad slot");
  if (s->sub) {
    if (s->status != EDUS_INST_DONE) return fail(EDUS_EINVAL, "the Coulomb instance is still running");
    int rc = edus_obs_get(s->sub, first, count, out);
    if (!rc) b->d2h_bytes += (long long)(sizeof(edus_obs) * count);
    return rc;
  }
  if (first < 0 || count < 0 || first + count > s->nlog) return fail(EDUS_EINVAL, "range outside the log");
  BCK(cudaSetDevice(b->device));
  BCK(cudaMemcpyAsync(out, s->inst.log + first, sizeof(edus_obs) * count, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  b->d2h_bytes += (long long)(sizeof(edus_obs) * count);
  return 0;
}

int edus_batch_get_state(edus_batch* b, int32_t slot, double* rho) {
  Slot* s = slot_of(b, slot);
  if (!s || !rho || s->status == EDUS_INST_FREE) return fail(EDUS_EINVAL, "bad slot");
  if (s->sub) {
    int rc = edus_get_state(s->sub, rho);
    if (!rc) b->d2h_bytes += (long long)(16 * (size_t)s->nk * s->n * s->n);
    return rc;
  }
  BCK(cudaSetDevice(b->device));
  const int n = s->n, nk = s->nk;
  std::vector<double2> pl((size_t)s->ntri * nk);
  BCK(cudaMemcpyAsync(pl.data(), s->inst.P0, sizeof(double2) * pl.size(), cudaMemcpyDeviceToHost, b->stream));
  std::vector<double2> eq;
  if (s->inst.Peq) {
    // mixed precision keeps the deviation from rho_eq
    eq.resize(pl.size());
    BCK(cudaMemcpyAsync(eq.data(), s->inst.Peq, sizeof(double2) * eq.size(), cudaMemcpyDeviceToHost, b->stream));
  }
  BCK(cudaStreamSynchronize(b->stream));
  b->d2h_bytes += (long long)(sizeof(double2) * (pl.size() + eq.size()));
  for (size_t q = 0; q < eq.size(); q++) pl[q] = cadd(pl[q], eq[q]);
  cd* o = (cd*)rho;
  for (int k = 0; k < nk; k++)
    for (int i = 0; i < n; i++)
      for (int j = i; j < n; j++) {
        const double2 v = pl[(size_t)tri_index(i, j, n) * nk + k];
        o[((size_t)k * n + i) * n + j] = cd(v.x, v.y);
        if (i != j) o[((size_t)k * n + j) * n + i] = cd(v.x, -v.y);
      }
  return 0;
}

int edus_batch_release(edus_batch* b, int32_t slot) {
  Slot* s = slot_of(b, slot);
  if (!s) return fail(EDUS_EINVAL, "bad slot");
  if (s->status == EDUS_INST_FREE) return 0;
  BCK(cudaSetDevice(b->device));
  if (s->sub) {
    edus_destroy(s->sub);  // waits for the context's stream
    b->bytes_used -= s->bytes;
    *s = Slot();
    return 0;
  }
  if (s->status == EDUS_INST_RUNNING) {
    ClassTab& c = b->classes[s->n];
    c.tiles.erase(std::remove_if(c.tiles.begin(), c.tiles.end(), [&](const Tile& t) { return t.inst == slot; }), c.tiles.end());
    c.dirty = true;
    // the tile table is rewritten before the next chunk; nothing reads the slot after that
    int rc = sync_tiles(b);
    if (rc) return rc;
  }
  free_slot_mem(b, *s);
  b->bytes_used -= s->bytes;
  *s = Slot();
  return 0;
}

int edus_batch_stats_get(edus_batch* b, edus_batch_stats* out) {
  if (!b || !out) return fail(EDUS_EINVAL, "null argument");
  memset(out, 0, sizeof(*out));
  out->ticks = b->tick;
  for (const auto& s : b->slots) {
    if (s.status == EDUS_INST_RUNNING) out->active++;
    if (s.status == EDUS_INST_DONE) out->done++;
    if (s.status == EDUS_INST_FREE) out->free_slots++;
  }
  out->bytes_used = b->bytes_used;
  out->bytes_budget = b->budget;
  out->device_ms = b->device_ms;
  out->kpoint_steps = b->kpoint_steps;
  out->launches = b->launches;
  out->h2d_bytes = b->h2d_bytes;
  out->d2h_bytes = b->d2h_bytes;
  return 0;
}

int edus_batch_tile_k(edus_batch* b, int32_t nbands, int32_t* kt) {
  if (!b || !kt) return fail(EDUS_EINVAL, "null argument");
  *kt = tile_len(b, nbands);
  return 0;
}

int edus_batch_profile(edus_batch* b, int32_t nsteps, edus_kernel_time* out, int32_t cap, int32_t* n) {
  if (!b || nsteps < 0 || !out || cap < 0 || !n) return fail(EDUS_EINVAL, "bad argument");
  BCK(cudaSetDevice(b->device));
  std::map<std::pair<int, int>, edus_kernel_time> acc;
  const int S = b->opt.chunk_steps;
  for (int done = 0; done < nsteps; done += S) {
    // k points of each class in this chunk (before instances retire at its end)
    std::map<int, long long> kp;
    for (const auto& s : b->slots)
      if (s.status == EDUS_INST_RUNNING) kp[s.n] += s.nk;
    LaunchTimer tm;
    int rc = run_chunk(b, &tm);
    if (rc) return rc;
    for (size_t i = 0; i < tm.used; i++) {
      float ms = 0;
      BCK(cudaEventElapsedTime(&ms, tm.ev[2 * i], tm.ev[2 * i + 1]));
      edus_kernel_time& e = acc[{tm.nb[i], tm.kind[i]}];
      e.nbands = tm.nb[i];
      e.kind = tm.kind[i];
      e.launches++;
      e.total_ms += ms;
      e.kpoints = kp[tm.nb[i]];
    }
  }
  int m = 0;
  for (const auto& kv : acc)
    if (m < cap) out[m++] = kv.second;
  *n = m;
  return 0;
}

}  // extern "C"
