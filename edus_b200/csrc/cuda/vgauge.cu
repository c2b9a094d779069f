// vgauge.cu — velocity-gauge tables: H(k + A) and D(k + A) of a Wannier model
// at every k point of the grid, rebuilt for every RK4 stage.
//
// In the frame that moves with the vector potential, rho'(k, t) = rho(k + A(t), t)
// with A = -int E_pump dt, the length-gauge k-gradient term cancels and the
// model enters at k + A (the reference only integrates the length gauge; its
// Laser::A_crys, headers/Laser.h:191-213, is called from dead code). The
// tables are the reference's Fourier sums (headers/Wannier.h:278-304,336-471)
// with the imaginary part of the diagonal dropped (:489-492, :577-578) and
// the dipole made symmetric (Source_Main/save_HUD.cpp:47-51), here folded into
// the coefficients: c_x(R) = (r_x(R) + r_x(R)^T) / 2.
//
// One block per tile of KT consecutive k points; thread (kl, e) accumulates
// the four sums of upper-triangle element e for k point kl. The phases
// e^{2 pi i (k + A).R} of the tile's k points are computed for 32 R vectors at
// a time into shared memory and used by every element; each sum runs over R in
// list order, in FP64.
#include "kernels.hpp"

namespace edus {
namespace {

constexpr int kVgChunk = 32;

__host__ __device__ constexpr int vg_tile(int nt) { return (256 / nt) < 1 ? 1 : ((256 / nt) > 32 ? 32 : 256 / nt); }

template <int N>
__global__ void __launch_bounds__(((vg_tile(N * (N + 1) / 2) * N * (N + 1) / 2 + 31) / 32) * 32)
    k_vg_tables(VgArgs a) {
  constexpr int NT = N * (N + 1) / 2;
  constexpr int KT = vg_tile(NT);
  __shared__ double2 ph[KT][kVgChunk];
  const int tid = threadIdx.x;
  const int kl = tid % KT, e = tid / KT;
  const int k = blockIdx.x * KT + kl;
  const bool valid = e < NT && k < a.nk;
  int i = 0, j = 0;
  if (e < NT) {
    int r = e;
    while (r >= N - i) {
      r -= N - i;
      i++;
    }
    j = i + r;
  }
  double2 h = cz(), d[3] = {cz(), cz(), cz()};
  for (int r0 = 0; r0 < a.nr; r0 += kVgChunk) {
    const int rn = min(kVgChunk, a.nr - r0);
    __syncthreads();
    for (int q = tid; q < KT * kVgChunk; q += blockDim.x) {
      const int qk = q / kVgChunk, qr = q % kVgChunk;
      const int kk = blockIdx.x * KT + qk;
      double2 v = cz();
      if (kk < a.nk && qr < rn) {
        const double* kp = a.kpt + (size_t)kk * 3;
        const double* R = a.Rvec + (size_t)(r0 + qr) * 3;
        const double kR = (kp[0] + a.A[0]) * R[0] + (kp[1] + a.A[1]) * R[1] + (kp[2] + a.A[2]) * R[2];
        double s, c;
        sincospi(2.0 * kR, &s, &c);
        v = make_double2(c, s);
      }
      ph[qk][qr] = v;
    }
    __syncthreads();
    if (valid) {
      const double2* c0 = a.coef + ((size_t)0 * NT + e) * a.nr + r0;
      const double2* c1 = a.coef + ((size_t)1 * NT + e) * a.nr + r0;
      const double2* c2 = a.coef + ((size_t)2 * NT + e) * a.nr + r0;
      const double2* c3 = a.coef + ((size_t)3 * NT + e) * a.nr + r0;
      for (int rr = 0; rr < rn; rr++) {
        const double2 p = ph[kl][rr];
        h = cadd(h, cmul(p, c0[rr]));
        d[0] = cadd(d[0], cmul(p, c1[rr]));
        d[1] = cadd(d[1], cmul(p, c2[rr]));
        d[2] = cadd(d[2], cmul(p, c3[rr]));
      }
    }
  }
  if (!valid) return;
  if (i == j) {
    h.y = 0.;
    for (int x = 0; x < 3; x++) d[x].y = 0.;
  }
  const size_t o = (size_t)e * a.nk + k;
  a.H[o] = h;
  for (int x = 0; x < 3; x++) a.D[(size_t)x * NT * a.nk + o] = d[x];
}

template <int N>
cudaError_t vg_n(const VgArgs& a, cudaStream_t s) {
  constexpr int NT = N * (N + 1) / 2;
  constexpr int KT = vg_tile(NT);
  const int threads = ((KT * NT + 31) / 32) * 32;
  k_vg_tables<N><<<(a.nk + KT - 1) / KT, threads, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_vg_tables(const VgArgs& a, cudaStream_t s) {
  switch (a.n) {
    case 1: return vg_n<1>(a, s);
    case 2: return vg_n<2>(a, s);
    case 3: return vg_n<3>(a, s);
    case 4: return vg_n<4>(a, s);
    case 5: return vg_n<5>(a, s);
    case 8: return vg_n<8>(a, s);
    case 16: return vg_n<16>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace edus
