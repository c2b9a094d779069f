// problem.hpp — host-side description of one solve, built from edus_params.
#pragma once
#include <complex>
#include <string>
#include <vector>

#include "common.hpp"

namespace edus {

using cd = std::complex<double>;

struct Problem {
  edus_params p{};
  int ncv = 0, nch = 0, nv = 0, nc = 0, nbands = 0;  // nbands = Nch + Nv (filled)
  int nk = 0, n1 = 0, n2 = 0;
  double M[3][3]{}, MI[3][3]{}, jac = 0, det_a = 0, dk[3]{};
  std::vector<double> kpt;  // [nk][3] crystal coordinates
  // b-vector stencil (headers/CalculateWeigths.h)
  int nshell = 0, nnb = 0;
  std::vector<int> shell_n;       // vectors per shell
  std::vector<double> shell_w;    // weight per shell
  std::vector<double> bvec;       // [nnb][3] Cartesian
  std::vector<int> bshell;        // shell of each b
  std::vector<int> nbr;           // [nk][nnb] index of k+b
  // model tables in the reference layouts
  std::vector<cd> H, U, D, GE;    // H,U [nk][n][n]; D,GE [nk][n][n][3]
  std::vector<cd> P0;             // initial state [nk][n][n]
  // dissipation (headers/InitParameters.h:203-224)
  double T[EDUS_MAX_BANDS][EDUS_MAX_BANDS]{};
  std::vector<int> diss_i, diss_j;
  // Wannier model
  int nrpts = 0;
  std::vector<double> Rvec;       // [nr][3]
  std::vector<cd> HR;             // [n][n][nr]
  std::vector<cd> rR;             // [3][n][n][nr]
  // Crystal model (headers/Crystal_interface.h): H and the x, y Berry
  // connections sampled on an nkf x nkf crystal grid over [-0.5, 0.5], lower
  // triangle (i >= j) of the first n orbitals, [i*(i+1)/2 + j][k1][k2]
  int cy_nkf = 0;
  std::vector<cd> cyH, cyDx, cyDy;
  // Coulomb coefficients (Source_Main/Fourier_Coulomb.cpp:505-622)
  int ncut = 0;
  std::vector<cd> cA, cB, cC, cD; // [ncut^2][n^2]
  std::vector<cd> screen;         // [n^2]
  std::vector<double> VH;         // [n][n]
  // time grid
  double t_start = 0;
  int itfi = 0;                   // last iteration index (constant dt)
  int nsteps = 0, nprint = 0;
  // Wannier model left untabulated (H, U, D, GE, P0 empty): built on the device
  bool model_deferred = false;
};

int build_problem(const edus_params& p, const char* workdir, Problem& out, bool defer_model = false);
// Remove core bands the run never couples (see problem.cpp); EDUS_EUNSUPPORTED if coupled.
int drop_decoupled_core(Problem& P);
// H, U, D of the problem's model at one crystal k point (save_HUD.cpp conventions).
int model_hud(const Problem& P, const double* kcrys, cd* H, cd* U, cd* D);

// Hermitian eigen-decomposition (cyclic Jacobi), ascending eigenvalues,
// eigenvectors in the columns of Z (row-major n x n).
void eig_herm(int n, cd* A, double* evals, cd* Z);
// Gauss–Jordan inverse with partial pivoting (row-major).
int inv_gj(int n, const double* A, double* Ainv);

// Laser field of the run at time t: EF[0] = sum of pumps, EF[1] = probe / 2
// (Source_Main/RungeKutta.cpp:24-30).
void field_at(const edus_params& p, double t, double EF[2][3]);

}  // namespace edus

// Opaque handle of the C ABI.
struct edus_problem {
  edus::Problem P;
};
