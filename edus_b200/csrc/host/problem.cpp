// problem.cpp — builds the host Problem: k grid, b-vector stencil, model
// tables, dissipation tensor, initial state and Coulomb coefficients.
//
// Reference behaviour followed (anpicon/EDUS):
//   k grid            headers/InitParameters.h:13-40
//   shells & weights  headers/CalculateWeigths.h:1-138 (weights by least squares
//                     in extended precision instead of Armadillo pinv)
//   k+b lookup        headers/CalculateWeigths.h:145-226 (grid arithmetic, then the
//                     reference's tolerance test on the candidate)
//   TB models         headers/TightBinding.h:43-173,271-290,387-440,920-1003,1256-1421
//   Wannier model     headers/Wannier.h:47-148,278-304,336-551
//   tabulation        Source_Main/save_HUD.cpp:19-53,96-137
//   T tensor          headers/InitParameters.h:203-224, main_MPI.cpp:66-77
//   initial state     headers/InitialPopulation.h:2-39
//   Coulomb files     Source_Main/Fourier_Coulomb.cpp:505-622
#include "problem.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <strings.h>

namespace edus {

// ------------------------------------------------------------------ linear algebra

int inv_gj(int n, const double* A, double* Ainv) {
  std::vector<double> a((size_t)n * 2 * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < 2 * n; j++) a[i * 2 * n + j] = (j < n) ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(a[r * 2 * n + c]) > std::fabs(a[piv * 2 * n + c])) piv = r;
    if (a[piv * 2 * n + c] == 0.0) return -1;
    if (piv != c)
      for (int j = 0; j < 2 * n; j++) std::swap(a[c * 2 * n + j], a[piv * 2 * n + j]);
    double d = a[c * 2 * n + c];
    for (int j = 0; j < 2 * n; j++) a[c * 2 * n + j] /= d;
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      double f = a[r * 2 * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; j++) a[r * 2 * n + j] -= f * a[c * 2 * n + j];
    }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) Ainv[i * n + j] = a[i * 2 * n + n + j];
  return 0;
}

void eig_herm(int n, cd* A, double* evals, cd* Z) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) Z[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, diag = 0;
    for (int i = 0; i < n; i++) {
      diag += std::norm(A[i * n + i]);
      for (int j = i + 1; j < n; j++) off += std::norm(A[i * n + j]);
    }
    if (off <= 1e-34 * (diag + 1e-300)) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        cd apq = A[p * n + q];
        double mag = std::abs(apq);
        if (mag < 1e-300) continue;
        double app = A[p * n + p].real(), aqq = A[q * n + q].real();
        cd ph = apq / mag;
        double theta = 0.5 * std::atan2(2.0 * mag, aqq - app);
        double c = std::cos(theta), s = std::sin(theta);
        cd sp = s * ph, sc = s * std::conj(ph);
        for (int k = 0; k < n; k++) {
          cd akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - sc * akq;
          A[k * n + q] = sp * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          cd apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - sp * aqk;
          A[q * n + k] = sc * apk + c * aqk;
        }
        A[p * n + q] = 0;
        A[q * n + p] = 0;
        A[p * n + p] = A[p * n + p].real();
        A[q * n + q] = A[q * n + q].real();
        for (int k = 0; k < n; k++) {
          cd zkp = Z[k * n + p], zkq = Z[k * n + q];
          Z[k * n + p] = c * zkp - sc * zkq;
          Z[k * n + q] = sp * zkp + c * zkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; i++) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return A[a * n + a].real() < A[b * n + b].real(); });
  std::vector<cd> Zs((size_t)n * n);
  for (int j = 0; j < n; j++) {
    evals[j] = A[ord[j] * n + ord[j]].real();
    for (int i = 0; i < n; i++) Zs[i * n + j] = Z[i * n + ord[j]];
  }
  std::copy(Zs.begin(), Zs.end(), Z);
}

// Minimum-norm least squares w = A^+ q (A: rows x cols, row-major), the
// pseudo-inverse with singular values at or below 1e-16 dropped, as the
// reference solves for the b-shell weights (pinv(A, 1.e-16) * q,
// headers/CalculateWeigths.h:100). The singular value decomposition is a
// one-sided Jacobi one in long double: column rotations of A (accumulated in
// V) until the columns are orthogonal, whose norms are then the singular
// values. On a lattice whose shell equations are rank deficient (orthorhombic
// cells) the minimum-norm choice is what fixes the weights.
static void lstsq(int rows, int cols, const double* A, const double* q, double* w) {
  std::vector<long double> U((size_t)rows * cols), V((size_t)cols * cols, 0.0L);
  for (int i = 0; i < rows * cols; i++) U[i] = A[i];
  for (int i = 0; i < cols; i++) V[(size_t)i * cols + i] = 1.0L;
  for (int sweep = 0; sweep < 80; sweep++) {
    long double worst = 0;
    for (int p = 0; p < cols; p++)
      for (int r = p + 1; r < cols; r++) {
        long double app = 0, arr = 0, apr = 0;
        for (int i = 0; i < rows; i++) {
          const long double x = U[(size_t)i * cols + p], y = U[(size_t)i * cols + r];
          app += x * x;
          arr += y * y;
          apr += x * y;
        }
        if (apr == 0 || app == 0 || arr == 0) continue;
        const long double rel = std::fabs(apr) / std::sqrt(app * arr);
        worst = std::max(worst, rel);
        if (rel < 1e-19L) continue;
        const long double zeta = (arr - app) / (2 * apr);
        const long double t = (zeta >= 0 ? 1.0L : -1.0L) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
        const long double c = 1 / std::sqrt(1 + t * t), sn = c * t;
        for (int i = 0; i < rows; i++) {
          long double& x = U[(size_t)i * cols + p];
          long double& y = U[(size_t)i * cols + r];
          const long double x0 = x;
          x = c * x0 - sn * y;
          y = sn * x0 + c * y;
        }
        for (int i = 0; i < cols; i++) {
          long double& x = V[(size_t)i * cols + p];
          long double& y = V[(size_t)i * cols + r];
          const long double x0 = x;
          x = c * x0 - sn * y;
          y = sn * x0 + c * y;
        }
      }
    if (worst < 1e-19L) break;
  }
  std::vector<long double> coef(cols, 0.0L);
  for (int j = 0; j < cols; j++) {
    long double s2 = 0, uq = 0;
    for (int i = 0; i < rows; i++) {
      s2 += U[(size_t)i * cols + j] * U[(size_t)i * cols + j];
      uq += U[(size_t)i * cols + j] * q[i];
    }
    // column j of the rotated A is sigma_j u_j: (u_j . q) / sigma_j = (col . q) / sigma_j^2
    if (std::sqrt(s2) > 1e-16L) coef[j] = uq / s2;
  }
  for (int i = 0; i < cols; i++) {
    long double acc = 0;
    for (int j = 0; j < cols; j++) acc += V[(size_t)i * cols + j] * coef[j];
    w[i] = (double)acc;
  }
}

// ------------------------------------------------------------------ geometry

static void crys_to_cart(const Problem& P, const double* c, double* x) {
  for (int i = 0; i < 3; i++) x[i] = P.M[i][0] * c[0] + P.M[i][1] * c[1] + P.M[i][2] * c[2];
}
static void cart_to_crys(const Problem& P, const double* x, double* c) {
  for (int i = 0; i < 3; i++) c[i] = P.MI[i][0] * x[0] + P.MI[i][1] * x[1] + P.MI[i][2] * x[2];
}

static int setup_geometry(Problem& P) {
  double Mf[9], MIf[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      P.M[i][j] = P.p.b[j][i];
      Mf[i * 3 + j] = P.M[i][j];
    }
  if (inv_gj(3, Mf, MIf)) return fail(EDUS_EINVAL, "reciprocal lattice is singular");
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) P.MI[i][j] = MIf[i * 3 + j];
  const double(*m)[3] = P.M;
  P.jac = std::fabs(m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                    m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]));
  const double(*a)[3] = P.p.a;
  P.det_a = P.p.sample_110 ? std::fabs(a[0][0] * a[1][1] - a[0][1] * a[1][0]) : std::fabs(a[1][1] * a[2][2] - a[1][2] * a[2][1]);
  const int* Nk = P.p.nk;
  P.nk = Nk[0] * Nk[1] * Nk[2];
  P.n1 = Nk[1];
  P.n2 = Nk[2];
  for (int c = 0; c < 3; c++) P.dk[c] = 1.0 / Nk[c];
  P.kpt.assign((size_t)P.nk * 3, 0.0);
  if (P.p.kpt_read) {
    // nkpt read: the listed crystal coordinates (headers/ReadInput.h:429-437)
    std::ifstream f(P.p.input_path);
    if (!f) return fail(EDUS_EIO, "nkpt read: cannot reopen %s", P.p.input_path);
    f.seekg((std::streamoff)P.p.kpt_offset);
    for (int ik = 0; ik < P.nk; ik++)
      if (!(f >> P.kpt[ik * 3] >> P.kpt[ik * 3 + 1] >> P.kpt[ik * 3 + 2]))
        return fail(EDUS_EPARSE, "nkpt read: %d k points expected in %s", P.nk, P.p.input_path);
  } else {
    for (int ik = 0; ik < P.nk; ik++) {
      int iik[3] = {(ik / (Nk[2] * Nk[1])) % Nk[0], (ik / Nk[2]) % Nk[1], ik % Nk[2]};
      for (int c = 0; c < 3; c++) P.kpt[ik * 3 + c] = (P.dk[c] != 1.0) ? -0.5 + P.dk[c] * iik[c] : 0.0;
    }
  }
  // shells: each new shell is the next larger |k| over the grid points
  int plane = -1;
  for (int i = 0; i < 3; i++)
    if (Nk[i] == 1) plane = i;
  std::vector<double> nrm(P.nk);
  for (int ik = 0; ik < P.nk; ik++) {
    double x[3];
    crys_to_cart(P, &P.kpt[ik * 3], x);
    nrm[ik] = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  }
  std::vector<double> radii{1.e-08};
  bool enough = false;
  P.nshell = 0;
  P.shell_n.clear();
  P.bvec.clear();
  P.bshell.clear();
  while (!enough) {
    double rad = 1000.;
    for (int ik = 0; ik < P.nk; ik++) {
      bool in = false;
      for (double r : radii) in = in || (nrm[ik] <= r + 1.e-11);
      if (!in && nrm[ik] < rad) rad = nrm[ik];
    }
    radii.push_back(rad);
    int cnt = 0;
    for (int ik = 0; ik < P.nk; ik++)
      if (std::fabs(nrm[ik] - rad) < 1.e-11) {
        double x[3];
        crys_to_cart(P, &P.kpt[ik * 3], x);
        P.bvec.insert(P.bvec.end(), x, x + 3);
        P.bshell.push_back(P.nshell);
        cnt++;
      }
    P.shell_n.push_back(cnt);
    P.nshell++;
    int ns = P.nshell;
    std::vector<double> A(21 * ns, 0.0);
    int base = 0;
    for (int sh = 0; sh < ns; sh++) {
      const double* bv = &P.bvec[base * 3];
      int nb = P.shell_n[sh];
      int row = 0;
      for (int id = 0; id < 3; id++)
        if (id != plane) {
          for (int b = 0; b < nb; b++) A[row * ns + sh] += bv[b * 3 + id] * bv[b * 3 + id];
          row++;
        }
      for (int id = 0; id < 3; id++)
        for (int jd = id + 1; jd < 3; jd++)
          if (id != plane && jd != plane) {
            for (int b = 0; b < nb; b++) A[row * ns + sh] += bv[b * 3 + id] * bv[b * 3 + jd];
            row++;
          }
      row = 5;
      for (int id = 0; id < 3; id++)
        for (int jd = id; jd < 3; jd++)
          for (int ld = jd; ld < 3; ld++)
            for (int md = ld; md < 3; md++) {
              for (int b = 0; b < nb; b++) A[row * ns + sh] += bv[b * 3 + id] * bv[b * 3 + jd] * bv[b * 3 + ld] * bv[b * 3 + md];
              row++;
            }
      base += nb;
    }
    double q[21] = {0};
    q[0] = 1;
    q[1] = 1;
    q[2] = !(plane + 1);
    std::vector<double> w(ns, 0.0);
    lstsq(21, ns, A.data(), q, w.data());
    double r2 = 0;
    for (int r = 0; r < 21; r++) {
      double acc = 0;
      for (int sh = 0; sh < ns; sh++) acc += A[r * ns + sh] * w[sh];
      r2 += (acc - q[r]) * (acc - q[r]);
    }
    P.shell_w = w;
    enough = std::sqrt(r2) < 1.e-07;
    if (P.nshell >= 32 && !enough) return fail(EDUS_EINVAL, "More than 32 shells needed.");
  }
  P.nnb = (int)P.bshell.size();
  // k+b table: index arithmetic on the grid, checked with the reference's test
  P.nbr.assign((size_t)P.nk * P.nnb, -1);
  std::vector<int> off((size_t)P.nnb * 3);
  for (int b = 0; b < P.nnb; b++) {
    double c[3];
    cart_to_crys(P, &P.bvec[b * 3], c);
    for (int i = 0; i < 3; i++) off[b * 3 + i] = (int)std::lround(c[i] * Nk[i]);
  }
  int bad = 0;
  for (int ik = 0; ik < P.nk; ik++) {
    int iik[3] = {(ik / (Nk[2] * Nk[1])) % Nk[0], (ik / Nk[2]) % Nk[1], ik % Nk[2]};
    double kk[3];
    crys_to_cart(P, &P.kpt[ik * 3], kk);
    for (int b = 0; b < P.nnb; b++) {
      int j[3];
      for (int i = 0; i < 3; i++) j[i] = (((iik[i] + off[b * 3 + i]) % Nk[i]) + Nk[i]) % Nk[i];
      int cand = (j[0] * Nk[1] + j[1]) * Nk[2] + j[2];
      double x[3] = {kk[0] + P.bvec[b * 3], kk[1] + P.bvec[b * 3 + 1], kk[2] + P.bvec[b * 3 + 2]};
      double c[3];
      cart_to_crys(P, x, c);
      for (int i = 0; i < 3; i++) c[i] = std::fmod(c[i] + 0.5, 1.) - 0.5;
      auto match = [&](int k1) {
        for (int i = 0; i < 3; i++) {
          const double d = c[i] - P.kpt[(size_t)k1 * 3 + i];
          if (!(std::fabs(d) < 1.e-08 || std::fabs(d - 1.) < 1.e-08 || std::fabs(d + 1.) < 1.e-08)) return false;
        }
        return true;
      };
      // a listed grid: the first match in list order, as the reference searches
      // (headers/CalculateWeigths.h:170-200); the grid: its index, checked
      bool ok = false;
      if (P.p.kpt_read) {
        for (int k1 = 0; k1 < P.nk && !ok; k1++)
          if (match(k1)) {
            cand = k1;
            ok = true;
          }
      } else {
        ok = match(cand);
      }
      if (!ok) {
        bad++;
        cand = ik;
      }
      P.nbr[(size_t)ik * P.nnb + b] = cand;
    }
  }
  if (bad) return fail(EDUS_EINVAL, "k+b not found on the grid for %d stencil entries", bad);
  return 0;
}

// ------------------------------------------------------------------ models

namespace {

enum TbKind {
  kHaldaneN = 1,
  kHaldaneB,
  kGen2d,
  kBN,
  kCoreBNN,
  kCoreBNB,
  kGraphene,
  kCoreGraphene,
  kGrapheneCostD,
  kGrapheneSymD,
  kGrapheneZurron,
  kBN1b,
  kVampa,
  kGeS,
  kDLGraphene
};

// Vampa2015 model: cosine series of the two bands along each crystal axis,
// E_c(k) = sum_x sum_j v[c][x][j] cos(j k_x) (+ the gap for the conduction
// band); parameters as headers/TightBinding.h:98-122 tabulates them
constexpr double kVampaCoeff[2][3][6] = {
    {{-0.0928, 0.0705, 0.0200, -0.0012, 0.0029, 0.0006}, {-0.0307, 0.0307, 0, 0, 0, 0}, {-0.0059, 0.0059, 0, 0, 0, 0}},
    {{0.0898, -0.0814, -0.0024, -0.0048, -0.0003, -0.0009}, {0.1147, -0.1147, 0, 0, 0, 0}, {0.0435, -0.0435, 0, 0, 0, 0}}};

struct Tb {
  int kind = 0;
  double a = 2.5 * kSpaceAAu, b = 3.16 * kEnergyEvAu, g = 6.2 * kEnergyEvAu, t2 = 0, phi0 = 0, core = 0, rchv = 0, rchc = 0;
  double c = 0, d = 0, f = 0;  // GeS second-neighbour hoppings and first-neighbour hopping
};

int tb_setup(const edus_params& p, Tb& t) {
  std::string nm = p.tb_type;
  if (nm == "Haldane_CoreBN_Nedge" || nm == "Haldane_CoreBN_Bedge") {
    t.kind = nm == "Haldane_CoreBN_Nedge" ? kHaldaneN : kHaldaneB;
    t.g = p.hopping[0];
    t.b = p.hopping[1];
    t.t2 = p.hopping[2];
    t.phi0 = p.hopping[3];
  } else if (nm == "gen2d_hexagonal") {
    t.kind = kGen2d;
    t.a = p.hopping[0];
    t.g = p.hopping[1];
    t.b = p.hopping[2];
    t.t2 = p.hopping[3];
    t.phi0 = p.hopping[4];
    t.core = p.hopping[5];
    t.rchv = p.hopping[6];
    t.rchc = p.hopping[7];
  } else if (nm == "BoronNitride") {
    t.kind = kBN;
  } else if (nm == "BN1b") {
    t.kind = kBN1b;
  } else if (nm == "Vampa2015") {
    t.kind = kVampa;
    t.g = 0.1213;
  } else if (nm == "GeS" || nm == "GeS_HSE06") {
    // headers/TightBinding.h:135-154
    const double eV = kEnergyEvAu;
    t.kind = kGeS;
    const bool hse = nm == "GeS_HSE06";
    t.g = (hse ? 0.62 : 0.41) * eV;
    t.f = (hse ? 2.91 : -2.33) * eV;
    t.t2 = (hse ? -0.797 : 0.61) * eV;
    t.b = (hse ? -0.05 : 0.13) * eV;
    t.c = (hse ? -0.14 : 0.07) * eV;
    t.d = (hse ? 0.106 : -0.09) * eV;
  } else if (nm == "DLGraphene") {
    // headers/TightBinding.h:90-97: bilayer, interlayer distance c and hopping d
    t.kind = kDLGraphene;
    t.a = 2.46 * kSpaceAAu;
    t.b = 2.97 * kEnergyEvAu;
    t.c = 3.35 * kSpaceAAu;
    t.d = 0.39 * kEnergyEvAu;
    t.g = 0;
  } else if (nm == "CoreBN_Nedge" || nm == "CoreBN_Bedge") {
    t.kind = nm == "CoreBN_Nedge" ? kCoreBNN : kCoreBNB;
  } else if (nm == "Graphene" || nm == "CoreGraphene" || nm == "Graphene_costD" || nm == "Graphene_symmetricD" ||
             nm == "GrapheneZurron") {
    // headers/TightBinding.h:48-80: a = 2.46 A, b = 2.97 eV, no gap
    t.kind = nm == "Graphene"         ? kGraphene
             : nm == "CoreGraphene"   ? kCoreGraphene
             : nm == "Graphene_costD" ? kGrapheneCostD
             : nm == "GrapheneZurron" ? kGrapheneZurron
                                      : kGrapheneSymD;
    t.a = 2.46 * kSpaceAAu;
    t.b = 2.97 * kEnergyEvAu;
    t.g = 0;
  } else {
    return fail(EDUS_EUNSUPPORTED,
                "tight-binding model %s is not built (Haldane_CoreBN_Nedge/Bedge, CoreBN_Nedge/Bedge, gen2d_hexagonal, "
                "BoronNitride, BN1b, Graphene, CoreGraphene, Graphene_costD, Graphene_symmetricD, GrapheneZurron, "
                "DLGraphene, Vampa2015, GeS, GeS_HSE06 are)",
                nm.c_str());
  }
  return 0;
}

inline cd eiphi(double x) { return cd(std::cos(x), std::sin(x)); }

// H, U and D of one k (crystal k, Cartesian kc) for the tight-binding models.
void tb_eval(const Tb& t, int n, const double* k, const double* kc, cd* H, cd* U, cd* D) {
  const double k1 = k[1], k2 = k[2];
  for (int e = 0; e < n * n; e++) {
    H[e] = 0;
    U[e] = 0;
  }
  for (int e = 0; e < n * n * 3; e++) D[e] = 0;
  const double tp1 = 2. * kPi * k1, tp2 = 2. * kPi * k2;
  auto d = [&](int i, int j, int x) -> cd& { return D[(i * n + j) * 3 + x]; };
  if (t.kind == kCoreBNN || t.kind == kCoreBNB) {
    // headers/TightBinding.h:177-207 (energy), :894-921 (unitary), dipoles as the Haldane edges
    const cd f = (1. + eiphi(tp1)) + eiphi(tp2);
    H[0] = t.kind == kCoreBNN ? -15.06 : -6.91;
    H[1 * n + 1] = -t.g / 2.;
    H[1 * n + 2] = t.b * std::conj(f);
    H[2 * n + 1] = t.b * f;
    H[2 * n + 2] = t.g / 2.;
    const double E = std::sqrt(t.g * t.g + 4. * t.b * t.b * f * std::conj(f)).real() / 2.;
    const double a = std::sqrt((t.g + 2. * E) / (4. * E)), h = std::sqrt((2. * E - t.g) / (4. * E));
    U[0] = 1.;
    U[1 * n + 1] = a;
    U[1 * n + 2] = -h * std::conj(f) / std::abs(f);
    U[2 * n + 1] = h;
    U[2 * n + 2] = a * std::conj(f) / std::abs(f);
    const double ay = t.a / std::sqrt(3.);
    if (t.kind == kCoreBNN) {
      d(0, 1, 0) = d(1, 0, 0) = 0.0697595094;
      d(2, 2, 1) = ay;
    } else {
      d(0, 2, 0) = d(2, 0, 0) = 0.0869151662;
      d(2, 2, 1) = ay;
      d(0, 0, 1) = ay;
    }
    return;
  }
  if (t.kind == kBN1b) {
    // headers/TightBinding.h:307-311 (one band), :1147-1150 (U = 1), no dipoles
    const cd f = (eiphi(tp1) + 1.) + eiphi(tp2);
    H[0] = 0.5 * std::sqrt(t.g * t.g + 4. * t.b * t.b * f * std::conj(f)).real();
    U[0] = 1.;
    return;
  }
  if (t.kind == kVampa) {
    // headers/TightBinding.h:312-326 (energy), :1151-1155 (U = 1), dipoles 3.46 in x, y and 3.94 in z off the diagonal
    for (int c = 0; c < 2; c++) {
      cd e = 0.;
      for (int x = 0; x < 3; x++)
        for (int j = 0; j < 6; j++) e += kVampaCoeff[c][x][j] * std::cos(j * k[x]);
      if (c == 1) e += t.g;
      H[c * n + c] = e;
      U[c * n + c] = 1.;
    }
    d(0, 1, 0) = d(1, 0, 0) = d(0, 1, 1) = d(1, 0, 1) = 3.46;
    d(0, 1, 2) = d(1, 0, 2) = 3.94;
    return;
  }
  if (t.kind == kGeS) {
    // headers/TightBinding.h:441-462 (energy), :1005-1030 (unitary), :1339-1343 (dipole)
    const double tor = -2. * t.c * (std::cos(tp1) + std::cos(tp2)) - 2. * t.d * (std::cos(2. * kPi * (k1 - k2)));
    H[0] = t.g + tor;
    H[3] = -t.g + tor;
    const cd phix = eiphi(tp1) + eiphi(tp2);
    const cd tc = -t.f - t.t2 * phix - t.b * std::conj(phix);
    H[1] = std::conj(tc);
    H[2] = tc;
    const double Bx = tc.real(), By = tc.imag(), Bz = t.g;
    const double B = std::sqrt(Bx * Bx + By * By + Bz * Bz);
    const double phi = std::atan2(By, Bx) / 2.;
    const double c2 = std::sqrt((B + Bz) / 2. / B), s2 = std::sqrt((B - Bz) / 2. / B);
    U[0] = eiphi(phi) * s2;
    U[1] = -eiphi(-phi) * c2;
    U[2] = eiphi(phi) * c2;
    U[3] = eiphi(-phi) * s2;
    d(1, 1, 1) = 0.52 * kSpaceAAu;
    return;
  }
  if (t.kind == kDLGraphene) {
    // headers/TightBinding.h:291-312 (energy), :1083-1145 (unitary: the closed-form
    // eigenvectors, singular where f = 0), :1300-1308, 1376-1385, 1404-1413 (dipoles)
    const double b = t.b, dd = t.d;
    const cd f = (eiphi(tp1) + 1.) + eiphi(tp2);
    H[1] = H[2 * n + 3] = std::conj(f) * b;
    H[n] = H[3 * n + 2] = f * b;
    H[3] = H[3 * n] = dd;
    const cd s = std::sqrt(dd * dd + 4. * (b * b) * f * std::conj(f)), cs = std::conj(s);
    const cd bf = b * f, bfc = b * std::conj(f);
    auto sq = [](double x) { return x * x; };
    const double n1 = std::sqrt(8. + sq(std::abs((dd - s) / bfc)) + 16. * sq(std::abs(bf / (dd + s))));
    const double n2 = std::sqrt(8. + 16. * sq(std::abs(bf / (dd - s))) + sq(std::abs((dd + s) / bfc)));
    U[0] = -2. / n1;
    U[1] = (-dd + cs) / (bf * n1);
    U[2] = (-4. * b * f) / (n1 * (dd + cs));
    U[3] = 2. / n1;
    U[n] = 2. / n2;
    U[n + 1] = -((dd + cs) / (bf * n2));
    U[n + 2] = (4. * b * f) / (n2 * (dd - cs));
    U[n + 3] = 2. / n2;
    U[2 * n] = -2. / n2;
    U[2 * n + 1] = -((dd + cs) / (bf * n2));
    U[2 * n + 2] = (-4. * b * f) / (n2 * (dd - cs));
    U[2 * n + 3] = 2. / n2;
    U[3 * n] = 2. / n1;
    U[3 * n + 1] = (-dd + cs) / (bf * n1);
    U[3 * n + 2] = (4. * b * f) / (n1 * (dd + cs));
    U[3 * n + 3] = 2. / n1;
    d(2, 2, 0) = d(3, 3, 0) = t.c;
    d(1, 1, 1) = -t.a / std::sqrt(3.);
    d(2, 2, 1) = d(3, 3, 1) = t.a / (2. * std::sqrt(3.));
    d(2, 2, 2) = t.a / 2.;
    d(3, 3, 2) = -t.a / 2.;
    return;
  }
  if (t.kind == kGrapheneCostD || t.kind == kGrapheneSymD) {
    // headers/TightBinding.h:225-239 (energy), :1064-1070 (unitary: 1),
    // :1272-1283, 1349-1357, 1401-1405 (dipoles)
    const double modf = std::abs((eiphi(tp1) + 1.) + eiphi(tp2));
    H[0] = H[1 * n + 1] = -10.892178;
    H[2 * n + 2] = -t.b * modf;
    H[3 * n + 3] = t.b * modf;
    for (int i = 0; i < n; i++) U[i * n + i] = 1.;
    const double dx = 0.0780088 / std::sqrt(2.);
    d(0, 2, 0) = d(0, 3, 0) = d(1, 2, 0) = dx;
    d(1, 3, 0) = -dx;
    d(2, 0, 0) = d(3, 0, 0) = d(2, 1, 0) = dx;
    d(3, 1, 0) = -dx;
    const int ny = t.kind == kGrapheneSymD ? 2 : 1;  // the symmetric variant repeats y in z
    for (int x = 1; x <= ny; x++) {
      d(1, 1, x) = -2.68341111;
      d(2, 2, x) = d(3, 3, x) = -2.68341111 / 2;
      d(2, 3, x) = d(3, 2, x) = 2.68341111 / 2;
    }
    return;
  }
  if (t.kind == kGrapheneZurron) {
    // headers/TightBinding.h:257-269 (energy), :1072-1081 (unitary); no dipoles
    const double a = t.a;
    const cd f = eiphi(-a * kc[1] / std::sqrt(3.)) * (1. + 2. * eiphi(std::sqrt(3.) * a * kc[1] / 2.) * std::cos(a * kc[2] / 2.));
    H[1] = f * t.b;
    H[n] = std::conj(f) * t.b;
    U[0] = U[n] = 1. / std::sqrt(2.);
    U[1] = -f / (std::sqrt(2.) * std::abs(f));
    U[n + 1] = f / (std::sqrt(2.) * std::abs(f));
    return;
  }
  if (t.kind == kGraphene || t.kind == kCoreGraphene) {
    // headers/TightBinding.h:209-255 (energy), :1032-1059 (unitary), :1280-1285, 1345-1360 (dipoles)
    const int o2 = t.kind == kCoreGraphene ? 2 : 0;
    if (o2) {
      H[0] = H[1 * n + 1] = -10.892178;
      U[0] = U[1 * n + 1] = 1.;
      d(0, 2, 0) = d(1, 3, 0) = d(2, 0, 0) = d(3, 1, 0) = 0.0780088;
      d(1, 1, 1) = d(3, 3, 1) = -2.68341111;
    } else {
      d(1, 1, 1) = -2.68341111;
    }
    const cd f = (eiphi(tp1) + 1.) + eiphi(tp2);
    H[o2 * n + o2 + 1] = std::conj(f) * t.b;
    H[(o2 + 1) * n + o2] = f * t.b;
    const cd fm = (eiphi(-tp1) + 1.) + eiphi(-tp2);
    U[o2 * n + o2] = U[(o2 + 1) * n + o2] = 1. / std::sqrt(2.);
    U[o2 * n + o2 + 1] = -fm / (std::sqrt(2.) * std::abs(fm));
    U[(o2 + 1) * n + o2 + 1] = fm / (std::sqrt(2.) * std::abs(fm));
    return;
  }
  double Bx = t.b * (1. + std::cos(tp1) + std::cos(tp2));
  double By = t.b * (std::sin(tp1) + std::sin(tp2));
  double Bz = -t.g / 2.;
  int o = 1;
  if (t.kind == kBN) {
    o = 0;
    cd f = (eiphi(tp1) + 1.) + eiphi(tp2);
    H[0] = -t.g / 2;
    H[3] = t.g / 2;
    H[1] = std::conj(f) * t.b;
    H[2] = f * t.b;
    D[(1 * n + 1) * 3 + 1] = t.a / std::sqrt(3);
  } else {
    H[0] = t.kind == kHaldaneN ? -15.06 : (t.kind == kHaldaneB ? -6.91 : t.core);
    cd f2 = eiphi(tp1 - tp2) + eiphi(tp2) + eiphi(-tp1);
    cd f = 1. + eiphi(-tp1) + eiphi(-tp2);
    H[1 * n + 1] = -t.g / 2. + 2. * (t.t2 * eiphi(t.phi0) * f2).real();
    H[1 * n + 2] = t.b * f;
    H[2 * n + 1] = t.b * std::conj(f);
    H[2 * n + 2] = t.g / 2. + 2. * (t.t2 * eiphi(-t.phi0) * f2).real();
    Bz = -t.g / 2. - 2. * t.t2 * std::sin(t.phi0) * (std::sin(-tp2 + tp1) + std::sin(tp2) + std::sin(-tp1));
    U[0] = 1.;
    double ay = t.a / std::sqrt(3.);
    if (t.kind == kHaldaneN) {
      d(0, 1, 0) = d(1, 0, 0) = 0.0697595094;
      d(2, 2, 1) = ay;
    } else if (t.kind == kHaldaneB) {
      d(0, 2, 0) = d(2, 0, 0) = 0.0869151662;
      d(2, 2, 1) = ay;
      d(0, 0, 1) = ay;
    } else {
      d(0, 1, 0) = d(1, 0, 0) = t.rchv;
      d(0, 2, 0) = d(2, 0, 0) = t.rchc;
      d(2, 2, 1) = -ay;
      if (std::fabs(t.rchc) > 1.e-6) d(0, 0, 1) = -ay;
    }
  }
  double B = std::sqrt(Bx * Bx + By * By + Bz * Bz);
  double phi = std::atan2(By, Bx) / 2.;
  double c2 = std::sqrt((B + Bz) / 2. / B), s2 = std::sqrt((B - Bz) / 2. / B);
  U[o * n + o] = eiphi(phi) * s2;
  U[o * n + o + 1] = -eiphi(-phi) * c2;
  U[(o + 1) * n + o] = eiphi(phi) * c2;
  U[(o + 1) * n + o + 1] = eiphi(-phi) * s2;
}

int read_wannier(Problem& P, const char* workdir) {
  std::string path = std::string(workdir ? workdir : ".") + "/" + P.p.ref_coord + "_tb.dat";
  std::ifstream f(path);
  if (!f) return fail(EDUS_EIO, "No path %s file found.", path.c_str());
  std::string line;
  for (int i = 0; i < 4; i++) std::getline(f, line);
  int nw = 0, nr = 0;
  f >> nw >> nr;
  if (!f || nw != P.ncv) return fail(EDUS_EIO, "%s: num_wann %d does not match %d bands", path.c_str(), nw, P.ncv);
  int n = nw;
  P.nrpts = nr;
  std::vector<double> ndeg(nr);
  for (int i = 0; i < nr; i++) f >> ndeg[i];
  P.Rvec.assign((size_t)nr * 3, 0);
  P.HR.assign((size_t)n * n * nr, 0);
  P.rR.assign((size_t)3 * n * n * nr, 0);
  for (int iR = 0; iR < nr; iR++) {
    f >> P.Rvec[iR * 3] >> P.Rvec[iR * 3 + 1] >> P.Rvec[iR * 3 + 2];
    for (int in = 0; in < n; in++)
      for (int im = 0; im < n; im++) {
        int t1, t2;
        double hr, hi;
        f >> t1 >> t2 >> hr >> hi;
        P.HR[((size_t)im * n + in) * nr + iR] = cd(hr / ndeg[iR] * kEnergyEvAu, hi / ndeg[iR] * kEnergyEvAu);
      }
  }
  for (int iR = 0; iR < nr; iR++) {
    double R[3];
    f >> R[0] >> R[1] >> R[2];
    for (int in = 0; in < n; in++)
      for (int im = 0; im < n; im++) {
        int t1, t2;
        double v[6];
        f >> t1 >> t2 >> v[0] >> v[1] >> v[2] >> v[3] >> v[4] >> v[5];
        for (int x = 0; x < 3; x++)
          P.rR[(((size_t)x * n + im) * n + in) * nr + iR] = cd(v[2 * x] / ndeg[iR] * kSpaceAAu, v[2 * x + 1] / ndeg[iR] * kSpaceAAu);
      }
  }
  if (!f) return fail(EDUS_EIO, "%s: truncated _tb.dat", path.c_str());
  return 0;
}

// Whitespace-separated tokens of one line (headers/ReadInput.h:1-30 splits on blanks).
std::vector<std::string> tokens(const std::string& line) {
  std::vector<std::string> t;
  std::string cur;
  for (char c : line) {
    if (c == ' ' || c == '\t' || c == '\r' || c == '\n') {
      if (!cur.empty()) t.push_back(cur);
      cur.clear();
    } else {
      cur += c;
    }
  }
  if (!cur.empty()) t.push_back(cur);
  return t;
}

bool last_is(const std::vector<std::string>& t, const char* w) { return !t.empty() && strcasecmp(t.back().c_str(), w) == 0; }

// Crystal model files in the working directory (headers/Crystal_interface.h:19-208):
// kmesh_data.dat gives the in-plane lattice (a[0] = 15 x, b[0] = x / 15), the
// orbital count after the line ending in "basis" and the grid size nkf after the
// line ending in "direction"; hk_orthonormal.dat holds per grid point (k1 major)
// the lower triangle of Re H, a separator, Im H, two separators;
// bc_betabetap_{real,imag}.dat hold the x and y Berry connections the same way.
int read_crystal(Problem& P, const char* workdir) {
  const std::string wd = workdir ? workdir : ".";
  const int n = P.ncv;
  int norb = 0, nkf = 0;
  {
    std::string path = wd + "/kmesh_data.dat";
    std::ifstream f(path);
    if (!f) return fail(EDUS_EIO, "cannot read %s", path.c_str());
    std::string line;
    double v[4][2];
    for (int r = 0; r < 4; r++) {
      std::getline(f, line);
      if (!std::getline(f, line)) return fail(EDUS_EIO, "%s: truncated lattice block", path.c_str());
      auto t = tokens(line);
      if (t.size() < 2) return fail(EDUS_EIO, "%s: lattice row %d needs two numbers", path.c_str(), r);
      v[r][0] = std::atof(t[0].c_str());
      v[r][1] = std::atof(t[1].c_str());
    }
    double(*a)[3] = P.p.a;
    double(*b)[3] = P.p.b;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) a[i][j] = b[i][j] = 0;
    a[0][0] = 15.;
    a[1][1] = v[0][0];
    a[1][2] = v[0][1];
    a[2][1] = v[1][0];
    a[2][2] = v[1][1];
    b[0][0] = 1. / 15.;
    b[1][1] = v[2][0];
    b[1][2] = v[2][1];
    b[2][1] = v[3][0];
    b[2][2] = v[3][1];
    bool found = false;
    while (std::getline(f, line))
      if (last_is(tokens(line), "basis")) {
        found = true;
        break;
      }
    if (!found || !std::getline(f, line) || tokens(line).empty())
      return fail(EDUS_EIO, "%s: no orbital count after the basis block", path.c_str());
    norb = std::atoi(tokens(line)[0].c_str());
    found = false;
    while (std::getline(f, line))
      if (last_is(tokens(line), "direction")) {
        found = true;
        break;
      }
    if (!found || !std::getline(f, line) || tokens(line).empty())
      return fail(EDUS_EIO, "%s: no k-point count after the direction line", path.c_str());
    nkf = std::atoi(tokens(line)[0].c_str());
  }
  if (norb < n) return fail(EDUS_EINVAL, "kmesh_data.dat has %d orbitals, the input %d bands", norb, n);
  if (nkf < 2) return fail(EDUS_EINVAL, "kmesh_data.dat grid of %d points per direction (2 or more)", nkf);
  const size_t g2 = (size_t)nkf * nkf, ne = (size_t)n * (n + 1) / 2;
  P.cy_nkf = nkf;
  P.cyH.assign(ne * g2, 0);
  P.cyDx.assign(ne * g2, 0);
  P.cyDy.assign(ne * g2, 0);
  // one block of norb lower-triangle rows; row i keeps its first min(i, n-1)+1 numbers
  auto block = [&](std::istream& f, const std::string& path, size_t g, std::vector<cd>& dst, bool imag) -> int {
    std::string line;
    for (int i = 0; i < norb; i++) {
      if (!std::getline(f, line)) return fail(EDUS_EIO, "%s: truncated", path.c_str());
      if (i >= n) continue;
      auto t = tokens(line);
      if ((int)t.size() < i + 1) return fail(EDUS_EIO, "%s: row %d needs %d numbers", path.c_str(), i, i + 1);
      for (int j = 0; j <= i; j++) {
        const double x = std::atof(t[j].c_str());
        cd& d = dst[((size_t)i * (i + 1) / 2 + j) * g2 + g];
        d = imag ? cd(d.real(), d.imag() + x) : cd(d.real() + x, d.imag());
      }
    }
    return 0;
  };
  {
    std::string path = wd + "/hk_orthonormal.dat";
    std::ifstream f(path);
    if (!f) return fail(EDUS_EIO, "cannot read %s", path.c_str());
    std::string line;
    for (size_t g = 0; g < g2; g++) {
      int rc = block(f, path, g, P.cyH, false);
      if (rc) return rc;
      std::getline(f, line);
      rc = block(f, path, g, P.cyH, true);
      if (rc) return rc;
      std::getline(f, line);
      std::getline(f, line);
    }
  }
  {
    std::string pr = wd + "/bc_betabetap_real.dat", pi = wd + "/bc_betabetap_imag.dat";
    std::ifstream fr(pr), fi(pi);
    if (!fr) return fail(EDUS_EIO, "cannot read %s", pr.c_str());
    if (!fi) return fail(EDUS_EIO, "cannot read %s", pi.c_str());
    std::string line;
    for (size_t g = 0; g < g2; g++) {
      std::vector<cd>* dst[2] = {&P.cyDx, &P.cyDy};
      for (int x = 0; x < 2; x++) {
        int rc = block(fr, pr, g, *dst[x], false);
        if (!rc) rc = block(fi, pi, g, *dst[x], true);
        if (rc) return rc;
        std::getline(fr, line);
        std::getline(fi, line);
      }
      std::getline(fr, line);
      std::getline(fi, line);
    }
  }
  return 0;
}

// The Crystal model's periodic bicubic interpolation of one sampled element
// (headers/Interpolation.h:120-146, 254-264, the two-dimensional case): the
// grid spacing is 1/(nkf-1) from -0.5 and the nkf samples repeat with period
// nkf; inside a cell the value is the Catmull-Rom cubic in k2 of the four rows'
// Catmull-Rom cubics in k1, written here as the tensor product of the two
// one-dimensional weight vectors.
cd crystal_interp(const Problem& P, const std::vector<cd>& tab, int e, const double* k) {
  const int N = P.cy_nkf;
  const double h = 1. / (N - 1);
  int ci[2];
  double t[2];
  for (int x = 0; x < 2; x++) {
    double u = std::fmod((k[x + 1] + 0.5) / h, (double)N);
    if (u < 0) u += N;
    const int c = (int)std::floor(u);
    ci[x] = c;
    t[x] = u - c;
  }
  double w[2][4];
  for (int x = 0; x < 2; x++) {
    const double s = t[x], s2 = s * s, s3 = s2 * s;
    w[x][0] = -0.5 * s + s2 - 0.5 * s3;
    w[x][1] = 1. - 2.5 * s2 + 1.5 * s3;
    w[x][2] = 0.5 * s + 2. * s2 - 1.5 * s3;
    w[x][3] = -0.5 * s2 + 0.5 * s3;
  }
  const cd* g = &tab[(size_t)e * N * N];
  cd acc = 0;
  for (int r = 0; r < 4; r++) {
    const int i1 = ((ci[0] - 1 + r) % N + N) % N;
    cd row = 0;
    for (int c = 0; c < 4; c++) row += w[1][c] * g[(size_t)i1 * N + ((ci[1] - 1 + c) % N + N) % N];
    acc += w[0][r] * row;
  }
  return acc;
}

int read_coulomb(Problem& P, const char* workdir) {
  int n = P.ncv, n2 = n * n, c2 = P.ncut * P.ncut;
  std::string wd = workdir ? workdir : ".";
  std::string lab = P.p.coulomb_label;
  {
    std::string path = wd + "/Output/Coulomb/V_Hartree_" + lab + ".txt";
    std::ifstream f(path);
    if (!f) return fail(EDUS_EIO, "cannot read %s", path.c_str());
    P.VH.assign((size_t)n * n, 0);
    for (int i = 0; i < n * n; i++) f >> P.VH[i];
    if (!f) return fail(EDUS_EIO, "truncated %s", path.c_str());
  }
  const char* nm[4] = {"A", "B", "C", "D"};
  std::vector<cd>* dst[4] = {&P.cA, &P.cB, &P.cC, &P.cD};
  for (int q = 0; q < 4; q++) {
    std::string path = wd + "/Output/Coulomb/" + nm[q] + "_coeff" + lab + ".txt";
    std::ifstream f(path);
    if (!f) return fail(EDUS_EIO, "cannot read %s", path.c_str());
    dst[q]->assign((size_t)c2 * n2, 0);
    for (size_t i = 0; i < (size_t)c2 * n2; i++) {
      double re, im;
      f >> re >> im;
      (*dst[q])[i] = cd(re, im);
    }
    if (!f) return fail(EDUS_EIO, "truncated %s (need %d x %d complex)", path.c_str(), c2, n2);
  }
  {
    std::string path = wd + "/Output/Coulomb/Screen_const_" + lab + ".txt";
    std::ifstream f(path);
    if (!f) return fail(EDUS_EIO, "cannot read %s", path.c_str());
    P.screen.assign(n2, 0);
    for (int i = 0; i < n2; i++) {
      double re, im;
      f >> re >> im;
      P.screen[i] = cd(re, im);
    }
    if (!f) return fail(EDUS_EIO, "truncated %s", path.c_str());
  }
  return 0;
}

// One k point as Source_Main/save_HUD.cpp:19-53 stores it: the model's H, U, D
// (gHUD, headers/HUD.h:5-20), the scissor shift of the conduction bands added to
// H, and the Wannier dipole made symmetric, D := (D + D^T)/2.
void eval_k(const Problem& P, const Tb& tb, const double* k, cd* H, cd* U, cd* D) {
  const int n = P.ncv, nr = P.nrpts;
  const bool isW = P.p.mode == EDUS_MODE_WANNIER;
  cd Hk[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Uk[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Dk[EDUS_MAX_BANDS * EDUS_MAX_BANDS * 3];
  if (isW) {
    std::vector<cd> ph(nr);
    for (int iR = 0; iR < nr; iR++) {
      double kR = 0.;
      for (int l = 0; l < 3; l++) kR += k[l] * P.Rvec[iR * 3 + l];
      kR *= 2 * kPi;
      ph[iR] = cd(std::cos(kR), std::sin(kR));
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        cd h = 0, d[3] = {0, 0, 0};
        for (int iR = 0; iR < nr; iR++) {
          h += ph[iR] * P.HR[((size_t)i * n + j) * nr + iR];
          for (int x = 0; x < 3; x++) d[x] += ph[iR] * P.rR[(((size_t)x * n + i) * n + j) * nr + iR];
        }
        Hk[i * n + j] = (i == j) ? cd(h.real(), 0.) : h;
        for (int x = 0; x < 3; x++) Dk[(i * n + j) * 3 + x] = (i == j) ? cd(d[x].real(), 0.) : d[x];
      }
    cd A[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Z[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    double ev[EDUS_MAX_BANDS];
    std::copy(Hk, Hk + n * n, A);
    eig_herm(n, A, ev, Z);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) Uk[i * n + j] = std::conj(Z[j * n + i]);
  } else if (P.p.mode == EDUS_MODE_CRYSTAL) {
    // headers/Crystal_interface.h:212-304: H and D from the interpolants (the
    // upper triangle as the conjugate of the lower), D in the order (z, x, y)
    // with real diagonals, U^dagger the eigenvectors of H
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        const int lo = i >= j ? i : j, hi = i >= j ? j : i, e = lo * (lo + 1) / 2 + hi;
        cd h = crystal_interp(P, P.cyH, e, k), dx = crystal_interp(P, P.cyDx, e, k), dy = crystal_interp(P, P.cyDy, e, k);
        if (i < j) {
          h = std::conj(h);
          dx = std::conj(dx);
          dy = std::conj(dy);
        }
        if (i == j) {
          dx = dx.real();
          dy = dy.real();
        }
        Hk[i * n + j] = h;
        Dk[(i * n + j) * 3 + 0] = 0.;
        Dk[(i * n + j) * 3 + 1] = dx;
        Dk[(i * n + j) * 3 + 2] = dy;
      }
    cd A[EDUS_MAX_BANDS * EDUS_MAX_BANDS], Z[EDUS_MAX_BANDS * EDUS_MAX_BANDS];
    double ev[EDUS_MAX_BANDS];
    std::copy(Hk, Hk + n * n, A);
    eig_herm(n, A, ev, Z);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) Uk[i * n + j] = std::conj(Z[j * n + i]);
  } else {
    double kc[3];
    crys_to_cart(P, k, kc);
    tb_eval(tb, n, k, kc, Hk, Uk, Dk);
  }
  double S[EDUS_MAX_BANDS];
  const double gapc = P.p.conduction_shift;
  for (int i = 0; i < n; i++) S[i] = (gapc > 1e-16 && i >= P.p.nb[1]) ? gapc : 0.0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      cd value = 0.;
      if (gapc > 1e-16)
        for (int ii = 0; ii < n; ii++) value += std::conj(Uk[ii * n + i]) * S[ii] * Uk[ii * n + j];
      H[i * n + j] = Hk[i * n + j] + value;
      U[i * n + j] = Uk[i * n + j];
      for (int x = 0; x < 3; x++)
        D[(i * n + j) * 3 + x] = isW ? 0.5 * (Dk[(i * n + j) * 3 + x] + Dk[(j * n + i) * 3 + x]) : Dk[(i * n + j) * 3 + x];
    }
}

}  // namespace

int model_hud(const Problem& P, const double* kcrys, cd* H, cd* U, cd* D) {
  Tb tb;
  if (P.p.mode == EDUS_MODE_TB) {
    int rc = tb_setup(P.p, tb);
    if (rc) return rc;
  }
  eval_k(P, tb, kcrys, H, U, D);
  return 0;
}

int build_problem(const edus_params& p, const char* workdir, Problem& P, bool defer_model) {
  P = Problem();
  P.p = p;
  P.nch = p.nb[0];
  P.nv = p.nb[1];
  P.nc = p.nb[2];
  P.ncv = P.nch + P.nv + P.nc;
  P.nbands = P.nch + P.nv;
  const int n = P.ncv;
  if (n < 1 || n > EDUS_MAX_BANDS) return fail(EDUS_EINVAL, "band count %d outside 1..%d", n, EDUS_MAX_BANDS);
  if (p.dt <= 0) return fail(EDUS_EINVAL, "dt must be positive");
  if (p.solver != EDUS_SOLVER_RK4 && (p.order < 1 || p.order > 8)) return fail(EDUS_EINVAL, "solver order %d out of range", p.order);
  if (p.solver == EDUS_SOLVER_TAYLOR && p.order < 2) return fail(EDUS_EINVAL, "Taylor order must be >= 2");
  int rc = 0;
  if (p.mode == EDUS_MODE_CRYSTAL) {
    // the lattice and the model come from the crystal files (Source_Main/input.cpp:57)
    rc = read_crystal(P, workdir);
    if (rc) return rc;
  }
  rc = setup_geometry(P);
  if (rc) return rc;
  const int nk = P.nk;
  const size_t st = (size_t)nk * n * n;
  const bool isW = p.mode == EDUS_MODE_WANNIER;
  // a deferred Wannier model keeps only H(R), r(R); the device tabulates it
  P.model_deferred = isW && defer_model;
  const size_t sk = P.model_deferred ? 0 : st;
  P.H.assign(sk, 0);
  P.U.assign(sk, 0);
  P.D.assign(sk * 3, 0);
  Tb tb;
  if (isW) {
    rc = read_wannier(P, workdir);
  } else if (p.mode == EDUS_MODE_TB) {
    rc = tb_setup(p, tb);
  }
  if (rc) return rc;
  if (!P.model_deferred) {
#pragma omp parallel for schedule(static)
    for (int ik = 0; ik < nk; ik++)
      eval_k(P, tb, &P.kpt[ik * 3], &P.H[(size_t)ik * n * n], &P.U[(size_t)ik * n * n], &P.D[(size_t)ik * n * n * 3]);
  }
  // gradient of the energy (Source_Main/save_HUD.cpp:96-137)
  P.GE.assign(sk * 3, 0);
  if (p.current && !P.model_deferred) {
#pragma omp parallel for schedule(static)
    for (int ik = 0; ik < nk; ik++)
      for (int x = 0; x < 3; x++)
        for (int i = 0; i < n; i++)
          for (int j = 0; j < n; j++) {
            cd acc = 0;
            for (int b = 0; b < P.nnb; b++) {
              int kb = P.nbr[(size_t)ik * P.nnb + b];
              acc += P.shell_w[P.bshell[b]] * P.bvec[b * 3 + x] * (P.H[((size_t)kb * n + i) * n + j] - P.H[((size_t)ik * n + i) * n + j]);
            }
            P.GE[(((size_t)ik * n + i) * n + j) * 3 + x] = acc;
          }
  }
  // dissipation tensor
  const int nch = P.nch;
  for (int ic = nch; ic < n; ic++)
    for (int jc = nch; jc < n; jc++) P.T[ic][jc] = (ic == jc) ? p.T1 : p.T2;
  for (int ic = 0; ic < nch; ic++) {
    for (int jc = 0; jc < nch; jc++) P.T[ic][jc] = p.Tch;
    for (int jc = nch; jc < n; jc++) P.T[ic][jc] = p.Tch / 2.;
  }
  for (int ic = 0; ic < n; ic++)
    for (int jc = ic + 1; jc < n; jc++) P.T[jc][ic] = P.T[ic][jc];
  for (int ic = 0; ic < n; ic++)
    for (int jc = 0; jc < n; jc++)
      if (std::fabs(P.T[ic][jc]) > 1e-24) {
        P.diss_i.push_back(ic);
        P.diss_j.push_back(jc);
      }
  // initial population (rows/columns swapped as in the reference)
  P.P0.assign(sk, 0);
  for (int ik = 0; ik < (P.model_deferred ? 0 : nk); ik++)
    for (int ia = 0; ia < n; ia++)
      for (int ib = 0; ib < n; ib++) {
        cd acc = 0;
        for (int ii = 0; ii < P.nbands; ii++) acc += P.U[((size_t)ik * n + ii) * n + ia] * std::conj(P.U[((size_t)ik * n + ii) * n + ib]);
        P.P0[((size_t)ik * n + ia) * n + ib] = acc;
      }
  // Coulomb
  if (p.coulomb) {
    if (!p.read_from_files)
      return fail(EDUS_EUNSUPPORTED,
                  "Coulomb coefficients are read from files (Read_Coulomb_from_files); edus_coulomb_generate computes them");
    if (p.ncut < 1 || p.ncut > 64) return fail(EDUS_EINVAL, "Ncut %d out of range", p.ncut);
    if (p.kpt_read) return fail(EDUS_EUNSUPPORTED, "Coulomb with nkpt read (the transforms run on the grid's rows)");
    P.ncut = p.ncut;
    rc = read_coulomb(P, workdir);
    if (rc) return rc;
  }
  // time grid (Source_Main/const_dt_evolution.cpp:1-10)
  P.t_start = -0.21 / kTimeAuFs;
  P.itfi = (int)((p.t_fin - P.t_start) / p.dt);
  P.nsteps = P.itfi + 1;
  int res = p.it_resolution > 0 ? p.it_resolution : 1;
  P.nprint = P.itfi / res + 1;
  return 0;
}

// Drop core bands that no term of the run couples to the other bands: H, D and
// GradientEnergy have no core/non-core entries (or only dipole components the
// pump field never has), the probe is off and nothing dissipates. The core
// rows of the equations of motion are then constant (rho_cc = 1), and the
// remaining block evolves exactly as in the full problem.
int drop_decoupled_core(Problem& P) {
  const int nch = P.nch, n = P.ncv, nk = P.nk;
  if (nch == 0) return fail(EDUS_EINVAL, "no core band to drop");
  if (P.model_deferred) return fail(EDUS_EUNSUPPORTED, "model tables are not tabulated on the host");
  if (!P.diss_i.empty()) return fail(EDUS_EUNSUPPORTED, "core band is coupled: dissipation is on");
  if (P.p.probe.E0 != 0.0) return fail(EDUS_EUNSUPPORTED, "core band is coupled: the probe field is on");
  if (P.p.coulomb) return fail(EDUS_EUNSUPPORTED, "core band is coupled: Coulomb mean field is on");
  bool field_x[3] = {false, false, false};
  for (int ip = 0; ip < P.p.n_pumps; ip++)
    for (int x = 0; x < 3; x++)
      if (P.p.pump[ip].pol1[x] != 0.0 || P.p.pump[ip].pol2[x] != 0.0) field_x[x] = true;
  for (int k = 0; k < nk; k++)
    for (int i = 0; i < nch; i++)
      for (int j = nch; j < n; j++) {
        const size_t ij = ((size_t)k * n + i) * n + j, ji = ((size_t)k * n + j) * n + i;
        if (P.H[ij] != 0.0 || P.H[ji] != 0.0) return fail(EDUS_EUNSUPPORTED, "core band is coupled through H");
        for (int x = 0; x < 3; x++) {
          if (field_x[x] && (P.D[ij * 3 + x] != 0.0 || P.D[ji * 3 + x] != 0.0))
            return fail(EDUS_EUNSUPPORTED, "core band is coupled through the dipole along the field");
          if (P.GE[ij * 3 + x] != 0.0 || P.GE[ji * 3 + x] != 0.0) return fail(EDUS_EUNSUPPORTED, "core band is coupled through dH/dk");
        }
      }
  const int m = n - nch;
  auto shrink = [&](std::vector<cd>& A, int comps) {
    if (A.empty()) return;
    std::vector<cd> B((size_t)nk * m * m * comps);
    for (int k = 0; k < nk; k++)
      for (int i = 0; i < m; i++)
        for (int j = 0; j < m; j++)
          for (int x = 0; x < comps; x++)
            B[(((size_t)k * m + i) * m + j) * comps + x] = A[(((size_t)k * n + i + nch) * n + j + nch) * comps + x];
    A.swap(B);
  };
  // U rows are eigenvectors; the model's non-core rows have no core components
  for (int k = 0; k < nk; k++)
    for (int i = nch; i < n; i++)
      for (int c = 0; c < nch; c++)
        if (P.U[((size_t)k * n + i) * n + c] != 0.0) return fail(EDUS_EUNSUPPORTED, "core band mixes into the band basis");
  shrink(P.H, 1);
  shrink(P.U, 1);
  shrink(P.D, 3);
  shrink(P.GE, 3);
  shrink(P.P0, 1);
  P.ncv = m;
  P.nch = 0;
  P.nbands = P.nv;
  P.p.nb[0] = 0;
  return 0;
}

}  // namespace edus
