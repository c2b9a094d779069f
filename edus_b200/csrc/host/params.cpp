// params.cpp — input.txt reader producing edus_params.
//
// Follows the grammar of the reference's Read_Input (headers/ReadInput.h:332-815)
// and the laser resolution of Laser's setters (headers/Laser.h:29-37,82-106) and
// BZ_parameters (headers/InitParameters.h:1-11). Where the reference reads past
// the end of a token vector or loops forever (blank line after a laser header,
// headers/ReadInput.h:267; "dt 0.1" without units, :493-497) this reader takes the
// evident meaning (skip blank lines, units default to a.u.) and says so in
// edus_last_error only when it must refuse.
#include <strings.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "common.hpp"

namespace edus {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}
void clear_error() { g_last_error.clear(); }

namespace {

// Mirror of the reference Laser's stateful setters; the resulting values depend
// on the order in which keys appear in the section, exactly as there.
struct LaserBuilder {
  edus_laser L{};
  void set_freq(double a) {
    L.wl = a;
    L.lambdanm = 2. * kPi * kC * 0.0529 / L.wl;
    L.period = 2 * kPi / L.wl;
    if (L.intensity != 0) {
      L.A0 = std::sqrt(L.intensity / kLaserIntensityConst) / L.wl;
      L.E0 = L.A0 * L.wl;
    }
    if (L.ncycle != 0) L.tf = L.t0 + L.ncycle * L.period;
  }
  void set_lambdanm(double a) {
    L.lambdanm = a;
    L.wl = 2. * kPi * kC * 0.0529 / L.lambdanm;
    L.period = 2 * kPi / L.wl;
    if (L.intensity != 0) {
      L.A0 = std::sqrt(L.intensity / kLaserIntensityConst) / L.wl;
      L.E0 = L.A0 * L.wl;
    }
    if (L.ncycle != 0) L.tf = L.t0 + L.ncycle * L.period;
  }
  void set_intensity(double a) {
    L.intensity = a;
    if (L.wl != 0) {
      L.A0 = std::sqrt(L.intensity / kLaserIntensityConst) / L.wl;
      L.E0 = L.A0 * L.wl;
    }
  }
  void set_ncycle_sigma(double a) {
    L.ncycle = a;
    L.sigma = a;
    if (L.period != 0) L.tf = L.t0 + L.ncycle * L.period;
  }
  void set_t0(double a) {
    L.t0 = a;
    if (L.tf != 0.) L.tf += L.t0;
  }
  // headers/Laser.h:82-106
  int set_pol(double a0, double a1, double a2, double b0, double b1, double b2) {
    if ((b0 != 0. && b1 != 0. && b2 != 0.) &&
        (std::fabs(a0 / (b0 + 1e-11) - a1 / (b1 + 1e-11)) < 1e-9 && std::fabs(a1 / (b1 + 1e-11) - a2 / (b2 + 1e-11)) < 1e-9))
      return fail(EDUS_EPARSE, "care! you defined a plane with two parallel vectors!");
    if (std::fabs(a0 * b0 + a1 * b1 + a2 * b2) >= 1e-7) {
      double f = (a0 * b0 + a1 * b1 + a2 * b2) / (a0 * a0 + a1 * a1 + a2 * a2);
      b0 -= f * a0;
      b1 -= f * a1;
      b2 -= f * a2;
      double v = std::sqrt(b0 * b0 + b1 * b1 + b2 * b2);
      b0 /= v;
      b1 /= v;
      b2 /= v;
    }
    L.pol1[0] = a0;
    L.pol1[1] = a1;
    L.pol1[2] = a2;
    L.pol2[0] = b0;
    L.pol2[1] = b1;
    L.pol2[2] = b2;
    return 0;
  }
};

bool ieq(const std::string& a, const char* b) { return strcasecmp(a.c_str(), b) == 0; }

// headers/ReadInput.h:1-33: split on ' ' only, up to pos.
std::vector<std::string> split(const std::string& s, size_t pos) {
  std::vector<std::string> out;
  std::string cur;
  std::string t = s.substr(0, std::min(pos, s.size()));
  for (char c : t) {
    if (c != ' ') {
      cur += c;
    } else if (!cur.empty()) {
      out.push_back(cur);
      cur.clear();
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

bool has_close(const std::string& s) { return s.find('}') != std::string::npos; }

void recip(const double a[3][3], double b[3][3]) {
  // headers/crystal.h VecProd/DotProd + ReadInput.h:388-391
  auto cross = [](const double* x, const double* y, double* r) {
    r[0] = (x[1] * y[2] - x[2] * y[1]);
    r[1] = (x[2] * y[0] - x[0] * y[2]);
    r[2] = (x[0] * y[1] - x[1] * y[0]);
  };
  cross(a[1], a[2], b[0]);
  cross(a[2], a[0], b[1]);
  cross(a[0], a[1], b[2]);
  for (int i = 0; i < 3; i++) {
    double v = (a[i][0] * b[i][0] + a[i][1] * b[i][1] + a[i][2] * b[i][2]) / 2. / kPi;
    b[i][0] /= v;
    b[i][1] /= v;
    b[i][2] /= v;
  }
}

struct Reader {
  std::ifstream in;
  bool next(std::string& s) {
    if (!std::getline(in, s)) return false;
    if (!s.empty() && s.back() == '\r') s.pop_back();
    return true;
  }
};

// End_Section (headers/ReadInput.h:54-81)
int end_section(Reader& r, const char* name) {
  std::string s;
  while (r.next(s)) {
    if (s.empty()) continue;
    bool blank = s.find_first_not_of(' ') == std::string::npos;
    if (blank) continue;
    if (!has_close(s)) return fail(EDUS_EPARSE, "Cannot find end of %s. Correct your input.", name);
    return 0;
  }
  return 0;
}

double to_d(const std::vector<std::string>& v, size_t i) { return i < v.size() ? std::atof(v[i].c_str()) : 0.0; }

// headers/ReadInput.h:135-159
int read_polarization(const std::vector<std::string>& str, LaserBuilder& lb) {
  if (str.size() < 2) return fail(EDUS_EPARSE, "polarization needs components");
  if (ieq(str[1], "circular")) {
    if (str.size() < 8) return fail(EDUS_EPARSE, "circular polarization needs 6 components");
    double v1 = to_d(str, 2), v2 = to_d(str, 3), v3 = to_d(str, 4), v4 = to_d(str, 5), v5 = to_d(str, 6), v6 = to_d(str, 7);
    double v = std::sqrt(v1 * v1 + v2 * v2 + v3 * v3);
    v1 /= v;
    v2 /= v;
    v3 /= v;
    v = std::sqrt(v4 * v4 + v5 * v5 + v6 * v6);
    v4 /= v;
    v5 /= v;
    v6 /= v;
    return lb.set_pol(v1, v2, v3, v4, v5, v6);
  }
  if (ieq(str[1], "linear"))
    return fail(EDUS_EPARSE, "'polarization linear x y z' reads the word 'linear' as a number in the reference; write 'polarization x y z'");
  if (str.size() == 4) {
    double v1 = to_d(str, 1), v2 = to_d(str, 2), v3 = to_d(str, 3);
    double v = std::sqrt(v1 * v1 + v2 * v2 + v3 * v3);
    return lb.set_pol(v1 / v, v2 / v, v3 / v, 0., 0., 0.);
  }
  return 0;
}

int read_pump(Reader& r, const std::vector<std::string>& head, LaserBuilder& lb, bool& gaussian, double& sigma) {
  // headers/ReadInput.h:236-326
  bool pw = false, sin2 = false;
  double t0 = 0;
  gaussian = false;
  if (head.size() < 2) return fail(EDUS_EPARSE, "in laserpump you have to specify laser type: gaussian or sin2.");
  if (ieq(head[1], "gaussian"))
    gaussian = true;
  else if (head[1] == "sin2")
    sin2 = true;
  else if (head[1] == "pw")
    pw = true;
  else
    return fail(EDUS_EPARSE, "Allowed types for laserpump: gaussian, sin2. Your type \"%s\" is not available.", head[1].c_str());
  lb.L.envelope_kind = gaussian ? EDUS_ENV_GAUSS : (sin2 ? EDUS_ENV_SIN2 : EDUS_ENV_PW);
  lb.L.envelope_only = 0;
  std::string s;
  if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of laserpump section.");
  while (!has_close(s) || s.empty()) {
    auto str = split(s, s.size());
    if (!str.empty()) {
      const std::string& k = str[0];
      if (ieq(k, "frequency")) {
        if (str.size() != 2) return fail(EDUS_EPARSE, "Cannot understand %s as units.", str.size() > 2 ? str[2].c_str() : "");
        lb.set_freq(to_d(str, 1));
      } else if (ieq(k, "phase")) {
        lb.L.phase = to_d(str, 1);
      } else if (ieq(k, "window")) {
        if (!pw) return fail(EDUS_EPARSE, "You defined a window for a pulse that is not pseudoPW!! Error.");
        double w1 = to_d(str, 1), w2 = to_d(str, 2);
        if (str.size() > 3 && ieq(str[3], "fs")) {
          w1 *= kTimeFsAu;
          w2 *= kTimeFsAu;
        }
        lb.L.w1 = w1;
        lb.L.w2 = w2;
      } else if (ieq(k, "wavelength")) {
        if (str.size() == 2 || (str.size() > 2 && ieq(str[2], "nm")))
          lb.set_lambdanm(to_d(str, 1));
        else if (ieq(str[2], "au") || ieq(str[2], "atomicunit"))
          lb.set_lambdanm(to_d(str, 1) * 10. * kSpaceAuA);
        else
          return fail(EDUS_EPARSE, "Cannot understand %s as units.", str[2].c_str());
      } else if (ieq(k, "intensity")) {
        if (str.size() == 2 || (str.size() > 2 && ieq(str[2], "wcm2")))
          lb.set_intensity(to_d(str, 1));
        else if (ieq(str[2], "au") || ieq(str[2], "atomicunit"))
          lb.set_intensity(to_d(str, 1) * kIntensityAuWcm2);
        else
          return fail(EDUS_EPARSE, "Cannot understand %s as units.", str[2].c_str());
      } else if (ieq(k, "polarization")) {
        int rc = read_polarization(str, lb);
        if (rc) return rc;
      } else if (ieq(k, "sigma")) {
        if (sin2) return fail(EDUS_EPARSE, "You can't define sigma for sin2 wave. Change your input.");
        if (str.size() < 3)
          sigma = to_d(str, 1);
        else if (ieq(str[2], "fs"))
          sigma = to_d(str, 1) * kTimeFsAu;
        else if (ieq(str[2], "au") || ieq(str[2], "atomicunit"))
          sigma = to_d(str, 1);
        lb.set_ncycle_sigma(sigma);
      } else if (ieq(k, "cycles")) {
        if (gaussian) return fail(EDUS_EPARSE, "You can't define cycles for gaussian wave. Change your input.");
        sigma = to_d(str, 1);
        lb.set_ncycle_sigma(sigma);
      } else if (ieq(k, "t0_pulse")) {
        t0 = to_d(str, 1);
        if (str.size() > 2 && ieq(str[2], "fs")) t0 *= kTimeFsAu;
      } else {
        return fail(EDUS_EPARSE, "cannot recognize key %s", s.c_str());
      }
    }
    if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of laserpump section.");
  }
  if (gaussian) t0 += 4. * sigma;
  lb.set_t0(t0);
  return 0;
}

// Lattice and band counts per TB type (headers/ReadInput.h:857-891).
int set_tb_type(edus_params* p, const std::vector<std::string>& str) {
  std::string t = str[1];
  snprintf(p->tb_type, sizeof(p->tb_type), "%s", t.c_str());
  double (*a)[3] = p->a;
  auto hexa = [&](double lc, double ang, bool cos_both) {
    a[0][0] = 6.3303100000;
    a[0][1] = 0.0;
    a[0][2] = 0.0;
    a[1][0] = 0.0;
    a[1][1] = lc * std::cos(ang);
    a[1][2] = cos_both ? lc * std::cos(ang) : lc * std::sin(ang);
    a[2][0] = 0.0;
    a[2][1] = lc * std::cos(ang);
    a[2][2] = cos_both ? -lc * std::cos(ang) : -lc * std::sin(ang);
  };
  auto setnb = [&](int c, int v, int cc) {
    p->nb[0] = c;
    p->nb[1] = v;
    p->nb[2] = cc;
  };
  const char* s = t.c_str();
  if (ieq(t, "graphene") || ieq(t, "GrapheneZurron")) {
    hexa(2.46 * kSpaceAAu, kPi / 6., false);
    setnb(0, 1, 1);
  } else if (ieq(t, "CoreGraphene") || ieq(t, "Graphene_costD") || ieq(t, "Graphene_symmetricD")) {
    hexa(2.46 * kSpaceAAu, kPi / 6., false);
    setnb(2, 1, 1);
  } else if (ieq(t, "BoronNitride")) {
    hexa(2.5 * kSpaceAAu, kPi / 6., false);
    setnb(0, 1, 1);
  } else if (ieq(t, "CoreBN_Nedge") || ieq(t, "CoreBN_Bedge")) {
    hexa(2.5 * kSpaceAAu, kPi / 6., false);
    setnb(1, 1, 1);
  } else if (ieq(t, "BN1b")) {
    hexa(2.5 * kSpaceAAu, kPi / 6., true);
    setnb(0, 1, 0);
  } else if (ieq(t, "DLGraphene")) {
    double v[3][3] = {{6.33031, 0, 0}, {0, 4.02574074, -2.324263}, {0, 4.02574074, 2.324263}};
    memcpy(a, v, sizeof(v));
    setnb(0, 2, 2);
  } else if (ieq(t, "Vampa2015")) {
    double v[3][3] = {{5.32, 0, 0}, {0, 6.14, 0}, {0, 0, 9.83}};
    memcpy(a, v, sizeof(v));
    setnb(0, 1, 1);
  } else if (ieq(t, "GeS") || ieq(t, "GeS_HSE06")) {
    double ax = (4.53 / 2.) * kSpaceAAu, ay = (3.63 / 2.) * kSpaceAAu;
    double v[3][3] = {{6.33031, 0, 0}, {0, ax, ay}, {0, ax, -ay}};
    memcpy(a, v, sizeof(v));
    setnb(0, 1, 1);
  } else if (ieq(t, "Haldane_CoreBN_Bedge") || ieq(t, "Haldane_CoreBN_Nedge")) {
    hexa(2.5 * kSpaceAAu, 1.0 * kPi / 6., false);
    setnb(1, 1, 1);
    p->n_hopping = 4;
    for (int i = 0; i < 4; i++) p->hopping[i] = 0;
    for (size_t i = 2; i < str.size(); i++) {
      double nxt = (i + 1 < str.size()) ? std::atof(str[i + 1].c_str()) : 0.0;
      if (ieq(str[i], "gap="))
        p->hopping[0] = nxt * kEnergyEvAu;
      else if (ieq(str[i], "t1="))
        p->hopping[1] = nxt * kEnergyEvAu;
      if (ieq(str[i], "t2="))
        p->hopping[2] = nxt * kEnergyEvAu;
      else if (ieq(str[i], "phi0="))
        p->hopping[3] = nxt;
    }
  } else if (ieq(t, "gen2d_hexagonal")) {
    p->n_hopping = 8;
    for (int i = 0; i < 8; i++) p->hopping[i] = 0;
    for (size_t i = 2; i < str.size(); i++) {
      double nxt = (i + 1 < str.size()) ? std::atof(str[i + 1].c_str()) : 0.0;
      if (ieq(str[i], "a="))
        p->hopping[0] = nxt * kSpaceAAu;
      else if (ieq(str[i], "gap="))
        p->hopping[1] = nxt * kEnergyEvAu;
      else if (ieq(str[i], "t1="))
        p->hopping[2] = nxt * kEnergyEvAu;
      else if (ieq(str[i], "t2="))
        p->hopping[3] = nxt * kEnergyEvAu;
      else if (ieq(str[i], "phi0="))
        p->hopping[4] = nxt;
      else if (ieq(str[i], "core="))
        p->hopping[5] = nxt * kEnergyEvAu;
      else if (ieq(str[i], "chv_dipole="))
        p->hopping[6] = nxt;
      else if (ieq(str[i], "chc_dipole="))
        p->hopping[7] = nxt;
    }
    hexa(p->hopping[0], kPi / 6., false);
    setnb(1, 1, 1);
  }
  (void)s;
  recip(p->a, p->b);
  p->mode = EDUS_MODE_TB;
  return 0;
}

int read_units_time(const std::vector<std::string>& str, double& out, const char* what) {
  // dt / t_fin (headers/ReadInput.h:491-530)
  if (str.size() < 2) return fail(EDUS_EPARSE, "%s needs a value", what);
  if (str.size() == 2 || ieq(str[2], "au") || ieq(str[2], "atomicunit"))
    out = to_d(str, 1);
  else if (ieq(str[2], "fs"))
    out = to_d(str, 1) * kTimeFsAu;
  else
    return fail(EDUS_EPARSE, "Units %s aren't allowed for dt.", str[2].c_str());
  return 0;
}

int read_decoherence_value(const std::vector<std::string>& str, double& out) {
  out = to_d(str, 1);
  if (str.size() == 3) {
    if (ieq(str[2], "meV"))
      out *= kEnergyEvAu / 1000.;
    else if (!(ieq(str[2], "au") || ieq(str[2], "atomicunit")))
      return fail(EDUS_EPARSE, "Can't understand units %s in decoherence.", str[2].c_str());
  }
  return 0;
}

}  // namespace
}  // namespace edus

using namespace edus;

extern "C" const char* edus_last_error(void) { return g_last_error.c_str(); }

extern "C" int edus_params_default(edus_params* p) {
  // Source_Main/variables.cpp:8-123
  if (!p) return EDUS_EINVAL;
  memset(p, 0, sizeof(*p));
  p->ncut = 30;
  p->dt = 0.1;
  p->it_resolution = 10;
  p->tabs = 1;
  p->current = 0;
  p->vectorization = 1;
  p->epsilon_static = 1.0;
  p->G_distance = 50;
  p->r0 = 18.89726;
  snprintf(p->coulomb_label, sizeof(p->coulomb_label), "_");
  p->solver = EDUS_SOLVER_RK4;
  p->order = 5;
  p->eps_step_abs = 1e-2;
  p->print_start = 0.0;
  p->print_end = 100.0 * kTimeAuFs;
  p->print_step = 20.0 * kTimeAuFs;
  for (int i = 0; i < 3; i++) {
    p->a[i][i] = 1.;
    p->b[i][i] = 1.;
  }
  p->n_pumps = 1;
  p->precision = EDUS_PREC_FP64;
  return 0;
}

extern "C" int edus_parse_input(const char* path, edus_params* out) {
  clear_error();
  if (!path || !out) return fail(EDUS_EINVAL, "null argument");
  edus_params P;
  edus_params_default(&P);
  Reader r;
  r.in.open(path);
  if (!r.in.is_open()) return fail(EDUS_EIO, "error opening file %s", path);
  {
    char full[4096];
    snprintf(P.input_path, sizeof(P.input_path), "%s", realpath(path, full) ? full : path);
  }
  std::string ref;
  r.in >> ref;
  snprintf(P.ref_coord, sizeof(P.ref_coord), "%s", ref.c_str());
  std::vector<LaserBuilder> pumps(1);
  LaserBuilder probe;
  probe.L.envelope_only = 1;
  bool gaussian1 = false, have_g1 = false;
  double sigma1 = 0;
  int i_pump = 0, num_pump = 1;
  double delay = 0;
  bool have_probe = false;
  std::string s;
  while (r.next(s)) {
    if (s.empty()) continue;
    if (s.find_first_not_of(' ') == std::string::npos) continue;
    size_t pos = s.find('{');
    if (pos == std::string::npos)
      return fail(EDUS_EPARSE, "Can't find the character { in the string \" %s \". Please, review your input.", s.c_str());
    auto str = split(s, pos);
    if (str.empty()) return fail(EDUS_EPARSE, "section without name: %s", s.c_str());
    const std::string& key = str[0];
    int rc = 0;
    if (ieq(key, "unitcell")) {
      double* a = &P.a[0][0];
      for (int i = 0; i < 9; i++)
        if (!(r.in >> a[i])) return fail(EDUS_EPARSE, "Cannot read unit cell because the file ended. Correct your input.");
      recip(P.a, P.b);
      if (str.size() == 2) {
        if (ieq(str[1], "angstrom")) {
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
              P.a[i][j] *= kSpaceAAu;
              P.b[i][j] /= kSpaceAAu;
            }
        }
      }
      rc = end_section(r, "unitcell");
    } else if (ieq(key, "nkpt")) {
      if (!(r.in >> P.nk[0] >> P.nk[1] >> P.nk[2])) return fail(EDUS_EPARSE, "Cannot read Nkpt because the file ended. Correct your input.");
      if (str.size() == 2) {
        if (ieq(str[1], "read")) {
          // the listed k points follow; set-up reads them again from the file
          P.kpt_read = 1;
          P.kpt_offset = (int64_t)r.in.tellg();
          const long nl = (long)P.nk[0] * P.nk[1] * P.nk[2];
          for (long q = 0; q < nl; q++) {
            double k0, k1, k2;
            if (!(r.in >> k0 >> k1 >> k2)) return fail(EDUS_EPARSE, "nkpt read: %ld k points expected", nl);
          }
        }
      }
      rc = end_section(r, "nkpt");
    } else if (ieq(key, "bands")) {
      s.clear();
      while (s.empty())
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of bands section.");
      while (!has_close(s) || s.empty()) {
        auto t = split(s, s.size());
        if (!t.empty()) {
          if (ieq(t[0], "conduction"))
            P.nb[2] = std::atoi(t.size() > 1 ? t[1].c_str() : "0");
          else if (ieq(t[0], "valence"))
            P.nb[1] = std::atoi(t.size() > 1 ? t[1].c_str() : "0");
          else if (ieq(t[0], "core"))
            P.nb[0] = std::atoi(t.size() > 1 ? t[1].c_str() : "0");
          else if (ieq(t[0], "conduction_shift"))
            P.conduction_shift = to_d(t, 1);
          else
            return fail(EDUS_EPARSE, "Can't recognize band type %s. Possible band types: conduction, valence, core.", t[0].c_str());
        }
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of bands section.");
      }
    } else if (ieq(key, "laserpump")) {
      if (i_pump >= num_pump) return fail(EDUS_EPARSE, "more laserpump sections than num_pump_pulses");
      LaserBuilder lb;
      rc = read_pump(r, str, lb, gaussian1, sigma1);
      have_g1 = true;
      if (!rc) pumps[i_pump++] = lb;
    } else if (ieq(key, "laserprobe")) {
      // headers/ReadInput.h:492-728
      have_probe = true;
      bool g2 = false, sin2 = false, pw = false;
      double sigma2 = 0;
      if (str.size() < 2) return fail(EDUS_EPARSE, "in laserprobe you have to specify laser type: gaussian or sin2.");
      if (ieq(str[1], "gaussian"))
        g2 = true;
      else if (str[1] == "sin2")
        sin2 = true;
      else if (str[1] == "pw")
        pw = true;
      else
        return fail(EDUS_EPARSE, "Allowed types for laserprobe: gaussian, sin2.");
      if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of laserprobe section.");
      probe.L.envelope_only = 1;
      probe.L.envelope_kind = g2 ? EDUS_ENV_GAUSS : (sin2 ? EDUS_ENV_SIN2 : EDUS_ENV_PW);
      while (!has_close(s) || s.empty()) {
        auto t = split(s, s.size());
        if (!t.empty()) {
          const std::string& k = t[0];
          if (ieq(k, "frequency")) {
            if (t.size() != 2) return fail(EDUS_EPARSE, "Cannot understand units of frequency");
            probe.set_freq(to_d(t, 1));
          } else if (ieq(k, "wavelength")) {
            if (t.size() == 2 || ieq(t[2], "nm"))
              probe.set_lambdanm(to_d(t, 1));
            else if (ieq(t[2], "au") || ieq(t[2], "atomicunit"))
              probe.set_lambdanm(to_d(t, 1) * 10. * kSpaceAuA);
            else
              return fail(EDUS_EPARSE, "Cannot understand %s as units.", t[2].c_str());
          } else if (ieq(k, "window")) {
            if (!pw) return fail(EDUS_EPARSE, "You defined a window for a pulse that is not pseudoPW!! Error.");
            double w1 = to_d(t, 1), w2 = to_d(t, 2);
            if (t.size() > 3 && ieq(t[3], "fs")) {
              w1 *= kTimeFsAu;
              w2 *= kTimeFsAu;
            }
            probe.L.w1 = w1;
            probe.L.w2 = w2;
          } else if (ieq(k, "intensity")) {
            if (t.size() == 2 || ieq(t[2], "wcm2"))
              probe.set_intensity(to_d(t, 1));
            else if (ieq(t[2], "au") || ieq(t[2], "atomicunit"))
              probe.set_intensity(to_d(t, 1) * kIntensityAuWcm2);
            else
              return fail(EDUS_EPARSE, "Cannot understand %s as units.", t[2].c_str());
          } else if (ieq(k, "polarization")) {
            rc = read_polarization(t, probe);
            if (rc) return rc;
          } else if (ieq(k, "sigma")) {
            if (sin2) return fail(EDUS_EPARSE, "You can't define sigma for sin2 wave. Change your input.");
            if (t.size() < 3)
              sigma2 = to_d(t, 1);
            else if (ieq(t[2], "fs"))
              sigma2 = to_d(t, 1) * kTimeFsAu;
            else if (ieq(t[2], "au") || ieq(t[2], "atomicunit"))
              sigma2 = to_d(t, 1);
            probe.set_ncycle_sigma(sigma2);
          } else if (ieq(k, "delay")) {
            if (t.size() == 2 || ieq(t[2], "fs"))
              delay = to_d(t, 1) * kTimeFsAu;
            else if (ieq(t[2], "au") || ieq(t[2], "atomicunit"))
              delay = to_d(t, 1);
            else
              return fail(EDUS_EPARSE, "Error in reading time delay. Please review your input.");
          } else if (ieq(k, "cycles")) {
            if (g2) return fail(EDUS_EPARSE, "You can't define cycles for gaussian wave. Change your input.");
            sigma2 = to_d(t, 1);
            probe.set_ncycle_sigma(sigma2);
          }
          // unknown keys: the reference prints a message and continues
        }
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of laserprobe section.");
      }
      double t0;
      if (!have_g1) return fail(EDUS_EPARSE, "laserprobe before any laserpump reads an uninitialised flag in the reference");
      if (gaussian1)
        t0 = 4. * sigma1 + delay;
      else
        t0 = (pumps[0].L.tf - pumps[0].L.t0) / 2. + delay - probe.L.ncycle / 2. * probe.L.period;
      probe.set_t0(t0);
      P.delay = delay;
    } else if (ieq(key, "TDSE")) {
      if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of tdse section.");
      while (!has_close(s)) {
        auto t = split(s, s.size());
        if (!t.empty()) {
          const std::string& k = t[0];
          if (ieq(k, "Wannier")) {
            P.mode = EDUS_MODE_WANNIER;
          } else if (ieq(k, "Crystal")) {
            // headers/ReadInput.h:748-751; the lattice comes from kmesh_data.dat at set-up
            P.mode = EDUS_MODE_CRYSTAL;
          } else if (ieq(k, "tightbinding")) {
            if (t.size() < 2) return fail(EDUS_EPARSE, "Please specify the TightBinding type.");
            rc = set_tb_type(&P, t);
            if (rc) return rc;
          } else if (ieq(k, "FermiEnergy")) {
            if (t.size() >= 3) return fail(EDUS_EPARSE, "FermiEnergy takes one value");
            P.fermi_energy = to_d(t, 1);
          } else if (ieq(k, "dt")) {
            rc = read_units_time(t, P.dt, "dt");
            if (rc) return rc;
          } else if (ieq(k, "t_fin")) {
            rc = read_units_time(t, P.t_fin, "t_fin");
            if (rc) return rc;
          } else if (ieq(k, "epsStepAbs")) {
            P.eps_step_abs = to_d(t, 1);
          } else if (ieq(k, "dynamical_dt_evolution")) {
            P.dynamical_dt = 1;
          } else if (ieq(k, "No_Vectorization")) {
            P.vectorization = 0;
          } else if (ieq(k, "Taylor")) {
            P.solver = EDUS_SOLVER_TAYLOR;
          } else if (ieq(k, "num_pump_pulses")) {
            num_pump = (int)to_d(t, 1);
            if (num_pump < 1 || num_pump > EDUS_MAX_PUMPS) return fail(EDUS_EINVAL, "num_pump_pulses out of range 1..%d", EDUS_MAX_PUMPS);
            pumps.resize(num_pump);
          } else if (ieq(k, "TaylorOrder")) {
            P.order = (int)to_d(t, 1);
          } else if (ieq(k, "Adams_Bashforth")) {
            P.solver = EDUS_SOLVER_AB;
            if (t.size() > 1) P.order = (int)to_d(t, 1);
            if (P.order > 5) P.order = 5;
          } else if (ieq(k, "Adams_Bashforth_RK4_startup")) {
            P.ab_rk4_startup = 1;
          } else if (ieq(k, "velocity_gauge")) {
            P.velocity_gauge = 1;
          } else if (ieq(k, "Gap_correction")) {
            P.gap_correction = to_d(t, 1);
          }
        }
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of tdse section.");
      }
    } else if (ieq(key, "observables")) {
      if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of observables section.");
      while (!has_close(s)) {
        auto t = split(s, s.size());
        if (!t.empty()) {
          const std::string& k = t[0];
          if (ieq(k, "wfd")) {
            // k-distribution movie for an external code: accepted, not written
          } else if (ieq(k, "Current"))
            P.current = 1;
          else if (ieq(k, "it_resolution"))
            P.it_resolution = (int)to_d(t, 1);
          else if (ieq(k, "PrintPopulation")) {
            P.print_population = 1;
            if (t.size() > 1) {
              P.print_start = to_d(t, 1);
              P.print_end = to_d(t, 2);
              P.print_step = to_d(t, 3);
            }
          } else if (ieq(k, "Coulomb_band_reconstruction"))
            P.coulomb = 1;
          else if (ieq(k, "TransientAbsorption") || ieq(k, "TAbs"))
            P.tabs = 1;
          else if (ieq(k, "kresolvedTAbs") || ieq(k, "kTAbs") || ieq(k, "kTransientAbsorption"))
            P.tabs_k = 1;
          else
            return fail(EDUS_EPARSE, "option %s not available in the observables.", k.c_str());
        }
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of observables section.");
      }
    } else if (ieq(key, "TAbsK")) {
      // headers/ReadInput.h:1047-1083: the number of k points, then one
      // "k0 k1 k2" line each (crystal coordinates)
      if (!P.tabs_k)
        return fail(EDUS_EPARSE,
                    "Error in the input. You defined the section TAbsK without putting it in the observables.");
      s.clear();
      while (s.empty())
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of TAbsK section.");
      auto t = split(s, s.size());
      if (t.size() != 1) return fail(EDUS_EPARSE, "Error in TAbsK. you didn't define in the first line the number of k points.");
      const int nt = std::atoi(t[0].c_str());
      if (nt < 0) return fail(EDUS_EPARSE, "Error in TAbsK: %d k points", nt);
      if (nt > EDUS_MAX_TABSK) return fail(EDUS_EUNSUPPORTED, "TAbsK: %d k points (at most %d)", nt, EDUS_MAX_TABSK);
      P.n_tabs_k = nt;
      for (int i = 0; i < nt; i++) {
        if (!r.next(s)) s.clear();
        auto q = split(s, s.size());
        if (q.size() != 3) return fail(EDUS_EPARSE, "Error in defining k points in TAbsK. Please review your input.");
        for (int j = 0; j < 3; j++) P.tabs_k_pts[i][j] = to_d(q, j);
      }
      rc = end_section(r, "TAbsK");
    } else if (ieq(key, "Coulomb")) {
      P.coulomb = 1;
      if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of Coulomb section.");
      while (!has_close(s)) {
        auto t = split(s, s.size());
        if (!t.empty()) {
          const std::string& k = t[0];
          if (ieq(k, "qTF")) P.qTF = to_d(t, 1);
          if (ieq(k, "r0")) P.r0 = to_d(t, 1);
          if (ieq(k, "G_distance")) P.G_distance = to_d(t, 1);
          if (ieq(k, "Rytova_Keldysh")) P.rytova_keldysh = 1;
          if (ieq(k, "epsilon_static")) P.epsilon_static = to_d(t, 1);
          if (ieq(k, "Coulomb_diag_basis")) P.diag_basis = 1;
          if (ieq(k, "Read_Coulomb_from_files")) P.read_from_files = 1;
          if (ieq(k, "labelInput") && t.size() > 1) snprintf(P.coulomb_label, sizeof(P.coulomb_label), "%s", t[1].c_str());
          if (ieq(k, "Print_new_band_dispersion")) P.print_band_dispersion = 1;
          if (ieq(k, "Ncut")) P.ncut = (int)to_d(t, 1);
        }
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of Coulomb section.");
      }
    } else if (ieq(key, "decoherence")) {
      if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of decoherence section.");
      while (!has_close(s)) {
        auto t = split(s, s.size());
        if (!t.empty()) {
          if (t.size() < 2) return fail(EDUS_EPARSE, "You have to specify a number for the decoherence term.");
          if (ieq(t[0], "diagonal"))
            rc = read_decoherence_value(t, P.T1);
          else if (ieq(t[0], "offdiagonal"))
            rc = read_decoherence_value(t, P.T2);
          else if (ieq(t[0], "corehole"))
            rc = read_decoherence_value(t, P.Tch);
          else
            return fail(EDUS_EPARSE, "Unknow key %s in decoherence.", t[0].c_str());
          if (rc) return rc;
        }
        if (!r.next(s)) return fail(EDUS_EPARSE, "Can't find the end of decoherence section.");
      }
    } else {
      // The reference silently ignores unknown section names.
    }
    if (rc) return rc;
  }
  // BZ_parameters (headers/InitParameters.h:1-11): set_pol again on the Cartesian vectors.
  P.n_pumps = num_pump;
  for (int i = 0; i < num_pump; i++) {
    LaserBuilder& lb = pumps[i];
    int rc = lb.set_pol(lb.L.pol1[0], lb.L.pol1[1], lb.L.pol1[2], lb.L.pol2[0], lb.L.pol2[1], lb.L.pol2[2]);
    if (rc) return rc;
    P.pump[i] = lb.L;
  }
  {
    int rc = probe.set_pol(probe.L.pol1[0], probe.L.pol1[1], probe.L.pol1[2], probe.L.pol2[0], probe.L.pol2[1], probe.L.pol2[2]);
    if (rc) return rc;
  }
  if (!have_probe) probe.L.envelope_kind = EDUS_ENV_NONE;
  P.probe = probe.L;
  // Source_Main/input.cpp:65: sample orientation
  P.sample_110 = (P.nk[2] < P.nk[1]) ? 1 : 0;
  // Source_Main/runge_kutta_init.cpp:15-30: default final time = pump duration
  if (!(P.t_fin > 0)) {
    double tf = (P.pump[0].envelope_kind == EDUS_ENV_GAUSS) ? 8 * P.pump[0].sigma : P.pump[0].ncycle * P.pump[0].period;
    int nstep = (int)(tf / P.dt);
    P.t_fin = nstep * P.dt;
  }
  if (P.mode == 0) return fail(EDUS_EPARSE, "iMode = none is incorrect (no tightbinding/Wannier/Crystal in tdse)");
  if (P.nk[0] <= 0 || P.nk[1] <= 0 || P.nk[2] <= 0) return fail(EDUS_EPARSE, "nkpt section missing");
  *out = P;
  return EDUS_OK;
}
