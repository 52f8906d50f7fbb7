// problem.cpp -- host-side problem setup for the grhd2_gpu C-ABI (see include/grhd2_host.h).
//
// Restates the reference's init-time routines: the .par reader (parameters.f90:95-357,
// keys and value syntax), the presets (initialization.f90:483-821), the grid
// (initialization.f90:84-263), the metric cache (initialization.f90:265-391), the analytic
// metrics (metrics.f90:209-1242), the initial conditions (conditions.f90:26-582) and the
// perturbations (conditions.f90:585-768).  Nothing here runs per stage.
#include "grhd2_host.h"
#include "metric_eval.h"

#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

namespace {

const double PI = std::acos(-1.0);  // variables.f90:104
const double EPS = DBL_EPSILON;

enum Geom { CART = 0, CYL = 1, SPH = 2, SPHEROID = 3 };
enum Metric { MINK = 0, EF = 1, KS = 2 };

struct Params {
  int case_id = 0;
  int geom = CART, metric = MINK;
  bool log_r = false, shock_sensor = true;
  int nx = 0, ny = 0, nz = 0, nghost = 0;
  double r_min = 0, r_max = 0, y_min = 0, y_max = 0, z_min = 0, z_max = 0;
  double adb = 0, bh_mass = 0, a_spin = 0;
  int rec = 5, lim = 3, rs = 1;
  double final_time = 0, cfl = 0;
  // perturbation controls (variables.f90:141-157)
  int pert_type = 1;
  bool apply_pert = false;
  long long pert_seed = 3435;
  double pert_time = 1000.0, pert_amp = 0.01, pert_mode = 1.0;
  // initial-condition parameters (variables.f90:165-226)
  double sod_if = 0.5, sod_rl = 1.0, sod_rr = 0.125, sod_pl = 1.0, sod_pr = 0.1;
  double sod_vl = 0.0, sod_vr = 0.0;  // extension: shock-tube velocities (default 0 = reference)
  double st_if = 0.5, st_rl = 1.0, st_rr = 1.0, st_pl = 1000.0, st_pr = 0.01;
  double shu_if = 0.5, shu_rl = 5.0, shu_pl = 50.0, shu_rr = 2.0, shu_amp = 0.3, shu_k = 50.0, shu_pr = 5.0;
  double khi_hw = 0.25, khi_ri = 2.0, khi_ro = 1.0, khi_vi = 0.5, khi_vo = -0.5, khi_p = 2.5;
  double khi_pa = 0.01, khi_pk = 10.0, khi_pw = 0.05;
  double jet_ar = 10.0, jet_ap = 0.01, jet_av = 0.0, jet_nr = 1.0, jet_nl = 1.0, jet_r = 0.1, jet_p = 0.01, jet_v = 0.99;
  double cv_rho = 1.0, cv_amp = 0.1, cv_v = 0.5, cv_p = 1.0, cv_k = 2.0;
  double mi_rc = 100.0, mi_rhoc = 0.1;
  double dust_c = -0.5;
  double oa_rc = 15.0, oa_phic = PI, oa_w = 1.5, oa_bd = 0.1, oa_bp = 0.1, oa_da = 1.0, oa_pa = 1.0;
  double fm_rin = 6.25, fm_rmax = 9.25, fm_k = 0.0015;
  // derived
  double g1 = 0, rho_floor = 0, p_floor = 0;
};

// ------------------------------------------------------------------------------------
// metrics.f90: the analytic 3+1 quantities and the set_metric_type dispatch live in
// metric_eval.h, which the device metric-cache build compiles too.
// ------------------------------------------------------------------------------------
using grhd2_metric::MetricOut;

inline double sq(double x) { return x * x; }

grhd2_metric::Kind metric_kind(const Params &P) {
  return grhd2_metric::Kind{P.metric, P.geom, P.log_r ? 1 : 0, P.ny, P.bh_mass, P.a_spin};
}
void eval_metric(const Params &P, double x, double y, bool want_gmunu, MetricOut &m) {
  grhd2_metric::eval_metric(metric_kind(P), x, y, want_gmunu, m);
}
void eval_chris_dg(const Params &P, double x, double y, double *ch, double *dg) {
  grhd2_metric::eval_chris_dg(metric_kind(P), x, y, ch, dg);
}

}  // namespace

// ------------------------------------------------------------------------------------
// problem object
// ------------------------------------------------------------------------------------
struct grhd2_problem {
  Params P;
  double dx = 0, dy = 0, dz = 0, x_min = 0, x_max = 0;
  std::vector<double> x, y, z, x_face, y_face, z_face;
  // metric tables (k = 1 slices)
  std::vector<double> alpha_c, beta_c, gamma_c, gamma_inv_c, gmunu_c, sqg_c, chris_c, dg_c, dlna_c;
  std::vector<double> a_fx, b_fx, g_fx, s_fx, a_fy, b_fy, g_fy, s_fy, a_fz, b_fz, g_fz, s_fz;
  std::vector<double> p;  // (5,-g:nx+g,-g:ny+g,-g:nz+g)
  std::vector<double> michel_injector, dust_outer;
  double fm_l = 0, fm_w_in = 0;
  bool metric_cache = true;  // false: the tables are built on the device instead

  size_t pidx(int v, int i, int j, int k) const {
    const int g = P.nghost;
    size_t sx = 5, sy = 5 * (size_t)(P.nx + 2 * g + 1), sz = sy * (size_t)(P.ny + 2 * g + 1);
    return (size_t)v + sx * (size_t)(i + g) + sy * (size_t)(j + g) + sz * (size_t)(k + g);
  }
  double &X(int i) { return x[i + P.nghost]; }
  double &Y(int j) { return y[j + P.nghost]; }
  double &Z(int k) { return z[k + P.nghost]; }
};

namespace {

struct ParError {
  std::string msg;
};
[[noreturn]] void fail(const std::string &m) { throw ParError{m}; }

std::string lower(std::string s) {
  for (auto &ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}
std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  return s.substr(a, b - a + 1);
}
double parse_real(const std::string &v) {
  std::string t = v;
  for (auto &ch : t) if (ch == 'd' || ch == 'D') ch = 'e';  // Fortran 1.0d0
  char *end = nullptr;
  double r = std::strtod(t.c_str(), &end);
  if (end == t.c_str() || trim(end).size() != 0) fail("expected a real number: " + v);
  return r;
}
long long parse_int(const std::string &v) {
  char *end = nullptr;
  long long r = std::strtoll(v.c_str(), &end, 10);
  if (end == v.c_str() || trim(end).size() != 0) fail("expected an integer: " + v);
  return r;
}
bool parse_bool(const std::string &v) {
  std::string t = lower(v);
  if (t == "1" || t == "true" || t == ".true." || t == "yes" || t == "si") return true;
  if (t == "0" || t == "false" || t == ".false." || t == "no") return false;
  fail("expected true/false, yes/no or 1/0: " + v);
}
// parameters.f90:808-835: a number or a fraction "a/b", in units of pi
double parse_pi(const std::string &v) {
  size_t s = v.find('/');
  if (s == std::string::npos) return parse_real(v);
  if (s == 0 || s == v.size() - 1 || v.find('/', s + 1) != std::string::npos) fail("invalid pi fraction: " + v);
  double num = parse_real(trim(v.substr(0, s))), den = parse_real(trim(v.substr(s + 1)));
  if (den == 0.0) fail("invalid or zero denominator: " + v);
  return num / den;
}

// initialization.f90:483-821
void apply_preset(Params &P) {
  switch (P.case_id) {
  case 1:
    P.geom = CART; P.metric = MINK; P.shock_sensor = false; P.adb = 1.4;
    P.sod_if = 0.5; P.sod_rl = 1.0; P.sod_rr = 0.125; P.sod_pl = 1.0; P.sod_pr = 0.1;
    P.nx = 200; P.r_min = 0.0; P.r_max = 1.0; P.ny = 1; P.y_min = 0; P.y_max = 1; P.nz = 1; P.z_min = 0; P.z_max = 1;
    P.final_time = 0.4; P.cfl = 0.4;
    break;
  case 2:
    P.geom = CART; P.metric = MINK; P.shock_sensor = false; P.adb = 5.0 / 3.0;
    P.nx = 400; P.r_min = 0.0; P.r_max = 1.0; P.ny = 1; P.y_min = 0; P.y_max = 1; P.nz = 1; P.z_min = 0; P.z_max = 1;
    P.final_time = 0.4; P.cfl = 0.4;
    break;
  case 3:
    P.geom = CART; P.metric = MINK; P.shock_sensor = false; P.adb = 5.0 / 3.0;
    P.nx = 400; P.r_min = 0.0; P.r_max = 1.0; P.ny = 1; P.y_min = 0; P.y_max = 1; P.nz = 1; P.z_min = 0; P.z_max = 1;
    P.final_time = 0.4; P.cfl = 0.4;
    break;
  case 4:
    P.geom = CART; P.metric = MINK; P.shock_sensor = false; P.adb = 5.0 / 3.0;
    P.nx = 400; P.r_min = -0.5; P.r_max = 0.5; P.ny = 1; P.y_min = 0; P.y_max = 1; P.nz = 400; P.z_min = -0.5; P.z_max = 0.5;
    P.final_time = 3.0; P.cfl = 0.25;
    break;
  case 5:
    P.geom = CYL; P.metric = MINK; P.shock_sensor = true; P.adb = 5.0 / 3.0;
    P.nx = 320; P.r_min = 0.0; P.r_max = 16.0; P.ny = 1; P.y_min = 0; P.y_max = PI; P.nz = 800; P.z_min = 0; P.z_max = 40.0;
    P.final_time = 120.0; P.cfl = 0.25;
    break;
  case 6:
    P.geom = CART; P.metric = MINK; P.shock_sensor = false; P.adb = 4.0 / 3.0;
    P.nx = 2048; P.r_min = 0.0; P.r_max = 1.0; P.ny = 1; P.y_min = 0; P.y_max = 1; P.nz = 1; P.z_min = 0; P.z_max = 1;
    P.final_time = 0.7; P.cfl = 0.10;
    break;
  case 7:
    P.geom = SPH; P.metric = EF; P.shock_sensor = false; P.adb = 4.0 / 3.0; P.bh_mass = 1.0;
    P.mi_rc = 100.0; P.mi_rhoc = 0.1;
    P.nx = 400; P.r_min = 1.01; P.r_max = 51.0; P.ny = 1; P.y_min = 0; P.y_max = PI; P.nz = 200; P.z_min = 0; P.z_max = 2.0 * PI;
    P.final_time = 500.0; P.cfl = 0.5;
    break;
  case 8:
    P.geom = SPH; P.metric = EF; P.shock_sensor = true; P.adb = 4.0 / 3.0; P.bh_mass = 1.0; P.dust_c = -0.5;
    P.nx = 500; P.r_min = 1.0; P.r_max = 51.0; P.ny = 1; P.y_min = 0; P.y_max = PI; P.nz = 4; P.z_min = 0; P.z_max = 2.0 * PI;
    P.final_time = 500.0; P.cfl = 0.5;
    break;
  case 9:
    P.geom = SPH; P.metric = EF; P.shock_sensor = true; P.adb = 4.0 / 3.0; P.bh_mass = 1.0;
    P.nx = 400; P.r_min = 1.0; P.r_max = 121.0; P.ny = 1; P.y_min = 0; P.y_max = PI; P.nz = 200; P.z_min = 0; P.z_max = 2.0 * PI;
    P.final_time = 2000.0; P.cfl = 0.4;
    break;
  case 10:
    P.geom = SPHEROID; P.metric = KS; P.shock_sensor = false; P.log_r = true; P.adb = 4.0 / 3.0;
    P.bh_mass = 1.0; P.a_spin = 0.9; P.fm_rin = 6.25; P.fm_rmax = 9.25; P.fm_k = 0.0015;
    P.nx = 400; P.r_min = 1.2; P.r_max = 40.0; P.ny = 1; P.y_min = 0; P.y_max = PI; P.nz = 200; P.z_min = 0; P.z_max = 2.0 * PI;
    P.final_time = 1000.0; P.cfl = 0.4;
    break;
  case 11:
    P.geom = SPH; P.metric = EF; P.shock_sensor = true; P.log_r = true; P.adb = 4.0 / 3.0;
    P.bh_mass = 1.0; P.fm_rin = 6.25; P.fm_rmax = 9.25; P.fm_k = 0.0015;
    P.nx = 400; P.r_min = 2.0; P.r_max = 200.0; P.ny = 200; P.y_min = 0; P.y_max = PI; P.nz = 1; P.z_min = 0; P.z_max = 2.0 * PI;
    P.final_time = 0.0; P.cfl = 0.4;
    break;
  case 12:
    P.geom = SPH; P.metric = EF; P.shock_sensor = true; P.adb = 4.0 / 3.0; P.bh_mass = 1.0;
    P.fm_rin = 6.0; P.fm_rmax = 12.0; P.fm_k = 0.015;
    P.nx = 100; P.r_min = 1.0; P.r_max = 121.0; P.ny = 100; P.y_min = 0; P.y_max = PI; P.nz = 100; P.z_min = 0; P.z_max = 2.0 * PI;
    P.final_time = 35.0; P.cfl = 0.4;
    break;
  default:
    fail("invalid problem identifier");
  }
}

int parse_problem(const std::string &v) {
  std::string t = lower(v);
  if (t == "sod") return 1;
  if (t == "strong_shock" || t == "blast_wave") return 2;
  if (t == "shu_osher") return 3;
  if (t == "kelvin_helmholtz" || t == "khi") return 4;
  if (t == "axisymmetric_jet" || t == "jet") return 5;
  if (t == "convergence" || t == "convergence_test") return 6;
  if (t == "michel" || t == "michel_accretion") return 7;
  if (t == "dust" || t == "dust_accretion") return 8;
  if (t == "offaxis_blast" || t == "off_axis_blast") return 9;
  if (t == "fishbone_equatorial" || t == "fishbone_moncrief_equatorial") return 10;
  if (t == "fishbone_sagittal" || t == "fishbone_sagital" || t == "fishbone_moncrief_sagittal") return 11;
  if (t == "fishbone_3d" || t == "fishbone_moncrief_3d") return 12;
  fail("unknown problem: " + v);
}

bool ic_prefix_applies(const std::string &k, int case_id) {
  static const char *pref[] = {"", "sod_", "strong_", "shu_", "khi_", "jet_", "convergence_", "michel_",
                               "dust_", "offaxis_", "fm_", "fm_", "fm_"};
  if (case_id < 1 || case_id > 12) return false;
  return k.rfind(pref[case_id], 0) == 0;
}
bool is_ic_key(const std::string &k) {
  static const char *pref[] = {"sod_", "strong_", "shu_", "khi_", "jet_", "convergence_", "michel_", "dust_", "offaxis_", "fm_"};
  for (auto p : pref) if (k.rfind(p, 0) == 0) return true;
  return false;
}

// parameters.f90:95-357
void read_par(const std::string &text, Params &P) {
  std::vector<std::pair<std::string, std::string>> kv;
  std::set<std::string> seen;
  std::istringstream in(text);
  std::string line;
  int lineno = 0;
  bool have_problem = false;
  while (std::getline(in, line)) {
    ++lineno;
    size_t c = line.find('#');
    if (c != std::string::npos) line = line.substr(0, c);
    c = line.find('!');
    if (c != std::string::npos) line = line.substr(0, c);
    if (trim(line).empty()) continue;
    size_t e = line.find('=');
    if (e == std::string::npos || e == 0 || trim(line.substr(e + 1)).empty())
      fail("line " + std::to_string(lineno) + ": expected name = value");
    if (line.find('=', e + 1) != std::string::npos) fail("line " + std::to_string(lineno) + ": more than one '='");
    std::string k = lower(trim(line.substr(0, e))), v = trim(line.substr(e + 1));
    if (!seen.insert(k).second) fail("duplicate parameter: " + k);
    if (k == "problem") { P.case_id = parse_problem(v); have_problem = true; continue; }
    kv.emplace_back(k, v);
  }
  if (!have_problem) fail("missing mandatory parameter: problem");
  apply_preset(P);
  for (auto &[k, v] : kv) {
    if (is_ic_key(k) && !ic_prefix_applies(k, P.case_id)) fail("parameter does not apply to the selected problem: " + k);
    if (k == "metric") {
      std::string t = lower(v);
      if (t == "minkowski") P.metric = MINK;
      else if (t == "eddington_finkelstein" || t == "ef") P.metric = EF;
      else if (t == "kerr_schild" || t == "ks") P.metric = KS;
      else fail("unknown metric: " + v);
    } else if (k == "geometry") {
      std::string t = lower(v);
      if (t == "cartesian") P.geom = CART;
      else if (t == "cylindrical") P.geom = CYL;
      else if (t == "spherical") P.geom = SPH;
      else if (t == "spheroidal") P.geom = SPHEROID;
      else fail("unknown geometry: " + v);
    } else if (k == "bh_mass") P.bh_mass = parse_real(v);
    else if (k == "spin") P.a_spin = parse_real(v);
    else if (k == "adiabatic_index") P.adb = parse_real(v);
    else if (k == "nx") P.nx = (int)parse_int(v);
    else if (k == "ny") P.ny = (int)parse_int(v);
    else if (k == "nz") P.nz = (int)parse_int(v);
    else if (k == "r_min") P.r_min = parse_real(v);
    else if (k == "r_max") P.r_max = parse_real(v);
    else if (k == "theta_min") P.y_min = parse_pi(v) * PI;
    else if (k == "theta_max") P.y_max = parse_pi(v) * PI;
    else if (k == "phi_min") P.z_min = parse_pi(v) * PI;
    else if (k == "phi_max") P.z_max = parse_pi(v) * PI;
    else if (k == "y_min") P.y_min = parse_real(v);
    else if (k == "y_max") P.y_max = parse_real(v);
    else if (k == "z_min") P.z_min = parse_real(v);
    else if (k == "z_max") P.z_max = parse_real(v);
    else if (k == "logarithmic_r") P.log_r = parse_bool(v);
    else if (k == "sod_interface") P.sod_if = parse_real(v);
    else if (k == "sod_density_left") P.sod_rl = parse_real(v);
    else if (k == "sod_density_right") P.sod_rr = parse_real(v);
    else if (k == "sod_pressure_left") P.sod_pl = parse_real(v);
    else if (k == "sod_pressure_right") P.sod_pr = parse_real(v);
    else if (k == "sod_velocity_left") P.sod_vl = parse_real(v);
    else if (k == "sod_velocity_right") P.sod_vr = parse_real(v);
    else if (k == "strong_interface") P.st_if = parse_real(v);
    else if (k == "strong_density_left") P.st_rl = parse_real(v);
    else if (k == "strong_density_right") P.st_rr = parse_real(v);
    else if (k == "strong_pressure_left") P.st_pl = parse_real(v);
    else if (k == "strong_pressure_right") P.st_pr = parse_real(v);
    else if (k == "shu_interface") P.shu_if = parse_real(v);
    else if (k == "shu_density_left") P.shu_rl = parse_real(v);
    else if (k == "shu_pressure_left") P.shu_pl = parse_real(v);
    else if (k == "shu_density_right") P.shu_rr = parse_real(v);
    else if (k == "shu_density_amplitude") P.shu_amp = parse_real(v);
    else if (k == "shu_wave_number") P.shu_k = parse_real(v);
    else if (k == "shu_pressure_right") P.shu_pr = parse_real(v);
    else if (k == "khi_half_width") P.khi_hw = parse_real(v);
    else if (k == "khi_density_inner") P.khi_ri = parse_real(v);
    else if (k == "khi_density_outer") P.khi_ro = parse_real(v);
    else if (k == "khi_velocity_inner") P.khi_vi = parse_real(v);
    else if (k == "khi_velocity_outer") P.khi_vo = parse_real(v);
    else if (k == "khi_pressure") P.khi_p = parse_real(v);
    else if (k == "khi_perturbation_amplitude") P.khi_pa = parse_real(v);
    else if (k == "khi_perturbation_wave_number") P.khi_pk = parse_real(v);
    else if (k == "khi_perturbation_width") P.khi_pw = parse_real(v);
    else if (k == "jet_ambient_density") P.jet_ar = parse_real(v);
    else if (k == "jet_ambient_pressure") P.jet_ap = parse_real(v);
    else if (k == "jet_ambient_velocity") P.jet_av = parse_real(v);
    else if (k == "jet_nozzle_radius") P.jet_nr = parse_real(v);
    else if (k == "jet_nozzle_length") P.jet_nl = parse_real(v);
    else if (k == "jet_density") P.jet_r = parse_real(v);
    else if (k == "jet_pressure") P.jet_p = parse_real(v);
    else if (k == "jet_velocity") P.jet_v = parse_real(v);
    else if (k == "convergence_density") P.cv_rho = parse_real(v);
    else if (k == "convergence_amplitude") P.cv_amp = parse_real(v);
    else if (k == "convergence_velocity") P.cv_v = parse_real(v);
    else if (k == "convergence_pressure") P.cv_p = parse_real(v);
    else if (k == "convergence_wave_number") P.cv_k = parse_pi(v);
    else if (k == "michel_critical_radius") P.mi_rc = parse_real(v);
    else if (k == "michel_critical_density") P.mi_rhoc = parse_real(v);
    else if (k == "dust_accretion_constant") P.dust_c = parse_real(v);
    else if (k == "offaxis_radial_center") P.oa_rc = parse_real(v);
    else if (k == "offaxis_phi_center") P.oa_phic = parse_pi(v) * PI;
    else if (k == "offaxis_width") P.oa_w = parse_real(v);
    else if (k == "offaxis_background_density") P.oa_bd = parse_real(v);
    else if (k == "offaxis_background_pressure") P.oa_bp = parse_real(v);
    else if (k == "offaxis_density_amplitude") P.oa_da = parse_real(v);
    else if (k == "offaxis_pressure_amplitude") P.oa_pa = parse_real(v);
    else if (k == "fm_inner_radius") P.fm_rin = parse_real(v);
    else if (k == "fm_pressure_max_radius") P.fm_rmax = parse_real(v);
    else if (k == "fm_polytropic_constant") P.fm_k = parse_real(v);
    else if (k == "reconstruction") {
      std::string t = lower(v);
      if (t == "godunov") P.rec = 1; else if (t == "tvd") P.rec = 2; else if (t == "weno3") P.rec = 3;
      else if (t == "mp5") P.rec = 4; else if (t == "weno5") P.rec = 5;
      else fail("reconstruction must be godunov, tvd, weno3, mp5 or weno5");
    } else if (k == "riemann_solver") {
      std::string t = lower(v);
      if (t == "hlle") P.rs = 1; else if (t == "hllc") P.rs = 2; else fail("riemann_solver must be hlle or hllc");
    } else if (k == "tvd_limiter") {
      std::string t = lower(v);
      if (t == "minmod") P.lim = 1; else if (t == "superbee") P.lim = 2; else if (t == "mc") P.lim = 3;
      else fail("tvd_limiter must be minmod, superbee or mc");
    } else if (k == "shock_sensor") P.shock_sensor = parse_bool(v);
    else if (k == "final_time") P.final_time = parse_real(v);
    else if (k == "cfl") P.cfl = parse_real(v);
    else if (k == "perturbation") {
      std::string t = lower(v);
      if (t == "none") P.pert_type = 0; else if (t == "pressure_noise") P.pert_type = 1;
      else if (t == "density_noise") P.pert_type = 2; else if (t == "density_mode") P.pert_type = 3;
      else fail("perturbation must be none, pressure_noise, density_noise or density_mode");
      P.apply_pert = P.pert_type != 0;
    } else if (k == "perturbation_seed") P.pert_seed = parse_int(v);
    else if (k == "perturbation_time") P.pert_time = parse_real(v);
    else if (k == "perturbation_amplitude") P.pert_amp = parse_real(v);
    else if (k == "perturbation_mode") P.pert_mode = parse_real(v);
    else if (k == "save_interval" || k == "checkpoint_interval" || k == "output_prefix" ||
             k == "output_folder" || k == "vtk_mapping" || k == "extract_gw" || k == "extract_mdot" ||
             k == "ppi_diagnostics" || k == "diagnostic_stride" || k == "extraction_stride" ||
             k == "mass_monitor_stride") {
      // output controls of the Fortran driver: accepted, no effect on the hot path
    } else fail("unknown parameter: " + k);
  }
}

bool is_polar(const Params &P) { return P.geom == SPH || P.geom == SPHEROID; }

// parameters.f90:359-600 (the checks that matter to the hot path and the initial data)
void validate(Params &P) {
  if (P.nx < 1 || P.ny < 1 || P.nz < 1) fail("nx, ny and nz must be positive");
  if (P.nx < 2) fail("nx must be at least 2 (the x-face metric cache exists only for nx > 1)");
  if (P.r_max <= P.r_min) fail("r_max must be larger than r_min");
  if (P.log_r && !is_polar(P)) fail("a logarithmic radial grid requires spherical or spheroidal geometry");
  if (is_polar(P) && P.r_min <= 0.0) fail("spherical and spheroidal geometries require r_min > 0");
  if (P.adb <= 1.0) fail("adiabatic_index must be larger than 1");
  if (P.bh_mass < 0.0) fail("bh_mass cannot be negative");
  if (P.final_time < 0.0 || P.cfl <= 0.0) fail("final_time >= 0 and cfl > 0 are required");
  if (P.pert_seed < 0 || P.pert_time < 0.0 || P.pert_amp < 0.0 || P.pert_amp >= 1.0)
    fail("invalid perturbation controls");
  if (P.metric == KS && P.geom == SPH) P.geom = SPHEROID;  // parameters.f90:428-431
  if (P.metric == MINK) {
    if (std::fabs(P.a_spin) > 0.0 || std::fabs(P.bh_mass) > 0.0) fail("Minkowski requires spin = 0 and bh_mass = 0");
    if (P.geom == SPHEROID) fail("Minkowski requires cartesian, cylindrical or spherical geometry");
  } else if (P.metric == EF) {
    if (std::fabs(P.a_spin) > 0.0) fail("Eddington-Finkelstein requires spin = 0");
    if (P.bh_mass <= 0.0 || P.geom != SPH) fail("Eddington-Finkelstein requires bh_mass > 0 and spherical geometry");
  } else {
    if (P.bh_mass <= 0.0 || P.geom != SPHEROID) fail("Kerr-Schild requires bh_mass > 0 and spheroidal geometry");
    if (std::fabs(P.a_spin) > P.bh_mass + 64.0 * EPS * std::fmax(1.0, P.bh_mass)) fail("Kerr-Schild requires |spin| <= bh_mass");
  }
  if (is_polar(P)) {
    if (P.y_min < 0.0 || P.y_max > PI || P.y_max <= P.y_min) fail("0 <= theta_min < theta_max <= 1 (units of pi) required");
    if (P.z_max <= P.z_min || P.z_max - P.z_min > 2.0 * PI + 64.0 * EPS * PI) fail("the azimuthal interval must be in (0, 2 pi]");
  } else if (P.y_max <= P.y_min || P.z_max <= P.z_min) fail("coordinate limits must increase");
  const double at = 128.0 * EPS * PI;
  switch (P.case_id) {
  case 1:
    if (P.sod_if <= P.r_min || P.sod_if >= P.r_max || std::fmin(P.sod_rl, P.sod_rr) <= 0.0 ||
        std::fmin(P.sod_pl, P.sod_pr) <= 0.0 || std::fabs(P.sod_vl) >= 1.0 || std::fabs(P.sod_vr) >= 1.0)
      fail("invalid Sod parameters");
    break;
  case 7:
    if (P.bh_mass <= 0.0 || P.mi_rc <= 1.5 * P.bh_mass || P.mi_rhoc <= 0.0) fail("invalid Michel parameters");
    break;
  case 8:
    if (P.bh_mass <= 0.0 || P.dust_c >= 0.0) fail("invalid dust parameters");
    break;
  case 10: case 11: case 12:
    if (P.bh_mass <= 0.0 || P.fm_rin <= 0.0 || P.fm_rmax <= P.fm_rin || P.fm_k <= 0.0) fail("invalid Fishbone-Moncrief parameters");
    if (P.case_id == 10 && (P.ny != 1 || std::fabs(0.5 * (P.y_min + P.y_max) - 0.5 * PI) > at))
      fail("fishbone_equatorial requires ny=1 and the polar cell centred on theta=pi/2");
    if (P.case_id == 11 && (P.ny <= 1 || P.nz != 1 || std::fabs(P.y_min) > at || std::fabs(P.y_max - PI) > at))
      fail("fishbone_sagittal requires ny>1, nz=1 and theta=[0,1] in units of pi");
    if (P.case_id == 12 && (P.ny <= 1 || P.nz <= 1 || (P.nz % 2) != 0 || std::fabs(P.y_min) > at ||
                            std::fabs(P.y_max - PI) > at || std::fabs((P.z_max - P.z_min) - 2.0 * PI) > at))
      fail("fishbone_3d requires ny,nz>1, nz even, theta=[0,1] and a phi length of 2 [pi]");
    break;
  default:
    break;
  }
  // initialization.f90:452-457 and :23-79
  P.g1 = P.adb / (P.adb - 1.0);
  P.rho_floor = 1.0e-10;
  P.p_floor = P.rho_floor * 1.0e-3;
  P.nghost = (P.rec == 1) ? 1 : (P.rec == 2 || P.rec == 3) ? 2 : 3;
}

// conditions.f90:249-278
void dust_state(const Params &P, double coord, double *s) {
  double r = coord, jac = 1.0;
  if (P.log_r) { r = std::exp(coord); jac = r; }
  if (r <= 0.0 || P.bh_mass <= 0.0 || P.dust_c >= 0.0) fail("invalid stationary dust-accretion parameters");
  double ff = std::sqrt(2.0 * P.bh_mass / r);
  for (int v = 0; v < 5; ++v) s[v] = 0.0;
  s[0] = -P.dust_c / (sq(r) * ff);
  s[1] = P.p_floor;
  s[2] = -1.0 / (std::sqrt(1.0 + r / (2.0 * P.bh_mass)) * (1.0 + ff + 2.0 * P.bh_mass / r));
  s[2] = s[2] / jac;
}

// conditions.f90:575-582
void fm_components(const double alpha, const double *beta, const double *g, double &g_tt, double &g_tphi) {
  double mg[3];
  for (int i = 0; i < 3; ++i) {
    mg[i] = 0.0;
    for (int j = 0; j < 3; ++j) mg[i] += g[i + 3 * j] * beta[j];
  }
  double dp = 0.0;
  for (int i = 0; i < 3; ++i) dp += beta[i] * mg[i];
  g_tt = -sq(alpha) + dp;
  g_tphi = 0.0;
  for (int j = 0; j < 3; ++j) g_tphi += g[2 + 3 * j] * beta[j];
}

// conditions.f90:470-510
bool fm_prepare(const Params &P, double r_in, double r_max, double &l_ang, double &W_in) {
  l_ang = 0.0; W_in = 0.0;
  double M = P.bh_mass, a = P.a_spin;
  if (M <= 0.0 || r_in <= 0.0 || r_max <= r_in) return false;
  double sqMr = std::sqrt(M * r_max);
  double num = sqMr * (sq(r_max) - 2.0 * a * sqMr + sq(a));
  double den = sq(r_max) - 2.0 * M * r_max + a * sqMr;
  if (!std::isfinite(den) || std::fabs(den) <= DBL_MIN) return false;
  l_ang = num / den;
  if (!std::isfinite(l_ang)) return false;
  double coord_in = P.log_r ? std::log(r_in) : r_in;
  MetricOut m;
  eval_metric(P, coord_in, PI / 2.0, false, m);
  double g_tt, g_tphi;
  fm_components(m.alpha, m.beta, m.gamma, g_tt, g_tphi);
  double nut = sq(g_tphi) - g_tt * m.gamma[8];
  double dut = m.gamma[8] + 2.0 * l_ang * g_tphi + sq(l_ang) * g_tt;
  if (nut <= 0.0 || dut <= 0.0) return false;
  double ut_sq = nut / dut;
  if (!std::isfinite(ut_sq) || ut_sq <= 0.0) return false;
  W_in = 0.5 * std::log(ut_sq);
  return std::isfinite(W_in);
}

// conditions.f90:516-572
bool fm_state(const Params &P, double r, double r_in, double K, double l_ang, double W_in, double alpha,
              const double *beta, const double *g, double *pc) {
  for (int v = 0; v < 5; ++v) pc[v] = 0.0;
  pc[0] = P.rho_floor; pc[1] = P.p_floor;
  if (r < r_in || K <= 0.0 || alpha <= 0.0) return false;
  double g_tt, g_tphi;
  fm_components(alpha, beta, g, g_tt, g_tphi);
  double nut = sq(g_tphi) - g_tt * g[8];
  double dut = g[8] + 2.0 * l_ang * g_tphi + sq(l_ang) * g_tt;
  if (nut <= 0.0 || dut <= 0.0) return false;
  double ut_sq = nut / dut;
  if (!std::isfinite(ut_sq) || ut_sq <= 0.0) return false;
  double W_r = 0.5 * std::log(ut_sq);
  double enthalpy = std::exp(W_in - W_r);
  if (!std::isfinite(enthalpy) || enthalpy <= 1.0) return false;
  double density = std::pow((enthalpy - 1.0) * (P.adb - 1.0) / (K * P.adb), 1.0 / (P.adb - 1.0));
  double pressure = K * std::pow(density, P.adb);
  if (!std::isfinite(density) || !std::isfinite(pressure) || density <= P.rho_floor || pressure <= P.p_floor) return false;
  double od = g[8] + l_ang * g_tphi;
  if (!std::isfinite(od) || std::fabs(od) <= DBL_MIN) return false;
  double Omega = -(g_tphi + l_ang * g_tt) / od;
  if (!std::isfinite(Omega)) return false;
  pc[0] = density; pc[1] = pressure;
  pc[2] = beta[0] / alpha; pc[3] = beta[1] / alpha; pc[4] = (Omega + beta[2]) / alpha;
  for (int v = 0; v < 5; ++v)
    if (!std::isfinite(pc[v])) {
      for (int w = 0; w < 5; ++w) pc[w] = 0.0;
      pc[0] = P.rho_floor; pc[1] = P.p_floor;
      return false;
    }
  return true;
}

void build_metric_cache(grhd2_problem &pb);
void set_initial_conditions(grhd2_problem &pb);

void build(grhd2_problem &pb) {
  Params &P = pb.P;
  const int nx = P.nx, ny = P.ny, nz = P.nz, g = P.nghost;
  // allocate_and_grid, initialization.f90:84-215
  pb.x_min = P.log_r ? std::log(P.r_min) : P.r_min;
  pb.x_max = P.log_r ? std::log(P.r_max) : P.r_max;
  pb.dx = (pb.x_max - pb.x_min) / (double)std::max(1, nx);
  pb.dy = (P.y_max - P.y_min) / (double)std::max(1, ny);
  pb.dz = (P.z_max - P.z_min) / (double)std::max(1, nz);
  pb.x.assign(nx + 2 * g + 1, 0.0); pb.y.assign(ny + 2 * g + 1, 0.0); pb.z.assign(nz + 2 * g + 1, 0.0);
  pb.x_face.assign(nx + 1, 0.0); pb.y_face.assign(ny + 1, 0.0); pb.z_face.assign(nz + 1, 0.0);
  for (int i = 0; i <= nx; ++i) pb.x_face[i] = pb.x_min + (double)i * pb.dx;
  for (int i = -g; i <= nx + g; ++i) pb.X(i) = pb.x_min + ((double)i - 0.5) * pb.dx;
  for (int j = 0; j <= ny; ++j) pb.y_face[j] = P.y_min + (double)j * pb.dy;
  for (int j = -g; j <= ny + g; ++j) pb.Y(j) = P.y_min + ((double)j - 0.5) * pb.dy;
  for (int k = 0; k <= nz; ++k) pb.z_face[k] = P.z_min + (double)k * pb.dz;
  for (int k = -g; k <= nz + g; ++k) pb.Z(k) = P.z_min + ((double)k - 0.5) * pb.dz;

  // precalculate_metric_cache, initialization.f90:265-391 (k = 1 slice)
  if (pb.metric_cache) build_metric_cache(pb);
  set_initial_conditions(pb);
}

void build_metric_cache(grhd2_problem &pb) {
  const Params &P = pb.P;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const size_t nc = (size_t)nx * ny;
  pb.alpha_c.assign(nc, 0); pb.beta_c.assign(3 * nc, 0); pb.gamma_c.assign(9 * nc, 0);
  pb.gamma_inv_c.assign(9 * nc, 0); pb.gmunu_c.assign(16 * nc, 0); pb.sqg_c.assign(nc, 0);
  pb.chris_c.assign(64 * nc, 0); pb.dg_c.assign(48 * nc, 0); pb.dlna_c.assign(4 * nc, 0);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      size_t c = (size_t)(i - 1) + (size_t)nx * (j - 1);
      MetricOut m;
      eval_metric(P, pb.X(i), pb.Y(j), true, m);
      eval_chris_dg(P, pb.X(i), pb.Y(j), &pb.chris_c[64 * c], &pb.dg_c[48 * c]);
      pb.alpha_c[c] = m.alpha;
      for (int d = 0; d < 3; ++d) pb.beta_c[3 * c + d] = m.beta[d];
      for (int q = 0; q < 9; ++q) pb.gamma_c[9 * c + q] = m.gamma[q];
      for (int q = 0; q < 16; ++q) pb.gmunu_c[16 * c + q] = m.gmunu[q];
      for (int ii = 1; ii <= 3; ++ii)
        for (int jj = 1; jj <= 3; ++jj)
          pb.gamma_inv_c[9 * c + (ii - 1) + 3 * (jj - 1)] =
              m.gmunu[ii + 4 * jj] + (m.beta[ii - 1] * m.beta[jj - 1]) / sq(m.alpha);
      pb.sqg_c[c] = std::sqrt(m.det);
      for (int q = 0; q < 4; ++q) pb.dlna_c[4 * c + q] = m.dlna[q];
    }
  auto fill_face = [&](std::vector<double> &A, std::vector<double> &B, std::vector<double> &G,
                       std::vector<double> &S, size_t n) {
    A.assign(n, 0); B.assign(3 * n, 0); G.assign(9 * n, 0); S.assign(n, 0);
  };
  if (nx > 1) {
    size_t n = (size_t)(nx + 1) * ny;
    fill_face(pb.a_fx, pb.b_fx, pb.g_fx, pb.s_fx, n);
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx + 1; ++i) {
        size_t f = (size_t)(i - 1) + (size_t)(nx + 1) * (j - 1);
        MetricOut m;
        eval_metric(P, pb.x_face[i - 1], pb.Y(j), false, m);
        pb.a_fx[f] = m.alpha;
        for (int d = 0; d < 3; ++d) pb.b_fx[3 * f + d] = m.beta[d];
        for (int q = 0; q < 9; ++q) pb.g_fx[9 * f + q] = m.gamma[q];
        pb.s_fx[f] = std::sqrt(m.det);
      }
  }
  if (ny > 1) {
    size_t n = (size_t)nx * (ny + 1);
    fill_face(pb.a_fy, pb.b_fy, pb.g_fy, pb.s_fy, n);
    for (int j = 1; j <= ny + 1; ++j)
      for (int i = 1; i <= nx; ++i) {
        size_t f = (size_t)(i - 1) + (size_t)nx * (j - 1);
        MetricOut m;
        eval_metric(P, pb.X(i), pb.y_face[j - 1], false, m);
        pb.a_fy[f] = m.alpha;
        for (int d = 0; d < 3; ++d) pb.b_fy[3 * f + d] = m.beta[d];
        for (int q = 0; q < 9; ++q) pb.g_fy[9 * f + q] = m.gamma[q];
        if (is_polar(P) && std::fabs(std::sin(pb.y_face[j - 1])) <= 64.0 * EPS) pb.s_fy[f] = 0.0;
        else pb.s_fy[f] = std::sqrt(m.det);
      }
  }
  if (nz > 1) {
    size_t n = (size_t)nx * ny;
    fill_face(pb.a_fz, pb.b_fz, pb.g_fz, pb.s_fz, n);
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        size_t f = (size_t)(i - 1) + (size_t)nx * (j - 1);
        MetricOut m;
        eval_metric(P, pb.X(i), pb.Y(j), false, m);
        pb.a_fz[f] = m.alpha;
        for (int d = 0; d < 3; ++d) pb.b_fz[3 * f + d] = m.beta[d];
        for (int q = 0; q < 9; ++q) pb.g_fz[9 * f + q] = m.gamma[q];
        pb.s_fz[f] = std::sqrt(m.det);
      }
  }
}

void set_initial_conditions(grhd2_problem &pb) {
  const Params &P = pb.P;
  const int nx = P.nx, ny = P.ny, nz = P.nz, g = P.nghost;
  // set_initial_conditions, conditions.f90:26-214
  pb.p.assign((size_t)5 * (nx + 2 * g + 1) * (ny + 2 * g + 1) * (nz + 2 * g + 1), 0.0);
  auto Pv = [&](int v, int i, int j, int k) -> double & { return pb.p[pb.pidx(v, i, j, k)]; };
  auto all_jk = [&](int i, int v, double val) {
    for (int k = -g; k <= nz + g; ++k)
      for (int j = -g; j <= ny + g; ++j) Pv(v, i, j, k) = val;
  };
  switch (P.case_id) {
  case 1:
    for (int i = -g; i <= nx + g; ++i) {
      bool left = pb.X(i) < P.sod_if;
      all_jk(i, 0, left ? P.sod_rl : P.sod_rr);
      all_jk(i, 1, left ? P.sod_pl : P.sod_pr);
      if (P.sod_vl != 0.0 || P.sod_vr != 0.0) all_jk(i, 2, left ? P.sod_vl : P.sod_vr);
    }
    break;
  case 2:
    for (int i = -g; i <= nx + g; ++i) {
      bool left = pb.X(i) < P.st_if;
      all_jk(i, 0, left ? P.st_rl : P.st_rr);
      all_jk(i, 1, left ? P.st_pl : P.st_pr);
    }
    break;
  case 3:
    for (int i = -g; i <= nx + g; ++i) {
      if (pb.X(i) < P.shu_if) { all_jk(i, 0, P.shu_rl); all_jk(i, 1, P.shu_pl); }
      else { all_jk(i, 0, P.shu_rr + P.shu_amp * std::sin(P.shu_k * pb.X(i))); all_jk(i, 1, P.shu_pr); }
    }
    break;
  case 4:
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          double xp = pb.X(i), zp = pb.Z(k);
          if (std::fabs(zp) < P.khi_hw) { Pv(0, i, j, k) = P.khi_ri; Pv(2, i, j, k) = P.khi_vi; }
          else { Pv(0, i, j, k) = P.khi_ro; Pv(2, i, j, k) = P.khi_vo; }
          Pv(1, i, j, k) = P.khi_p;
          Pv(3, i, j, k) = 0.0;
          double dist = std::fabs(std::fabs(zp) - P.khi_hw);
          double env = std::exp(-0.5 * sq(dist / P.khi_pw));
          Pv(4, i, j, k) = P.khi_pa * std::sin(P.khi_pk * PI * xp) * env;
        }
    break;
  case 5:
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          Pv(0, i, j, k) = P.jet_ar; Pv(1, i, j, k) = P.jet_ap; Pv(4, i, j, k) = P.jet_av;
          if (pb.X(i) <= P.jet_nr && pb.Z(k) <= P.jet_nl) {
            Pv(0, i, j, k) = P.jet_r; Pv(1, i, j, k) = P.jet_p; Pv(4, i, j, k) = P.jet_v;
          }
        }
    break;
  case 6: {
    double sarg = 0.5 * P.cv_k * PI * pb.dx;
    double sf = (std::fabs(sarg) > EPS) ? std::sin(sarg) / sarg : 1.0;
    for (int i = 1; i <= nx; ++i) all_jk(i, 0, P.cv_rho + P.cv_amp * sf * std::sin(P.cv_k * PI * pb.X(i)));
    for (int i = -g; i <= nx + g; ++i) { all_jk(i, 2, P.cv_v); all_jk(i, 1, P.cv_p); }
    break;
  }
  case 7: {
    // setup_michel_accretion_initial on p(:, 1:nx+g, 1:ny, 1:nz), conditions.f90:284-410
    const double M = P.bh_mass, rc = P.mi_rc, rhoc = P.mi_rhoc, adb = P.adb, g1 = P.g1;
    double u_c = -std::sqrt(M / (2.0 * rc));
    double ut_c = std::sqrt(1.0 - 2.0 * M / rc + u_c * u_c);
    double Vc2 = sq(u_c / ut_c);
    double pres = (Vc2 * rhoc) / (adb - Vc2 * g1);
    double K_poly = pres / std::pow(rhoc, adb);
    double h_spec = 1.0 + g1 * pres / rhoc;
    double C1 = sq(rc) * rhoc * u_c;
    double C2 = sq(rc) * rhoc * h_spec * u_c * ut_c;
    const double eps_tol = 1.0e-6;
    for (int i = 1; i <= nx + g; ++i) {
      double r = P.log_r ? std::exp(pb.X(i)) : pb.X(i);
      double ur = -std::sqrt(2.0 * M / r), rho;
      for (int it = 1; it <= 40; ++it) {
        double ut = std::sqrt(1.0 - 2.0 * M / r + sq(ur));
        rho = C1 / (sq(r) * ur);
        double pr = K_poly * std::pow(rho, adb);
        double hs = 1.0 + g1 * pr / rho;
        double f = hs * ut - C2 / C1;
        double urp = ur + eps_tol, urm = ur - eps_tol;
        double utp = std::sqrt(1.0 - 2.0 * M / r + sq(urp));
        double rp = C1 / (sq(r) * urp);
        double pp = K_poly * std::pow(rp, adb);
        double hp = 1.0 + g1 * pp / rp;
        double fp = hp * utp - C2 / C1;
        double utm = std::sqrt(1.0 - 2.0 * M / r + sq(urm));
        double rm = C1 / (sq(r) * urm);
        double pm = K_poly * std::pow(rm, adb);
        double hm = 1.0 + g1 * pm / rm;
        double fm = hm * utm - C2 / C1;
        double df = (fp - fm) / (2.0 * eps_tol);
        ur = ur - f / df;
        if (std::fabs(f) < 1.0e-12) break;
      }
      rho = C1 / (sq(r) * ur);
      double pr = K_poly * std::pow(rho, adb);
      for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j) {
          MetricOut m;
          eval_metric(P, pb.X(i), pb.Y(j), false, m);
          double ux = P.log_r ? ur / r : ur;
          double g_tt = -sq(m.alpha);
          for (int ii = 0; ii < 3; ++ii)
            for (int jj = 0; jj < 3; ++jj) g_tt = g_tt + m.gamma[ii + 3 * jj] * m.beta[ii] * m.beta[jj];
          double g_tx = 0.0;
          for (int jj = 0; jj < 3; ++jj) g_tx = g_tx + m.gamma[0 + 3 * jj] * m.beta[jj];
          double A = g_tt, B = 2.0 * g_tx * ux, C = m.gamma[0] * sq(ux) + 1.0;
          double ut_contra = (-B - std::sqrt(sq(B) - 4.0 * A * C)) / (2.0 * A);
          double W = m.alpha * ut_contra;
          Pv(0, i, j, k) = rho;
          Pv(1, i, j, k) = pr;
          Pv(2, i, j, k) = ux / W + m.beta[0] / m.alpha;
          Pv(3, i, j, k) = m.beta[1] / m.alpha;
          Pv(4, i, j, k) = m.beta[2] / m.alpha;
        }
    }
    // cache_michel_injector, conditions.f90:229-246
    pb.michel_injector.assign((size_t)5 * g * ny * nz, 0.0);
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= g; ++i)
          for (int v = 0; v < 5; ++v)
            pb.michel_injector[v + 5 * ((i - 1) + (size_t)g * ((j - 1) + (size_t)ny * (k - 1)))] = Pv(v, nx + i, j, k);
    break;
  }
  case 8: {
    double s[5];
    for (int i = 1; i <= nx + g; ++i) {
      dust_state(P, pb.X(i), s);
      for (int k = -g; k <= nz + g; ++k)
        for (int j = -g; j <= ny + g; ++j)
          for (int v = 0; v < 5; ++v) Pv(v, i, j, k) = s[v];
    }
    for (int i = -g; i <= 0; ++i)
      for (int k = -g; k <= nz + g; ++k)
        for (int j = -g; j <= ny + g; ++j)
          for (int v = 0; v < 5; ++v) Pv(v, i, j, k) = Pv(v, 1, j, k);
    pb.dust_outer.assign((size_t)5 * g, 0.0);
    for (int gg = 1; gg <= g; ++gg) dust_state(P, pb.X(nx + gg), &pb.dust_outer[5 * (gg - 1)]);
    break;
  }
  case 9:
    for (int k = -g; k <= nz + g; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = -g; i <= nx + g; ++i) {
          double r = P.log_r ? std::exp(pb.X(i)) : pb.X(i);
          double d2 = sq(r) + sq(P.oa_rc) - 2.0 * P.oa_rc * r * std::cos(pb.Z(k) - P.oa_phic);
          double ex = -d2 / sq(P.oa_w);
          double gp = (ex < -40.0) ? 0.0 : std::exp(ex);
          Pv(0, i, j, k) = P.oa_bd + P.oa_da * gp;
          Pv(1, i, j, k) = P.oa_bp + P.oa_pa * gp;
        }
    break;
  case 10: case 11: case 12: {
    double r_in = P.fm_rin * P.bh_mass, r_mx = P.fm_rmax * P.bh_mass;
    if (!fm_prepare(P, r_in, r_mx, pb.fm_l, pb.fm_w_in)) fail("invalid Fishbone-Moncrief model parameters");
    // the centre metric from the cache (conditions.f90:450-452), or evaluated here when the
    // cache is built on the device (the same function at the same point: the same values)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double r = P.log_r ? std::exp(pb.X(i)) : pb.X(i);
        const size_t c = (size_t)(i - 1) + (size_t)nx * (j - 1);
        MetricOut m;
        if (!pb.metric_cache) eval_metric(P, pb.X(i), pb.Y(j), false, m);
        const double alpha = pb.metric_cache ? pb.alpha_c[c] : m.alpha;
        const double *beta = pb.metric_cache ? &pb.beta_c[3 * c] : m.beta;
        const double *gamma = pb.metric_cache ? &pb.gamma_c[9 * c] : m.gamma;
        double pc[5];
        fm_state(P, r, r_in, P.fm_k, pb.fm_l, pb.fm_w_in, alpha, beta, gamma, pc);
        for (int k = 1; k <= nz; ++k)
          for (int v = 0; v < 5; ++v) Pv(v, i, j, k) = pc[v];
      }
    break;
  }
  }
}

// SplitMix64 (Steele, Lea, Flood 2014), mapped to [0,1) with 53 bits
struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

// ------------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------------
extern "C" {

int grhd2_problem_create(const char *par_text, grhd2_problem **out, char *err, int errlen) {
  return grhd2_problem_create_ex(par_text, 0u, out, err, errlen);
}

int grhd2_problem_create_ex(const char *par_text, uint32_t flags, grhd2_problem **out, char *err, int errlen) {
  if (!par_text || !out) return GRHD2_ERR_ARG;
  *out = nullptr;
  if (flags & ~(uint32_t)GRHD2_PROBLEM_NO_METRIC_CACHE) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "unknown problem flags 0x%x", (unsigned)flags);
    return GRHD2_ERR_ARG;
  }
  grhd2_problem *pb = new (std::nothrow) grhd2_problem();
  if (!pb) return GRHD2_ERR_NOMEM;
  pb->metric_cache = !(flags & GRHD2_PROBLEM_NO_METRIC_CACHE);
  try {
    read_par(par_text, pb->P);
    validate(pb->P);
    build(*pb);
  } catch (const ParError &e) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", e.msg.c_str());
    delete pb;
    return GRHD2_ERR_ARG;
  } catch (const std::bad_alloc &) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "out of host memory");
    delete pb;
    return GRHD2_ERR_NOMEM;
  }
  *out = pb;
  return GRHD2_OK;
}

void grhd2_problem_destroy(grhd2_problem *pb) { delete pb; }

int grhd2_problem_config(const grhd2_problem *pb, int32_t precision_policy, grhd2_gpu_config *c) {
  if (!pb || !c) return GRHD2_ERR_ARG;
  const Params &P = pb->P;
  std::memset(c, 0, sizeof *c);
  c->nx = P.nx; c->ny = P.ny; c->nz = P.nz; c->nghost = P.nghost; c->neq = 5;
  c->rec_method = P.rec; c->tvd_limiter = P.lim; c->riemann = P.rs; c->shock_sensor = P.shock_sensor ? 1 : 0;
  c->metric_kind = P.metric; c->geom_kind = P.geom; c->use_log_r = P.log_r ? 1 : 0; c->case_id = P.case_id;
  c->precision_policy = precision_policy;
  c->dx = pb->dx; c->dy = pb->dy; c->dz = pb->dz; c->adb_idx = P.adb; c->g1 = P.g1; c->cfl = P.cfl;
  c->rho_floor = P.rho_floor; c->p_floor = P.p_floor; c->v_max = 1.0 - 1.0e-5;
  return GRHD2_OK;
}

int grhd2_problem_metric(const grhd2_problem *pb, grhd2_gpu_metric_view *mv) {
  if (!pb || !mv) return GRHD2_ERR_ARG;
  std::memset(mv, 0, sizeof *mv);
  if (!pb->metric_cache) {  // the face coordinates only
    mv->x_face = pb->x_face.data();
    mv->y_face = pb->y_face.data();
    return GRHD2_ERR_STATE;
  }
  mv->alpha_c = pb->alpha_c.data(); mv->beta_c = pb->beta_c.data(); mv->gamma_c = pb->gamma_c.data();
  mv->gamma_inv_c = pb->gamma_inv_c.data(); mv->gmunu_c = pb->gmunu_c.data(); mv->sqrt_gamma_c = pb->sqg_c.data();
  mv->chris_c = pb->chris_c.data(); mv->dg_c = pb->dg_c.data(); mv->dlna_c = pb->dlna_c.data();
  if (pb->P.nx > 1) { mv->alpha_f_x = pb->a_fx.data(); mv->beta_f_x = pb->b_fx.data(); mv->gamma_f_x = pb->g_fx.data(); mv->sqrt_gamma_f_x = pb->s_fx.data(); }
  if (pb->P.ny > 1) { mv->alpha_f_y = pb->a_fy.data(); mv->beta_f_y = pb->b_fy.data(); mv->gamma_f_y = pb->g_fy.data(); mv->sqrt_gamma_f_y = pb->s_fy.data(); }
  if (pb->P.nz > 1) { mv->alpha_f_z = pb->a_fz.data(); mv->beta_f_z = pb->b_fz.data(); mv->gamma_f_z = pb->g_fz.data(); mv->sqrt_gamma_f_z = pb->s_fz.data(); }
  mv->x_face = pb->x_face.data();
  mv->y_face = pb->y_face.data();
  return GRHD2_OK;
}

int grhd2_problem_bc(const grhd2_problem *pb, grhd2_gpu_bc_view *bv) {
  if (!pb || !bv) return GRHD2_ERR_ARG;
  std::memset(bv, 0, sizeof *bv);
  bv->michel_injector = pb->michel_injector.empty() ? nullptr : pb->michel_injector.data();
  bv->dust_outer = pb->dust_outer.empty() ? nullptr : pb->dust_outer.data();
  bv->x_c = pb->x.data();
  const Params &P = pb->P;
  bv->jet[0] = P.jet_ar; bv->jet[1] = P.jet_ap; bv->jet[2] = P.jet_av; bv->jet[3] = P.jet_nr;
  bv->jet[4] = P.jet_r; bv->jet[5] = P.jet_p; bv->jet[6] = P.jet_v;
  return GRHD2_OK;
}

int grhd2_problem_info_get(const grhd2_problem *pb, grhd2_problem_info *info) {
  if (!pb || !info) return GRHD2_ERR_ARG;
  const Params &P = pb->P;
  std::memset(info, 0, sizeof *info);
  info->case_id = P.case_id; info->nx = P.nx; info->ny = P.ny; info->nz = P.nz; info->nghost = P.nghost;
  info->perturbation_type = P.apply_pert ? P.pert_type : 0;
  info->perturbation_seed = P.pert_seed;
  info->final_time = P.final_time; info->cfl = P.cfl; info->perturbation_time = P.pert_time;
  info->perturbation_amplitude = P.pert_amp; info->perturbation_mode = P.pert_mode;
  info->x_min = pb->x_min; info->x_max = pb->x_max; info->y_min = P.y_min; info->y_max = P.y_max;
  info->z_min = P.z_min; info->z_max = P.z_max; info->bh_mass = P.bh_mass; info->a_spin = P.a_spin;
  info->fm_l = pb->fm_l; info->fm_w_in = pb->fm_w_in;
  return GRHD2_OK;
}

const double *grhd2_problem_prims(const grhd2_problem *pb) { return pb ? pb->p.data() : nullptr; }
int64_t grhd2_problem_prim_size(const grhd2_problem *pb) { return pb ? (int64_t)pb->p.size() : 0; }
int64_t grhd2_problem_cons_size(const grhd2_problem *pb) {
  return pb ? (int64_t)5 * pb->P.nx * pb->P.ny * pb->P.nz : 0;
}
const double *grhd2_problem_x(const grhd2_problem *pb) { return pb ? pb->x.data() : nullptr; }
const double *grhd2_problem_y(const grhd2_problem *pb) { return pb ? pb->y.data() : nullptr; }
const double *grhd2_problem_z(const grhd2_problem *pb) { return pb ? pb->z.data() : nullptr; }

// conditions.f90:603-768 (grhd2.f90:194-204 dispatch)
int grhd2_problem_perturb(const grhd2_problem *pb, double *p) {
  if (!pb || !p) return GRHD2_ERR_ARG;
  const Params &P = pb->P;
  if (!P.apply_pert || P.pert_type == 0) return GRHD2_OK;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  if (P.pert_amp < 0.0 || P.pert_amp >= 1.0) return GRHD2_ERR_ARG;
  if (P.pert_type == 3 && P.pert_mode < 1.0) return GRHD2_ERR_ARG;
  double rho_max = -HUGE_VAL;
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) rho_max = std::fmax(rho_max, p[pb->pidx(0, i, j, k)]);
  SplitMix64 rng{(uint64_t)P.pert_seed};
  for (int k = 1; k <= nz; ++k) {
    double phi = pb->z[k + P.nghost];
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double &rho = p[pb->pidx(0, i, j, k)], &pr = p[pb->pidx(1, i, j, k)];
        if (!(rho > 0.05 * rho_max)) continue;
        if (P.pert_type == 1) {
          double rv = 2.0 * rng.uniform() - 1.0;
          pr = pr * (1.0 + P.pert_amp * rv);
        } else if (P.pert_type == 2) {
          double rv = 2.0 * rng.uniform() - 1.0;
          double f = 1.0 + P.pert_amp * rv;
          rho = rho * f;
          pr = pr * std::pow(f, P.adb);
        } else {
          double f = 1.0 + P.pert_amp * std::cos(P.pert_mode * phi);
          rho = rho * f;
          pr = pr * std::pow(f, P.adb);
        }
      }
  }
  return GRHD2_OK;
}

int grhd2_problem_eval_metric(const grhd2_problem *pb, double x, double y, double *alpha, double *beta,
                              double *gamma, double *gmunu, double *det, double *dlnalpha, double *chris,
                              double *dg) {
  if (!pb) return GRHD2_ERR_ARG;
  MetricOut m;
  eval_metric(pb->P, x, y, true, m);
  if (alpha) *alpha = m.alpha;
  if (beta) std::memcpy(beta, m.beta, sizeof m.beta);
  if (gamma) std::memcpy(gamma, m.gamma, sizeof m.gamma);
  if (gmunu) std::memcpy(gmunu, m.gmunu, sizeof m.gmunu);
  if (det) *det = m.det;
  if (dlnalpha) std::memcpy(dlnalpha, m.dlna, sizeof m.dlna);
  if (chris || dg) {
    double ch[64], d[48];
    eval_chris_dg(pb->P, x, y, ch, d);
    if (chris) std::memcpy(chris, ch, sizeof ch);
    if (dg) std::memcpy(dg, d, sizeof d);
  }
  return GRHD2_OK;
}

namespace {
// module globals of a metric probe (metric_type, geom_type, use_log_r, bh_mass, a_spin, ny):
// set directly, without the .par checks, as the reference's set-up tests set them
bool probe_params(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass, double a_spin,
                  int32_t ny, Params &P) {
  if (metric_kind < MINK || metric_kind > KS || geom_kind < CART || geom_kind > SPHEROID || ny < 1) return false;
  P.metric = metric_kind;
  P.geom = geom_kind;
  P.log_r = use_log_r != 0;
  P.bh_mass = bh_mass;
  P.a_spin = a_spin;
  P.ny = ny;
  return true;
}
}  // namespace

int grhd2_host_metric_at(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass, double a_spin,
                         int32_t ny, double x, double y, double *alpha, double *beta, double *gamma, double *gmunu,
                         double *det, double *dlnalpha, double *chris, double *dg) {
  Params P;
  if (!probe_params(metric_kind, geom_kind, use_log_r, bh_mass, a_spin, ny, P)) return GRHD2_ERR_ARG;
  MetricOut m;
  eval_metric(P, x, y, true, m);
  if (alpha) *alpha = m.alpha;
  if (beta) std::memcpy(beta, m.beta, sizeof m.beta);
  if (gamma) std::memcpy(gamma, m.gamma, sizeof m.gamma);
  if (gmunu) std::memcpy(gmunu, m.gmunu, sizeof m.gmunu);
  if (det) *det = m.det;
  if (dlnalpha) std::memcpy(dlnalpha, m.dlna, sizeof m.dlna);
  if (chris || dg) {
    double ch[64], d[48];
    eval_chris_dg(P, x, y, ch, d);
    if (chris) std::memcpy(chris, ch, sizeof ch);
    if (dg) std::memcpy(dg, d, sizeof d);
  }
  return GRHD2_OK;
}

int grhd2_host_dust_state(int32_t use_log_r, double bh_mass, double dust_accretion_constant, double p_floor,
                          double x, double *state) {
  if (!state) return GRHD2_ERR_ARG;
  Params P;
  P.metric = EF;
  P.geom = SPH;
  P.log_r = use_log_r != 0;
  P.bh_mass = bh_mass;
  P.dust_c = dust_accretion_constant;
  P.p_floor = p_floor;
  try {
    dust_state(P, x, state);
  } catch (const ParError &) {
    return GRHD2_ERR_ARG;
  }
  return GRHD2_OK;
}

int grhd2_host_fm_prepare(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass, double a_spin,
                          double r_in, double r_max, double *l_ang, double *w_in, int32_t *ok) {
  Params P;
  if (!probe_params(metric_kind, geom_kind, use_log_r, bh_mass, a_spin, 1, P) || !l_ang || !w_in || !ok)
    return GRHD2_ERR_ARG;
  *ok = fm_prepare(P, r_in, r_max, *l_ang, *w_in) ? 1 : 0;
  return GRHD2_OK;
}

int grhd2_host_fm_state(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass, double a_spin,
                        double adiabatic_index, double rho_floor, double p_floor, double radius, double theta,
                        double r_in, double K, double l_ang, double w_in, double *state, int32_t *inside) {
  Params P;
  if (!probe_params(metric_kind, geom_kind, use_log_r, bh_mass, a_spin, 1, P) || !state || !inside)
    return GRHD2_ERR_ARG;
  P.adb = adiabatic_index;
  P.rho_floor = rho_floor;
  P.p_floor = p_floor;
  MetricOut m;
  eval_metric(P, P.log_r ? std::log(radius) : radius, theta, false, m);
  *inside = fm_state(P, radius, r_in, K, l_ang, w_in, m.alpha, m.beta, m.gamma, state) ? 1 : 0;
  return GRHD2_OK;
}

}  // extern "C"
