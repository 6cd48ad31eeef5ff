// qv_host.cpp -- host-side pieces of the Qvort driver that feed the path:
// the run.in reader (read_run_file, src/cdata.f90:420-807, the keys this path
// uses), the var-file reader (read_var_file, src/initial.f90:463-496) and
// writer (printf, src/output.f90:116-143), and the ring set-ups used by the
// benchmark configurations (setup_single_loop / setup_leap_frog,
// src/initial_loop.f90:11-38, 206-245).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qv.h"

namespace {

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// First item of a Fortran list-directed record (blank, comma or slash ends it;
// quotes are stripped).
std::string first_item(const std::string &v) {
  std::string s = trim(v);
  if (!s.empty() && (s[0] == '\'' || s[0] == '"')) {
    char q = s[0];
    size_t e = s.find(q, 1);
    return s.substr(1, e == std::string::npos ? std::string::npos : e - 1);
  }
  size_t e = s.find_first_of(" \t,/");
  return s.substr(0, e);
}

bool read_real(const std::string &v, double *out) {
  std::string s = first_item(v);
  if (s.empty()) return false;
  for (char &ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';  // Fortran double exponent
  char *end = nullptr;
  double d = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0') return false;
  *out = d;
  return true;
}

bool read_int(const std::string &v, int *out) {
  std::string s = first_item(v);
  if (s.empty()) return false;
  char *end = nullptr;
  long k = std::strtol(s.c_str(), &end, 10);
  if (end == s.c_str() || *end != '\0') return false;
  *out = (int)k;
  return true;
}

// list-directed logical: optional '.', then T or F (case-insensitive)
bool read_logical(const std::string &v, int *out) {
  std::string s = first_item(v);
  size_t k = (!s.empty() && s[0] == '.') ? 1 : 0;
  if (k >= s.size()) return false;
  char ch = (char)std::toupper((unsigned char)s[k]);
  if (ch == 'T') { *out = 1; return true; }
  if (ch == 'F') { *out = 0; return true; }
  return false;
}

}  // namespace

extern "C" int qv_read_run_file(const char *path, qv_run *r) {
  if (!path || !r) return QV_ERR_ARG;
  std::memset(r, 0, sizeof(*r));
  qv_default_params(&r->p);
  r->p.precision = QV_PREC_MIXED;
  r->nsteps = 0;
  r->shots = 1;
  r->readin_var_file = 1;  // src/cdata.f90:237
  std::FILE *f = std::fopen(path, "r");
  if (!f) return QV_ERR_ARG;
  char line[1024];
  int rc = QV_OK;
  std::string velocity = "BS", boundary = "open", order = "second";
  while (std::fgets(line, sizeof line, f)) {
    std::string buf(line);
    while (!buf.empty() && (buf.back() == '\n' || buf.back() == '\r')) buf.pop_back();
    // the label is the text up to the first blank (src/cdata.f90:439-441)
    size_t pos = buf.find(' ');
    if (pos == std::string::npos) continue;
    std::string label = buf.substr(0, pos), val = buf.substr(pos + 1);
    bool ok = true;
    if (label == "nsteps") ok = read_int(val, &r->nsteps);
    else if (label == "shots") ok = read_int(val, &r->shots);
    else if (label == "recon_shots") ok = read_int(val, &r->p.recon_shots);
    else if (label == "pcount") ok = read_int(val, &r->pcount);
    else if (label == "dt") ok = read_real(val, &r->p.dt);
    else if (label == "delta") ok = read_real(val, &r->p.delta);
    else if (label == "quant_circ") ok = read_real(val, &r->p.quant_circ);
    else if (label == "corea") ok = read_real(val, &r->p.corea);
    else if (label == "box_size") ok = read_real(val, &r->p.box_size);
    else if (label == "tree_theta") ok = read_real(val, &r->p.tree_theta);
    else if (label == "tree_extra_correction") ok = read_logical(val, &r->p.tree_extra_correction);
    else if (label == "fixed_LIA_beta") ok = read_logical(val, &r->p.fixed_lia_beta);
    else if (label == "runge_kutta") ok = read_logical(val, &r->p.runge_kutta);
    else if (label == "switch_off_recon") ok = read_logical(val, &r->switch_off_recon);
    else if (label == "readin_var_file") ok = read_int(val, &r->readin_var_file);
    else if (label == "velocity") { velocity = first_item(val); ok = !velocity.empty(); }
    else if (label == "boundary") { boundary = first_item(val); ok = !boundary.empty(); }
    else if (label == "deriv_order") { order = first_item(val); ok = !order.empty(); }
    else if (label == "initf") {
      std::string s = first_item(val);
      std::snprintf(r->initf, sizeof r->initf, "%s", s.c_str());
      ok = !s.empty();
    } else if (label == "gpu_precision") {
      // a key of this path only; the reference parser ignores unknown labels
      std::string s = first_item(val);
      if (s == "fp64") r->p.precision = QV_PREC_FP64;
      else if (s == "mixed") r->p.precision = QV_PREC_MIXED;
      else ok = false;
    }
    // a value that fails to read ends the file, as iostat /= 0 ends the loop
    if (!ok) { rc = QV_ERR_ARG; break; }
  }
  std::fclose(f);
  if (velocity == "Off") r->p.velocity = QV_VEL_OFF;
  else if (velocity == "LIA") r->p.velocity = QV_VEL_LIA;
  else if (velocity == "BS") r->p.velocity = QV_VEL_BS;
  else if (velocity == "Tree") r->p.velocity = QV_VEL_TREE;
  else r->p.velocity = -1;
  if (boundary == "open") r->p.boundary = QV_BC_OPEN;
  else if (boundary == "periodic") r->p.boundary = QV_BC_PERIODIC;
  else if (boundary == "openx") r->p.boundary = QV_BC_OPENX;
  else if (boundary == "openxy") r->p.boundary = QV_BC_OPENXY;
  else r->p.boundary = -1;  // mirror, open-remove: outside this path
  r->p.deriv_order = order == "fourth" ? 4 : 2;
  return rc;
}

// Stream layout of src/output.f90:124-142 (and of read_var_file, which reads
// its first six records): t, pcount, x(1..n), y, z, infront, u(1..3),
// u_mf(1..3), curv, stretch, f_mf(1..3).
extern "C" int qv_read_var_file(const char *path, int cap, int *n, double *t, double *x,
                                int *infront, int *behind) {
  if (!path || !n) return QV_ERR_ARG;
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return QV_ERR_ARG;
  double tt = 0.;
  int pc = 0;
  if (std::fread(&tt, sizeof tt, 1, f) != 1 || std::fread(&pc, sizeof pc, 1, f) != 1 || pc < 0) {
    std::fclose(f);
    return QV_ERR_ARG;
  }
  *n = pc;
  if (t) *t = tt;
  if (!x || !infront) { std::fclose(f); return QV_OK; }  // size query
  if (pc > cap) { std::fclose(f); return QV_ERR_ARG; }
  std::vector<double> c(pc);
  for (int k = 0; k < 3; k++) {
    if (std::fread(c.data(), sizeof(double), pc, f) != (size_t)pc) { std::fclose(f); return QV_ERR_ARG; }
    for (int i = 0; i < pc; i++) x[3 * i + k] = c[i];
  }
  if (std::fread(infront, sizeof(int), pc, f) != (size_t)pc) { std::fclose(f); return QV_ERR_ARG; }
  std::fclose(f);
  if (behind) {
    // behind(i) = the first active j with infront(j) == i (src/initial.f90:484-495)
    std::vector<int> first(pc + 1, 0);
    for (int j = pc; j >= 1; j--)
      if (infront[j - 1] > 0 && infront[j - 1] <= pc) first[infront[j - 1]] = j;
    for (int i = 1; i <= pc; i++) behind[i - 1] = infront[i - 1] == 0 ? 0 : first[i];
  }
  return QV_OK;
}

extern "C" int qv_write_var_file(const char *path, int n, double t, const double *x,
                                 const int *infront, const double *u) {
  if (!path || n < 0 || (n > 0 && (!x || !infront))) return QV_ERR_ARG;
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return QV_ERR_ARG;
  std::vector<double> c(n);
  bool ok = std::fwrite(&t, sizeof t, 1, f) == 1 && std::fwrite(&n, sizeof n, 1, f) == 1;
  for (int k = 0; k < 3 && ok; k++) {
    for (int i = 0; i < n; i++) c[i] = x[3 * i + k];
    ok = std::fwrite(c.data(), sizeof(double), n, f) == (size_t)n;
  }
  ok = ok && std::fwrite(infront, sizeof(int), n, f) == (size_t)n;
  for (int k = 0; k < 3 && ok; k++) {
    for (int i = 0; i < n; i++) c[i] = u ? u[3 * i + k] : 0.;
    ok = std::fwrite(c.data(), sizeof(double), n, f) == (size_t)n;
  }
  // u_mf(3), curv, stretch, f_mf(3) are not computed by this path: zeros
  std::fill(c.begin(), c.end(), 0.);
  for (int k = 0; k < 8 && ok; k++) ok = std::fwrite(c.data(), sizeof(double), n, f) == (size_t)n;
  std::fclose(f);
  return ok ? QV_OK : QV_ERR_ARG;
}

extern "C" int qv_setup_loops(const char *initf, int pcount, double delta, double *x,
                              int *infront, int *behind) {
  if (!initf || pcount < 1 || !x || !infront || !behind) return QV_ERR_ARG;
  const double pi = 3.14159265358979324;
  if (std::strcmp(initf, "single_loop") == 0) {
    // setup_single_loop, src/initial_loop.f90:11-38
    double radius = (0.75 * pcount * delta) / (2 * pi);
    for (int i = 1; i <= pcount; i++) {
      x[3 * (i - 1)] = radius * std::sin(pi * (double)(2 * i - 1) / pcount);
      x[3 * (i - 1) + 1] = radius * std::cos(pi * (double)(2 * i - 1) / pcount);
      x[3 * (i - 1) + 2] = 0.;
      behind[i - 1] = i == 1 ? pcount : i - 1;
      infront[i - 1] = i == pcount ? 1 : i + 1;
    }
    return QV_OK;
  }
  if (std::strcmp(initf, "leap-frog") == 0) {
    // setup_leap_frog, src/initial_loop.f90:206-245
    if (pcount % 2 != 0) return QV_ERR_ARG;
    int h = pcount / 2;
    double radius = (0.75 * pcount * delta) / (4 * pi);
    for (int i = 1; i <= pcount; i++) {
      int k = i <= h ? i : i - h;
      x[3 * (i - 1)] = radius * std::sin(pi * (double)(2 * k - 1) / h);
      x[3 * (i - 1) + 1] = radius * std::cos(pi * (double)(2 * k - 1) / h);
      x[3 * (i - 1) + 2] = i <= h ? 0. : 2. * delta;
      int lo = i <= h ? 1 : h + 1, hi = i <= h ? h : pcount;
      behind[i - 1] = i == lo ? hi : i - 1;
      infront[i - 1] = i == hi ? lo : i + 1;
    }
    return QV_OK;
  }
  return QV_ERR_UNSUPPORTED;
}
