// qv_host.cpp -- host-side pieces of the Qvort driver that feed the path:
// the run.in reader (read_run_file, src/cdata.f90:420-807, the keys this path
// uses), the var-file reader (read_var_file, src/initial.f90:463-496) and
// writer (printf, src/output.f90:116-143), and the ring set-ups used by the
// benchmark configurations (setup_single_loop / setup_leap_frog,
// src/initial_loop.f90:11-38, 206-245).
#include <cctype>
#include <cstdint>
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

// ------------------------------------------------------------ restart file
// data_dump / data_restore (src/output.f90:272-285, src/initial.f90:501-538):
// ./data/var.dat, an unformatted sequential file -- each write is one record
// framed by its byte length as a 4-byte integer before and after (gfortran's
// record markers) -- holding pcount, recon_count, itime, t, the whole f(:)
// array, quasi_pcount (and g), part_count (and p).  An element of f is the
// reference's type qvort (src/cdata.f90:20-39) under -fdefault-real-8, laid
// out in declaration order with natural alignment, 464 bytes:
namespace {
enum : size_t {
  F_X = 0, F_X_INTERP = 24, F_U = 48, F_U1 = 72, F_U2 = 96, F_U3 = 120, F_ACC = 144,
  F_U_SUP = 168, F_U_MF = 192, F_U_S_LI = 216, F_U_S_BS = 240, F_GHOSTI = 264, F_GHOSTB = 288,
  F_GHOSTII = 312, F_GHOSTBB = 336, F_F_MF = 360, F_STRETCH = 384, F_CURV = 392,
  F_INFRONT = 400, F_BEHIND = 404, F_CLOSEST = 408, F_CLOSESTD = 416, F_CLOSESTD_LOOP = 424,
  F_PINNEDI = 432, F_PINNEDB = 436, F_DELTA = 440, F_T_RECON = 448, F_SIZE = 464
};
// one record of gfortran's sequential unformatted layout; records of 2 GiB
// and more would be split into subrecords, which this writer does not do
bool put_rec(std::FILE *f, const void *p, size_t bytes) {
  if (bytes > 0x7fffffffu - 8) return false;
  const int32_t m = (int32_t)bytes;
  return std::fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || std::fwrite(p, bytes, 1, f) == 1) &&
         std::fwrite(&m, 4, 1, f) == 1;
}
bool get_rec(std::FILE *f, std::vector<unsigned char> &buf) {
  int32_t m = 0, m2 = 0;
  if (std::fread(&m, 4, 1, f) != 1 || m < 0) return false;
  buf.resize((size_t)m);
  if (m > 0 && std::fread(buf.data(), (size_t)m, 1, f) != 1) return false;
  return std::fread(&m2, 4, 1, f) == 1 && m2 == m;
}
template <class T> bool get_scalar(std::FILE *f, T *out) {
  std::vector<unsigned char> b;
  if (!get_rec(f, b) || b.size() != sizeof(T)) return false;
  std::memcpy(out, b.data(), sizeof(T));
  return true;
}
}  // namespace

extern "C" int qv_write_restart_file(const char *path, int n, int recon_count, int itime,
                                     double t, const qv_restart *s) {
  if (!path || !s || n < 0 || (n > 0 && (!s->x || !s->infront || !s->behind))) return QV_ERR_ARG;
  if ((size_t)n * F_SIZE > 0x7fffffffu - 8) return QV_ERR_ARG;
  std::vector<unsigned char> fa((size_t)n * F_SIZE, 0);
  auto put3 = [&](size_t off, const double *a, int i) {
    if (a) std::memcpy(&fa[(size_t)i * F_SIZE + off], a + 3 * (size_t)i, 24);
  };
  for (int i = 0; i < n; i++) {
    unsigned char *e = &fa[(size_t)i * F_SIZE];
    put3(F_X, s->x, i);
    put3(F_U, s->u, i);
    put3(F_U1, s->u1, i);
    put3(F_U2, s->u2, i);
    put3(F_U3, s->u3, i);
    put3(F_U_SUP, s->u, i);  // superfluid velocity = u with no normal fluid
    put3(F_U_S_LI, s->u_li, i);
    put3(F_U_S_BS, s->u_bs, i);
    put3(F_GHOSTI, s->gi, i);
    put3(F_GHOSTB, s->gb, i);
    put3(F_GHOSTII, s->gii, i);
    put3(F_GHOSTBB, s->gbb, i);
    std::memcpy(e + F_INFRONT, s->infront + i, 4);
    std::memcpy(e + F_BEHIND, s->behind + i, 4);
    if (s->closest) std::memcpy(e + F_CLOSEST, s->closest + i, 4);
    if (s->closestd) std::memcpy(e + F_CLOSESTD, s->closestd + i, 8);
    const double one = 1.;  // the per-point resolution factor (delta_adapt off)
    std::memcpy(e + F_DELTA, &one, 8);
  }
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return QV_ERR_ARG;
  const int zero = 0;
  bool ok = put_rec(f, &n, 4) && put_rec(f, &recon_count, 4) && put_rec(f, &itime, 4) &&
            put_rec(f, &t, 8) && put_rec(f, fa.data(), fa.size()) &&
            put_rec(f, &zero, 4) /* quasi_pcount */ && put_rec(f, &zero, 4) /* part_count */;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? QV_OK : QV_ERR_ARG;
}

extern "C" int qv_read_restart_file(const char *path, int cap, int *n, int *recon_count,
                                    int *itime, double *t, qv_restart *s) {
  if (!path || !n) return QV_ERR_ARG;
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return QV_ERR_ARG;
  int pc = 0, rc_ = 0, it = 0;
  double tt = 0.;
  std::vector<unsigned char> fa;
  bool ok = get_scalar(f, &pc) && get_scalar(f, &rc_) && get_scalar(f, &it) &&
            get_scalar(f, &tt) && pc >= 0;
  if (ok && s && s->x) ok = get_rec(f, fa) && fa.size() == (size_t)pc * F_SIZE;
  std::fclose(f);
  if (!ok) return QV_ERR_ARG;
  *n = pc;
  if (recon_count) *recon_count = rc_;
  if (itime) *itime = it;
  if (t) *t = tt;
  if (!s || !s->x) return QV_OK;
  if (pc > cap) return QV_ERR_ARG;
  auto get3 = [&](size_t off, double *a, int i) {
    if (a) std::memcpy(a + 3 * (size_t)i, &fa[(size_t)i * F_SIZE + off], 24);
  };
  for (int i = 0; i < pc; i++) {
    const unsigned char *e = &fa[(size_t)i * F_SIZE];
    get3(F_X, s->x, i);
    get3(F_U, s->u, i);
    get3(F_U1, s->u1, i);
    get3(F_U2, s->u2, i);
    get3(F_U3, s->u3, i);
    get3(F_U_S_LI, s->u_li, i);
    get3(F_U_S_BS, s->u_bs, i);
    get3(F_GHOSTI, s->gi, i);
    get3(F_GHOSTB, s->gb, i);
    get3(F_GHOSTII, s->gii, i);
    get3(F_GHOSTBB, s->gbb, i);
    if (s->infront) std::memcpy(s->infront + i, e + F_INFRONT, 4);
    if (s->behind) std::memcpy(s->behind + i, e + F_BEHIND, 4);
    if (s->closest) std::memcpy(s->closest + i, e + F_CLOSEST, 4);
    if (s->closestd) std::memcpy(s->closestd + i, e + F_CLOSESTD, 8);
  }
  return QV_OK;
}
