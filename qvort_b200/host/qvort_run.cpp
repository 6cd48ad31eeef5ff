// qvort_run -- a C++ stand-in for the reference's driver (src/run.f90) that
// runs the velocity-and-timestep path of this library from a run.in:
//   read_run_file -> initial condition (var_file, single_loop, leap-frog) ->
//   do itime = 1, nsteps: qv_steps between outputs (ghostp, construct_tree, pmotion /
//   pmotion_RK3, pinsert, candidate search, precon unless switch_off_recon,
//   premove, ghostp, boundary wrap), t = t + dt;
//   every `shots` steps: data/var%04d.log and a one-line summary, STOP file.
//
//   usage: qvort_run [run.in]        (run from the run directory)
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "qv.h"

static bool exists(const char *p) {
  struct stat st;
  return stat(p, &st) == 0;
}

int main(int argc, char **argv) {
  const char *runin = argc > 1 ? argv[1] : "run.in";
  qv_run r;
  int rc = qv_read_run_file(runin, &r);
  if (rc) {
    std::fprintf(stderr, "qvort_run: cannot read %s (status %d)\n", runin, rc);
    return 2;
  }
  std::vector<double> x;
  std::vector<int> inf, beh;
  int n = 0;
  double t = 0.;
  if (std::strcmp(r.initf, "var_file") == 0) {
    char name[64];
    std::snprintf(name, sizeof name, "./var%04d.log", r.readin_var_file);
    if ((rc = qv_read_var_file(name, 0, &n, &t, nullptr, nullptr, nullptr))) {
      std::fprintf(stderr, "qvort_run: cannot read %s\n", name);
      return 2;
    }
    x.resize(3 * (size_t)n);
    inf.resize(n);
    beh.resize(n);
    rc = qv_read_var_file(name, n, &n, &t, x.data(), inf.data(), beh.data());
    t = 0.;  // the reference discards the stored time (dummy_t)
  } else {
    n = r.pcount;
    x.resize(3 * (size_t)n);
    inf.resize(n);
    beh.resize(n);
    rc = qv_setup_loops(r.initf, n, r.p.delta, x.data(), inf.data(), beh.data());
  }
  if (rc) {
    std::fprintf(stderr, "qvort_run: initf '%s' is outside this path (status %d)\n", r.initf, rc);
    return 2;
  }
  // the line operations of src/run.f90:59-72 (they need a resolution delta)
  r.p.line_ops = r.p.delta > 0 ? (r.switch_off_recon ? 1 : 2) : 0;
  qv_ctx *ctx = nullptr;
  if ((rc = qv_create(&r.p, nullptr, &ctx))) {
    std::fprintf(stderr, "qvort_run: qv_create failed (status %d)\n", rc);
    return 2;
  }
  if ((rc = qv_set_points(ctx, n, x.data(), inf.data(), beh.data()))) {
    std::fprintf(stderr, "qvort_run: %s\n", qv_last_error(ctx));
    return 2;
  }
  mkdir("data", 0755);
  std::vector<double> u(3 * (size_t)n);
  int shot = 0;
  for (int first = 1; first <= r.nsteps;) {
    // the steps up to the next output in one call (qv_steps replays a CUDA
    // graph of a step when the options allow it)
    int itime = r.shots > 0 ? ((first + r.shots - 1) / r.shots) * r.shots : r.nsteps;
    if (itime > r.nsteps) itime = r.nsteps;
    if ((rc = qv_steps(ctx, first, itime - first + 1))) {
      std::fprintf(stderr, "qvort_run: steps %d-%d: %s\n", first, itime, qv_last_error(ctx));
      qv_destroy(ctx);
      return 3;
    }
    for (int k = first; k <= itime; k++) t = t + r.p.dt;
    first = itime + 1;
    if (r.shots > 0 && itime % r.shots == 0) {
      // insertion can raise the slot count and every line operation relinks
      qv_point_count(ctx, &n);
      x.resize(3 * (size_t)n);
      u.resize(3 * (size_t)n);
      inf.resize(n);
      beh.resize(n);
      qv_get_points(ctx, x.data(), u.data());
      qv_get_links(ctx, inf.data(), beh.data());
      char name[64];
      std::snprintf(name, sizeof name, "./data/var%04d.log", ++shot);
      qv_write_var_file(name, n, t, x.data(), inf.data(), u.data());
      double umax = 0.;
      for (int i = 0; i < n; i++) {
        if (!inf[i]) continue;
        double s = u[3 * i] * u[3 * i] + u[3 * i + 1] * u[3 * i + 1] + u[3 * i + 2] * u[3 * i + 2];
        if (s > umax) umax = s;
      }
      std::printf("itime %d t %.6e pcount %d maxu %.6e\n", itime, t, n, umax > 0 ? std::sqrt(umax) : 0.);
      std::fflush(stdout);
      if (exists("./STOP")) {  // src/run.f90:149-155
        std::printf("Encountered stop file, ending simulation\n");
        break;
      }
    }
  }
  qv_destroy(ctx);
  return 0;
}
