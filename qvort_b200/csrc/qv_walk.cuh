// qv_walk.cuh -- device helpers shared by the Barnes-Hut walks (single system
// and batched forest): the reference's FP64 distance and opening test
// (src/tree.f90:350-365, 394), the compensated FP32 accumulator and the
// stack entry of the mixed-precision walk.
#pragma once
#include "qv_f32x2.cuh"
#include "qv_internal.cuh"

__device__ __forceinline__ double shift_of(int m, double L) {
  return m == 0 ? 0. : (m > 0 ? L : -L);
}

// dist = |x_i - (cent + shift)| in the reference's operation order.
__device__ __forceinline__ double exact_dist(const double *xi, const WNode64 &h, const double *s) {
  double d0 = __dsub_rn(xi[0], __dadd_rn(h.cx, s[0]));
  double d1 = __dsub_rn(xi[1], __dadd_rn(h.cy, s[1]));
  double d2 = __dsub_rn(xi[2], __dadd_rn(h.cz, s[2]));
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
}

// theta test of src/tree.f90:354-365,394 on a non-leaf node; true = open.
__device__ __forceinline__ bool exact_open(double dist, const WNode64 &h, double theta_tree,
                                           int extra) {
  double th;
  if (extra) {
    double r = __dsub_rn(dist, h.geo);
    th = r > 0. ? __ddiv_rn(h.width, r) : __ddiv_rn(h.width, dist);
  } else {
    th = __ddiv_rn(h.width, dist);
  }
  return !(th < theta_tree);
}

// The root's opening test while its header holds the centroid estimate of
// k_root_est, whose distance from the exact (sequentially summed) centroid is
// at most delta.  Moving the centroid by delta moves dist and geo by at most
// delta each, so the test is decided for every centroid in that ball when
// width/(dist - geo) stays on one side of tree_theta over dist - geo +- 2 delta
// (and width/dist over dist +- delta where dist <= geo is possible); the margin
// also carries a relative 1e-14 for the rounding of the test itself.  A decided
// test returns its answer.  An undecided one returns "open" (the lane walks the
// image) and sets `unc`; the fix-up after the walk takes the exact decision and
// drops the image's sum if the root was in fact far.  delta = 0: the header
// holds the exact centroid and this is the reference's test.
__device__ __forceinline__ bool root_open(const double *xi, const WNode64 &r, const double *s,
                                          double theta, int extra, double delta, bool &unc) {
  const double dist = exact_dist(xi, r, s);
  const bool open = exact_open(dist, r, theta, extra);
  if (!(delta > 0.)) return open;
  const double m = delta + 1e-14 * (dist + r.geo + r.width);
  bool cfar, copen;
  if (extra) {
    const double rl = dist - r.geo - 2. * m, rh = dist - r.geo + 2. * m;
    cfar = rl > 0. && r.width < theta * rl;
    copen = (rh <= 0. || r.width >= theta * rh) && (rl > 0. || r.width >= theta * (dist + m));
  } else {
    cfar = r.width < theta * (dist - m);
    copen = r.width >= theta * (dist + m);
  }
  if (cfar) return false;
  if (copen) return true;
  unc = true;
  return true;
}

__device__ __forceinline__ void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

struct Kahan3w {
  float s[3], c[3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < 3; k++) s[k] = c[k] = 0.f;
  }
  __device__ __forceinline__ void add(float a0, float a1, float a2) {
    float a[3] = {a0, a1, a2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float y = __fsub_rn(a[k], c[k]);
      float t = __fadd_rn(s[k], y);
      c[k] = __fsub_rn(__fsub_rn(t, s[k]), y);
      s[k] = t;
    }
  }
  __device__ __forceinline__ double get(int k) const { return (double)s[k] - (double)c[k]; }
};

// Kahan3w for two targets at once: (s, c) hold target a in .x and target b
// in .y.  add() applies the scalar update's operations to both halves and
// keeps the new values only where the half's flag is set, so each half goes
// through exactly the sequence of updates a Kahan3w of its own would.
struct Kahan3x2 {
  float2 s[3], c[3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < 3; k++) s[k] = c[k] = make_float2(0.f, 0.f);
  }
  __device__ __forceinline__ void add(float2 a0, float2 a1, float2 a2, bool fx, bool fy) {
    const float2 a[3] = {a0, a1, a2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float2 y = sub2(a[k], c[k]);
      const float2 t = add2(s[k], y);
      const float2 cn = sub2(sub2(t, s[k]), y);
      s[k].x = fx ? t.x : s[k].x;
      s[k].y = fy ? t.y : s[k].y;
      c[k].x = fx ? cn.x : c[k].x;
      c[k].y = fy ? cn.y : c[k].y;
    }
  }
  // half H alone (a leaf pair of one of the two targets)
  template <int H>
  __device__ __forceinline__ void add1(float a0, float a1, float a2) {
    const float a[3] = {a0, a1, a2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float &sk = H ? s[k].y : s[k].x;
      float &ck = H ? c[k].y : c[k].x;
      const float y = __fsub_rn(a[k], ck);
      const float t = __fadd_rn(sk, y);
      ck = __fsub_rn(__fsub_rn(t, sk), y);
      sk = t;
    }
  }
  __device__ __forceinline__ double get(int h, int k) const {
    return (double)pick(s[k], h) - (double)pick(c[k], h);
  }
};

// Stack entry: the child's FP32 header, fetched when the child is pushed so
// that popping it costs a shared-memory read instead of a dependent global load,
// and the lane masks of the targets that opened the parent (mask: the warp's
// first 32 targets; mask2: the second 32 where a lane carries two).
struct __align__(16) StkEnt {
  WNode32 h;
  int node;
  unsigned mask, mask2;
  int pad;
};

