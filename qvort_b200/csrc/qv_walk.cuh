// qv_walk.cuh -- device helpers shared by the Barnes-Hut walks (single system
// and batched forest): the reference's FP64 distance and opening test
// (src/tree.f90:350-365, 394), the compensated FP32 accumulator and the
// stack entry of the mixed-precision walk.
#pragma once
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

// Stack entry: the child's FP32 header, fetched when the child is pushed so
// that popping it costs a shared-memory read instead of a dependent global load.
struct __align__(16) StkEnt {
  WNode32 h;
  int node;
  unsigned mask;
  int pad[2];
};

