// qv_lia.cuh -- the local (LIA) term of calc_velocity, written once for any
// scalar type T (double for the velocity, a dual number for its derivatives).
//
// get_deriv_1 / get_deriv_2 (src/derivatives.f90:11-75): second or fourth
// order non-uniform finite differences on the ghost stencil; the LIA arm
// (src/timestep.f90:196-217) and the local part of the BS/Tree arms
// (src/timestep.f90:221-225, 270-274).  For T = double and FMA contraction
// off, every operation is rounded in the reference's order.
#pragma once
#include "qv_internal.cuh"

template <typename T>
__device__ __forceinline__ T lia_dist(const T *a, const T *b) {
  T d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

template <typename T>
__device__ __forceinline__ void lia_derivs(int order, const T *x, const T *gi, const T *gb,
                                           const T *gii, const T *gbb, T *s1, T *s2) {
  T disti = lia_dist(x, gi), distb = lia_dist(x, gb);
  if (order != 4) {
    T den1 = 2. * distb * disti;
    T q1 = disti * (disti + distb), q2 = disti * distb, q3 = distb * (disti + distb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      s1[c] = (distb * gi[c] + (disti - distb) * x[c] - disti * gb[c]) / den1;
      s2[c] = 2. * (gi[c] / q1 - x[c] / q2 + gb[c] / q3);
    }
    return;
  }
  T dii = lia_dist(gii, gi), dbb = lia_dist(gbb, gb);
  T di2 = disti * disti, db2 = distb * distb;
  T dA = dbb * (dbb + distb) * (dbb + distb + disti) * (dbb + distb + disti + dii);
  T dB = dbb * distb * (distb + disti) * (distb + disti + dii);
  T dD = disti * dii * (distb + disti) * (dbb + distb + disti);
  T dE = dii * (disti + dii) * (distb + disti + dii) * (dbb + distb + disti + dii);
  T A = (distb * di2 + distb * disti * dii) / dA;
  T B = (-dbb * di2 - distb * di2 - dbb * disti * dii - distb * disti * dii) / dB;
  T D = (dbb * distb * disti + db2 * disti + dbb * distb * dii + db2 * dii) / dD;
  T E = (-disti * db2 - dbb * distb * disti) / dE;
  T C = -(A + B + D + E);
  T A2 = 2. * (-2. * distb * disti + di2 - distb * dii + disti * dii) / dA;
  T B2 = 2. * (2. * dbb * disti + 2. * distb * disti - di2 + dbb * dii + distb * dii - disti * dii) / dB;
  T D2 = 2. * (-dbb * distb - db2 + dbb * disti + 2. * distb * disti + dbb * dii + 2. * distb * dii) / dD;
  T E2 = 2. * (dbb * distb + db2 - dbb * disti - 2. * distb * disti) / dE;
  T C2 = -(A2 + B2 + D2 + E2);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    s1[c] = A * gbb[c] + B * gb[c] + C * x[c] + D * gi[c] + E * gii[c];
    s2[c] = A2 * gbb[c] + B2 * gb[c] + C2 * x[c] + D2 * gi[c] + E2 * gii[c];
  }
}

// The local velocity beta * s' x s'' for velocity LIA/BS/Tree (zero for Off).
template <typename T>
__device__ __forceinline__ void lia_term(int velocity, int order, int fixed_beta, double quant_circ,
                                         double corea, const T *X, const T *GI, const T *GB,
                                         const T *GII, const T *GBB, T *out) {
  out[0] = out[1] = out[2] = T(0.);
  if (velocity == QV_VEL_OFF) return;
  T s1[3], s2[3];
  lia_derivs(order, X, GI, GB, GII, GBB, s1, s2);
  T beta;
  if (velocity == QV_VEL_LIA) {
    if (fixed_beta) {
      beta = T(1.3E-3);
    } else {
      T curv = sqrt(s2[0] * s2[0] + s2[1] * s2[1] + s2[2] * s2[2]);
      curv = curv < QV_DEPS ? T(QV_DEPS) : 1. / curv;
      beta = (quant_circ / (4. * QV_PI)) * log(curv / corea);
    }
  } else {
    beta = (quant_circ / (4. * QV_PI)) * log((1.21 / corea) * sqrt(lia_dist(X, GI) * lia_dist(X, GB)));
  }
  out[0] = beta * (s1[1] * s2[2] - s1[2] * s2[1]);
  out[1] = beta * (s1[2] * s2[0] - s1[0] * s2[2]);
  out[2] = beta * (s1[0] * s2[1] - s1[1] * s2[0]);
}

// ------------------------------------------------------------- dual numbers
// Forward-mode derivative carrier: value and one directional derivative.
struct Dual {
  double v, d;
  __device__ __forceinline__ Dual() : v(0.), d(0.) {}
  __device__ __forceinline__ Dual(double a) : v(a), d(0.) {}
  __device__ __forceinline__ Dual(double a, double b) : v(a), d(b) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(double a, Dual b) { return Dual(a) / b; }
__device__ __forceinline__ bool operator<(Dual a, double b) { return a.v < b; }
__device__ __forceinline__ Dual sqrt(Dual a) {
  double s = ::sqrt(a.v);
  return Dual(s, s > 0. ? a.d / (2. * s) : 0.);
}
__device__ __forceinline__ Dual log(Dual a) { return Dual(::log(a.v), a.d / a.v); }
