// qv_ab.cuh -- the Adams-Bashforth ladder of pmotion (src/timestep.f90:48-71)
// and the periodic wrap of enforce_periodic (src/periodic.f90:188-214), one
// point at a time, shared by the update kernel and by the differentiable step
// (forward and adjoint) so that both take the same operations.
#pragma once
#include "qv_internal.cuh"

// Rung of the ladder from exact-zero tests of the stored history: 1 = Euler
// (u1 = 0), 2 = AB2 (u2 = 0), 3 = AB3 (u3 = 0), 4 = AB4.
__device__ __forceinline__ int ab_rung(const double *U1, const double *U2, const double *U3) {
  const bool z1 = fabs(U1[0]) == 0 && fabs(U1[1]) == 0 && fabs(U1[2]) == 0;
  const bool z2 = fabs(U2[0]) == 0 && fabs(U2[1]) == 0 && fabs(U2[2]) == 0;
  const bool z3 = fabs(U3[0]) == 0 && fabs(U3[1]) == 0 && fabs(U3[2]) == 0;
  return z1 ? 1 : z2 ? 2 : z3 ? 3 : 4;
}

// One component of the update in the reference's operation order, one
// rounding per operation (round-to-nearest intrinsics: no contraction).
__device__ __forceinline__ double ab_update(int rung, double dt, double X, double U, double U1,
                                            double U2, double U3) {
  const double three_twos = 3. / 2., one_half = 1. / 2., c23_12 = 23. / 12., c4_3 = 4. / 3.,
               c5_12 = 5. / 12.;
  double r;
  if (rung == 1) {
    r = __dadd_rn(X, __dmul_rn(dt, U));
  } else if (rung == 2) {
    r = __dadd_rn(X, __dmul_rn(__dmul_rn(three_twos, dt), U));
    r = __dsub_rn(r, __dmul_rn(__dmul_rn(one_half, dt), U1));
  } else if (rung == 3) {
    r = __dadd_rn(X, __dmul_rn(__dmul_rn(c23_12, dt), U));
    r = __dsub_rn(r, __dmul_rn(__dmul_rn(c4_3, dt), U1));
    r = __dadd_rn(r, __dmul_rn(__dmul_rn(c5_12, dt), U2));
  } else {
    double s = __dsub_rn(__dmul_rn(55., U), __dmul_rn(59., U1));
    s = __dadd_rn(s, __dmul_rn(37., U2));
    s = __dsub_rn(s, __dmul_rn(9., U3));
    r = __dadd_rn(X, __ddiv_rn(__dmul_rn(dt, s), 24.));
  }
  return r;
}

// d x_new / d (u, u1, u2, u3) of a rung (the update is linear in them, and
// d x_new / d x = 1).
__device__ __forceinline__ void ab_coef(int rung, double dt, double *c) {
  c[0] = c[1] = c[2] = c[3] = 0.;
  if (rung == 1) {
    c[0] = dt;
  } else if (rung == 2) {
    c[0] = 1.5 * dt; c[1] = -0.5 * dt;
  } else if (rung == 3) {
    c[0] = (23. / 12.) * dt; c[1] = -(4. / 3.) * dt; c[2] = (5. / 12.) * dt;
  } else {
    c[0] = 55. * dt / 24.; c[1] = -59. * dt / 24.; c[2] = 37. * dt / 24.; c[3] = -9. * dt / 24.;
  }
}

// enforce_periodic on one coordinate: x > L/2 -> x - L, x < -L/2 -> x + L.
__device__ __forceinline__ double wrap_coord(double v, double L) {
  const double h = L / 2.;
  if (v > h) return v - L;
  if (v < (-h)) return v + L;
  return v;
}
