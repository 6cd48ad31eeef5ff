// qv_adjoint.cu -- hand-written derivatives of the velocity path.
//
// qv_velocity_vjp: x_bar = J^T u_bar for u = calc_velocity(x) (src/timestep.f90:
// 180-309) through every piece of it:
//   * the local LIA term (forward-mode dual numbers over its 9- or 15-value
//     ghost stencil, the same templated formula as the velocity),
//   * the direct sum (hand-derived gradients of the straight-segment term,
//     a target pass and a source pass, no atomics),
//   * or the Barnes-Hut walk with the topology of the last build frozen
//     (hand-derived leaf and monopole+dipole gradients; the gradients that
//     belong to a source cell are reduced over the warp and added to a per-node
//     adjoint of (cent, circ, Cij), which a last kernel distributes to the
//     cell's points through the moment definitions of src/tree.f90:146-179),
//   * and the ghost gather (ghosti_i = x_infront(i) etc., src/periodic.f90:23-31),
//     whose adjoint is a gather over behind/infront.
// qv_energy_grad: energy_info (src/diagnostic.f90:259-280) and its gradients
// with respect to x and u.
// qv_field_velocity: biot_savart_general(_shift) (src/timestep.f90:516-563) at
// arbitrary points and its exact gradient, in place of the central
// differences of velocity_quasip (src/hamiltonian.f90:65-89).
//
// Segment term (leaf form of src/tree.f90:380-390, the same function as the
// direct form of src/timestep.f90:472-479):
//   u = f R1 x R2,  f = (a+b)/P,  P = a b (a b + d),  a=|R1|, b=|R2|, d=R1.R2
// For an upstream g:  Q = g.(R1 x R2),
//   dQ/dR1 = R2 x g,  dQ/dR2 = g x R1,
//   df/da = (P - (a+b) b(2ab+d))/P^2,  df/db = (P - (a+b) a(2ab+d))/P^2,
//   df/dd = -(a+b) ab / P^2,
//   grad_R1 (f Q) = Q (df/da R1/a + df/dd R2) + f (R2 x g),
//   grad_R2 (f Q) = Q (df/db R2/b + df/dd R1) + f (g x R1).
// Far cell (monopole + dipole, restated as in the walk):
//   u = r3 (circ x v - w) + 3 r5 v x z,  z = C^T v,  r3 = |v|^-3, r5 = |v|^-5,
//   grad_v (g.u) = -3 r5 (g.a) v + r3 g x circ - 15 r7 (g.b) v + 3 r5 (z x g + C (g x v)),
//   with a = circ x v - w, b = v x z;  d/dcirc = r3 v x g;  d/dw = -r3 g;
//   d/dz = 3 r5 g x v  ->  d/dC(p,l) = v_p (d/dz)_l.
#include <algorithm>
#include <vector>

#include "qv_internal.cuh"
#include "qv_ab.cuh"
#include "qv_lia.cuh"

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// ------------------------------------------------------------- segment term
__device__ __forceinline__ void seg_grad(const double *R1, const double *R2, const double *g,
                                         double *gR1, double *gR2) {
  double a = sqrt(R1[0] * R1[0] + R1[1] * R1[1] + R1[2] * R1[2]);
  double b = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
  double d = R1[0] * R2[0] + R1[1] * R2[1] + R1[2] * R2[2];
  double ab = a * b;
  double P = ab * (ab + d);
  double f = (a + b) / P;
  double cr[3] = {R1[1] * R2[2] - R1[2] * R2[1], R1[2] * R2[0] - R1[0] * R2[2],
                  R1[0] * R2[1] - R1[1] * R2[0]};
  double Q = g[0] * cr[0] + g[1] * cr[1] + g[2] * cr[2];
  double P2 = P * P, t = 2. * ab + d;
  double dfa = (P - (a + b) * b * t) / P2, dfb = (P - (a + b) * a * t) / P2;
  double dfd = -(a + b) * ab / P2;
  double r2g[3] = {R2[1] * g[2] - R2[2] * g[1], R2[2] * g[0] - R2[0] * g[2],
                   R2[0] * g[1] - R2[1] * g[0]};
  double gr1[3] = {g[1] * R1[2] - g[2] * R1[1], g[2] * R1[0] - g[0] * R1[2],
                   g[0] * R1[1] - g[1] * R1[0]};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    gR1[c] = Q * (dfa * R1[c] / a + dfd * R2[c]) + f * r2g[c];
    gR2[c] = Q * (dfb * R2[c] / b + dfd * R1[c]) + f * gr1[c];
  }
}

// ------------------------------------------------------------------- LIA
// Seeds input component k (0..14: x, gi, gb, gii, gbb) and returns the
// directional derivative of the local velocity.
__device__ void lia_vjp_point(int vel, int order, int fixed, double G, double a, const double *X,
                              const double *GI, const double *GB, const double *GII,
                              const double *GBB, const double *ub, double *bar) {
  const int nin = order == 4 ? 15 : 9;
  for (int k = 0; k < 15; k++) bar[k] = 0.;
  for (int k = 0; k < nin; k++) {
    Dual in[15];
    const double *src[5] = {X, GI, GB, GII, GBB};
    for (int q = 0; q < 15; q++) in[q] = Dual(src[q / 3][q % 3], q == k ? 1. : 0.);
    Dual out[3];
    lia_term(vel, order, fixed, G, a, in, in + 3, in + 6, in + 9, in + 12, out);
    bar[k] = ub[0] * out[0].d + ub[1] * out[1].d + ub[2] * out[2].d;
  }
}

__global__ void k_lia_vjp(int n, const double *__restrict__ x, const int *__restrict__ inf,
                          const double *__restrict__ gi, const double *__restrict__ gb,
                          const double *__restrict__ gii, const double *__restrict__ gbb,
                          const double *__restrict__ ubar, int vel, int order, int fixed, double G,
                          double a, double *xb, double *gib, double *gbb_, double *giib,
                          double *gbbb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double bar[15];
  if (inf[i] == 0) {
    for (int k = 0; k < 15; k++) bar[k] = 0.;
  } else {
    double X[3], GI[3], GB[3], GII[3], GBB[3], ub[3];
    for (int c = 0; c < 3; c++) {
      X[c] = x[3 * i + c]; GI[c] = gi[3 * i + c]; GB[c] = gb[3 * i + c];
      GII[c] = gii[3 * i + c]; GBB[c] = gbb[3 * i + c]; ub[c] = ubar[3 * i + c];
    }
    lia_vjp_point(vel, order, fixed, G, a, X, GI, GB, GII, GBB, ub, bar);
  }
  for (int c = 0; c < 3; c++) {
    xb[3 * i + c] = bar[c];
    gib[3 * i + c] = bar[3 + c];
    gbb_[3 * i + c] = bar[6 + c];
    giib[3 * i + c] = bar[9 + c];
    gbbb[3 * i + c] = bar[12 + c];
  }
}

// ------------------------------------------------------------ direct sum
__device__ __forceinline__ double shiftv(double v, int m, double L) {
  return m == 0 ? v : (m > 0 ? v + L : v - L);
}

#define VT 128
// Target pass: x_bar_i += -sum_j (grad_R1 + grad_R2) over sources j and images,
// with the skip rules of src/timestep.f90:471, 496.
template <int BC>
__global__ void __launch_bounds__(VT) k_dvjp_tgt(int na, const int *__restrict__ act,
                                                 const double *__restrict__ x,
                                                 const double *__restrict__ gi,
                                                 const int *__restrict__ beh,
                                                 const double *__restrict__ ubar, double gfac,
                                                 double L, double *xb) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  __shared__ double sx[VT][3], sg[VT][3];
  __shared__ int sj[VT];
  int q = blockIdx.x * VT + threadIdx.x;
  bool live = q < na;
  int i = live ? act[q] : 0;
  double xi[3] = {0., 0., 0.}, g[3] = {0., 0., 0.}, acc[3] = {0., 0., 0.};
  int bi = -1, ii = i + 1;
  if (live) {
    for (int c = 0; c < 3; c++) { xi[c] = x[3 * i + c]; g[c] = gfac * ubar[3 * i + c]; }
    bi = beh[i];
  }
  for (int t0 = 0; t0 < na; t0 += VT) {
    __syncthreads();
    int k = t0 + threadIdx.x;
    if (k < na) {
      int j = act[k];
      for (int c = 0; c < 3; c++) { sx[threadIdx.x][c] = x[3 * j + c]; sg[threadIdx.x][c] = gi[3 * j + c]; }
      sj[threadIdx.x] = j + 1;
    }
    __syncthreads();
    if (!live) continue;
    int m = min(VT, na - t0);
    for (int kk = 0; kk < m; kk++) {
      int jj = sj[kk];
      if (jj == bi) continue;
      for (int im = -1; im < NIMG; im++) {
        if (im < 0 && jj == ii) continue;
        int ma = 0, mb = 0, mc = 0;
        if (im >= 0) qv_img_shift(BC, im, &ma, &mb, &mc);
        double R1[3] = {shiftv(sx[kk][0], ma, L) - xi[0], shiftv(sx[kk][1], mb, L) - xi[1],
                        shiftv(sx[kk][2], mc, L) - xi[2]};
        double R2[3] = {shiftv(sg[kk][0], ma, L) - xi[0], shiftv(sg[kk][1], mb, L) - xi[1],
                        shiftv(sg[kk][2], mc, L) - xi[2]};
        double s[3] = {sg[kk][0] - sx[kk][0], sg[kk][1] - sx[kk][1], sg[kk][2] - sx[kk][2]};
        double cx = R1[1] * s[2] - R1[2] * s[1], cy = R1[2] * s[0] - R1[0] * s[2],
               cz = R1[0] * s[1] - R1[1] * s[0];
        if (cx * cx + cy * cy + cz * cz == 0.) continue;  // 4ac - b^2 == 0 (skipped forward)
        double a1[3], a2[3];
        seg_grad(R1, R2, g, a1, a2);
        for (int c = 0; c < 3; c++) acc[c] -= a1[c] + a2[c];
      }
    }
  }
  if (live)
    for (int c = 0; c < 3; c++) xb[3 * i + c] += acc[c];
}

// Source pass: x_bar_j += sum_i grad_R1, ghosti_bar_j += sum_i grad_R2.
template <int BC>
__global__ void __launch_bounds__(VT) k_dvjp_src(int na, const int *__restrict__ act,
                                                 const double *__restrict__ x,
                                                 const double *__restrict__ gi,
                                                 const int *__restrict__ beh,
                                                 const double *__restrict__ ubar, double gfac,
                                                 double L, double *xb, double *gib) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  __shared__ double tx[VT][3], tg[VT][3];
  __shared__ int tb[VT], ti[VT];
  int q = blockIdx.x * VT + threadIdx.x;
  bool live = q < na;
  int j = live ? act[q] : 0;
  double xj[3] = {0., 0., 0.}, gj[3] = {0., 0., 0.}, s[3], a1s[3] = {0., 0., 0.},
         a2s[3] = {0., 0., 0.};
  int jj = j + 1;
  if (live)
    for (int c = 0; c < 3; c++) { xj[c] = x[3 * j + c]; gj[c] = gi[3 * j + c]; }
  for (int c = 0; c < 3; c++) s[c] = gj[c] - xj[c];
  for (int t0 = 0; t0 < na; t0 += VT) {
    __syncthreads();
    int k = t0 + threadIdx.x;
    if (k < na) {
      int i = act[k];
      for (int c = 0; c < 3; c++) { tx[threadIdx.x][c] = x[3 * i + c]; tg[threadIdx.x][c] = gfac * ubar[3 * i + c]; }
      tb[threadIdx.x] = beh[i];
      ti[threadIdx.x] = i + 1;
    }
    __syncthreads();
    if (!live) continue;
    int m = min(VT, na - t0);
    for (int kk = 0; kk < m; kk++) {
      if (jj == tb[kk]) continue;
      for (int im = -1; im < NIMG; im++) {
        if (im < 0 && jj == ti[kk]) continue;
        int ma = 0, mb = 0, mc = 0;
        if (im >= 0) qv_img_shift(BC, im, &ma, &mb, &mc);
        double R1[3] = {shiftv(xj[0], ma, L) - tx[kk][0], shiftv(xj[1], mb, L) - tx[kk][1],
                        shiftv(xj[2], mc, L) - tx[kk][2]};
        double R2[3] = {shiftv(gj[0], ma, L) - tx[kk][0], shiftv(gj[1], mb, L) - tx[kk][1],
                        shiftv(gj[2], mc, L) - tx[kk][2]};
        double cx = R1[1] * s[2] - R1[2] * s[1], cy = R1[2] * s[0] - R1[0] * s[2],
               cz = R1[0] * s[1] - R1[1] * s[0];
        if (cx * cx + cy * cy + cz * cz == 0.) continue;
        double a1[3], a2[3];
        seg_grad(R1, R2, tg[kk], a1, a2);
        for (int c = 0; c < 3; c++) { a1s[c] += a1[c]; a2s[c] += a2[c]; }
      }
    }
  }
  if (live)
    for (int c = 0; c < 3; c++) { xb[3 * j + c] += a1s[c]; gib[3 * j + c] += a2s[c]; }
}

// ------------------------------------------------------------ tree walk
#define AW 4
#define ASTK (7 * QV_MAX_DEPTH + 16)
#define ANSPLIT 8

struct WalkVjpArgs {
  int n_act, ngroups;
  const int *perm, *inf, *beh;
  const double *x, *ubar;
  const WNode64 *w64;
  const WPay64 *p64;
  const int *first;
  double L, theta, gfac;
  int extra;
  double *xb, *gib, *nb;  // nb: per-node adjoint of (cent, circ, C) = 15 doubles
};

__device__ __forceinline__ double sh_of(int m, double L) { return m == 0 ? 0. : (m > 0 ? L : -L); }

__device__ __forceinline__ double wsum(double v, unsigned mask) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

__device__ __forceinline__ bool open_exact(const double *xi, const WNode64 &h, const double *s,
                                           double theta, int extra, double &dist) {
  double d0 = __dsub_rn(xi[0], __dadd_rn(h.cx, s[0]));
  double d1 = __dsub_rn(xi[1], __dadd_rn(h.cy, s[1]));
  double d2 = __dsub_rn(xi[2], __dadd_rn(h.cz, s[2]));
  dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
  double th;
  if (extra) {
    double r = __dsub_rn(dist, h.geo);
    th = r > 0. ? __ddiv_rn(h.width, r) : __ddiv_rn(h.width, dist);
  } else {
    th = __ddiv_rn(h.width, dist);
  }
  return !(th < theta);
}

template <int BC>
__global__ void __launch_bounds__(AW * 32, 5) k_walk_vjp(WalkVjpArgs a) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  __shared__ int2 stk[AW][ASTK];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int2 *st = stk[wid];
  const int items = a.ngroups * (ANSPLIT + NIMG);
  for (int item = blockIdx.x * AW + wid; item < items; item += gridDim.x * AW) {
    const int sl = item / a.ngroups, gg = item - sl * a.ngroups;
    int q = gg * 32 + lane;
    bool live = q < a.n_act;
    int i = live ? a.perm[q] : 0;
    double xi[3] = {0., 0., 0.}, g[3] = {0., 0., 0.}, acc[3] = {0., 0., 0.};
    int bi = -1, fi = -1, ii = -1;
    if (live) {
      for (int c = 0; c < 3; c++) { xi[c] = a.x[3 * i + c]; g[c] = a.gfac * a.ubar[3 * i + c]; }
      bi = a.beh[i]; fi = a.inf[i]; ii = i + 1;
    }
    int ma = 0, mb = 0, mc = 0;
    if (sl >= ANSPLIT) qv_img_shift(BC, sl - ANSPLIT, &ma, &mb, &mc);
    const double s[3] = {sh_of(ma, a.L), sh_of(mb, a.L), sh_of(mc, a.L)};
    int top = 0;
    if (sl >= ANSPLIT) {
      const unsigned lm = __ballot_sync(0xffffffffu, live);
      if (lane == 0) st[0] = make_int2(0, (int)lm);
      top = lm ? 1 : 0;
    } else {
      const WNode64 r = a.w64[0];
      if (r.count == 1) {
        const unsigned lm = __ballot_sync(0xffffffffu, live);
        if (sl == 0 && lane == 0) st[0] = make_int2(0, (int)lm);
        top = (sl == 0 && lm) ? 1 : 0;
      } else {
        bool ropen = false;
        double dd;
        if (live) ropen = open_exact(xi, r, s, a.theta, a.extra, dd);
        const unsigned om = __ballot_sync(0xffffffffu, ropen);
        if (om && sl < r.nchild) {
          if (lane == 0) st[0] = make_int2(r.child_first + sl, (int)om);
          top = 1;
        }
      }
    }
    __syncwarp();
    while (top > 0) {
      top--;
      int2 e = st[top];
      __syncwarp();
      const int node = e.x;
      const bool in = (((unsigned)e.y) >> lane) & 1u;
      const WNode64 h = a.w64[node];
      if (h.count == 1) {
        bool ev = false;
        double gR1[3] = {0., 0., 0.}, gR2[3] = {0., 0., 0.};
        if (in) {
          int j = h.jb;
          if (j != ii && j != bi && j != fi) {
            const WPay64 &P = a.p64[node];
            double R1[3], R2[3];
            for (int c = 0; c < 3; c++) {
              R1[c] = P.a[c] + s[c] - xi[c];
              R2[c] = P.b[c] + s[c] - xi[c];
            }
            seg_grad(R1, R2, g, gR1, gR2);
            for (int c = 0; c < 3; c++) acc[c] -= gR1[c] + gR2[c];
            ev = true;
          }
        }
        if (__any_sync(0xffffffffu, ev)) {
          double v[6];
          for (int c = 0; c < 3; c++) { v[c] = wsum(gR1[c], 0xffffffffu); v[3 + c] = wsum(gR2[c], 0xffffffffu); }
          if (lane == 0) {
            int p = a.first[node];
            for (int c = 0; c < 3; c++) {
              atomicAdd(&a.xb[3 * p + c], v[c]);
              atomicAdd(&a.gib[3 * p + c], v[3 + c]);
            }
          }
        }
      } else {
        bool open = false, far = false;
        double nbv[15];
        for (int k = 0; k < 15; k++) nbv[k] = 0.;
        if (in) {
          double dist;
          open = open_exact(xi, h, s, a.theta, a.extra, dist);
          if (!open && node != 0) {
            far = true;
            const WPay64 &P = a.p64[node];
            double v[3] = {xi[0] - (h.cx + s[0]), xi[1] - (h.cy + s[1]), xi[2] - (h.cz + s[2])};
            double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            double r1 = 1. / sqrt(d2);
            double r3 = r1 * r1 * r1, r5 = r3 / d2, r7 = r5 / d2;
            double z[3];
            for (int l = 0; l < 3; l++) z[l] = v[0] * P.C[l] + v[1] * P.C[3 + l] + v[2] * P.C[6 + l];
            double av[3] = {P.a[1] * v[2] - P.a[2] * v[1] - P.b[0], P.a[2] * v[0] - P.a[0] * v[2] - P.b[1],
                            P.a[0] * v[1] - P.a[1] * v[0] - P.b[2]};
            double bv[3] = {v[1] * z[2] - v[2] * z[1], v[2] * z[0] - v[0] * z[2], v[0] * z[1] - v[1] * z[0]};
            double ga = g[0] * av[0] + g[1] * av[1] + g[2] * av[2];
            double gb = g[0] * bv[0] + g[1] * bv[1] + g[2] * bv[2];
            double gxc[3] = {g[1] * P.a[2] - g[2] * P.a[1], g[2] * P.a[0] - g[0] * P.a[2],
                             g[0] * P.a[1] - g[1] * P.a[0]};
            double zxg[3] = {z[1] * g[2] - z[2] * g[1], z[2] * g[0] - z[0] * g[2], z[0] * g[1] - z[1] * g[0]};
            double gxv[3] = {g[1] * v[2] - g[2] * v[1], g[2] * v[0] - g[0] * v[2], g[0] * v[1] - g[1] * v[0]};
            double Cg[3];
            for (int p = 0; p < 3; p++) Cg[p] = P.C[3 * p] * gxv[0] + P.C[3 * p + 1] * gxv[1] + P.C[3 * p + 2] * gxv[2];
            double gv[3];
            for (int c = 0; c < 3; c++)
              gv[c] = -3. * r5 * ga * v[c] + r3 * gxc[c] - 15. * r7 * gb * v[c] + 3. * r5 * (zxg[c] + Cg[c]);
            for (int c = 0; c < 3; c++) acc[c] += gv[c];
            // node adjoint: cent (0-2), circ (3-5), C row-major (6-14)
            for (int c = 0; c < 3; c++) nbv[c] = -gv[c];
            double vxg[3] = {v[1] * g[2] - v[2] * g[1], v[2] * g[0] - v[0] * g[2], v[0] * g[1] - v[1] * g[0]};
            for (int c = 0; c < 3; c++) nbv[3 + c] = r3 * vxg[c];
            double zb[3] = {3. * r5 * gxv[0], 3. * r5 * gxv[1], 3. * r5 * gxv[2]};
            for (int p = 0; p < 3; p++)
              for (int l = 0; l < 3; l++) nbv[6 + 3 * p + l] = v[p] * zb[l];
            double wb[3] = {-r3 * g[0], -r3 * g[1], -r3 * g[2]};
            // w_0 = C12 - C21, w_1 = C20 - C02, w_2 = C01 - C10
            nbv[6 + 5] += wb[0]; nbv[6 + 7] -= wb[0];
            nbv[6 + 6] += wb[1]; nbv[6 + 2] -= wb[1];
            nbv[6 + 1] += wb[2]; nbv[6 + 3] -= wb[2];
          }
        }
        if (__any_sync(0xffffffffu, far)) {
          for (int k = 0; k < 15; k++) {
            double t = wsum(nbv[k], 0xffffffffu);
            if (lane == 0) atomicAdd(&a.nb[15 * node + k], t);
          }
        }
        unsigned om = __ballot_sync(0xffffffffu, open);
        if (om) {
          int nc = h.nchild;
          if (top + nc > ASTK) nc = 0;  // unreachable within QV_MAX_DEPTH
          if (lane < nc) st[top + lane] = make_int2(h.child_first + nc - 1 - lane, (int)om);
          top += nc;
        }
        __syncwarp();
      }
    }
    if (live)
      for (int c = 0; c < 3; c++) atomicAdd(&a.xb[3 * i + c], acc[c]);
  }
}

// Node adjoint -> point adjoints through cent = sum x / n, circ = sum (gi - x),
// C = sum x (gi - x)^T - cent circ^T (src/tree.f90:154-179).  One warp per node.
__global__ void k_moment_vjp(int n_nodes, const int *__restrict__ level,
                             const int *__restrict__ start, const int *__restrict__ count,
                             const int *__restrict__ ord, int cap_pts, const double *__restrict__ x,
                             const double *__restrict__ gi, const double *__restrict__ cent,
                             const double *__restrict__ circ, const double *__restrict__ nb,
                             double *xb, double *gib) {
  int lane = threadIdx.x & 31;
  int k = 1 + (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  if (k >= n_nodes) return;
  const double *B = nb + 15 * k;
  double Cb[9], cb[3], qb[3];
  bool any = false;
  for (int t = 0; t < 15; t++) any |= B[t] != 0.;
  if (!any) return;
  for (int t = 0; t < 9; t++) Cb[t] = B[6 + t];
  // C = C_raw - cent circ^T
  for (int r = 0; r < 3; r++) {
    cb[r] = B[r] - (Cb[3 * r] * circ[3 * k] + Cb[3 * r + 1] * circ[3 * k + 1] + Cb[3 * r + 2] * circ[3 * k + 2]);
    qb[r] = B[3 + r] - (Cb[r] * cent[3 * k] + Cb[3 + r] * cent[3 * k + 1] + Cb[6 + r] * cent[3 * k + 2]);
  }
  int n = count[k];
  const int *o = ord + (size_t)level[k] * cap_pts + start[k];
  for (int t = lane; t < n; t += 32) {
    int p = o[t];
    double X[3], GI[3], s[3];
    for (int c = 0; c < 3; c++) { X[c] = x[3 * p + c]; GI[c] = gi[3 * p + c]; s[c] = GI[c] - X[c]; }
    double dx[3], dg[3];
    for (int c = 0; c < 3; c++) {
      double Cs = Cb[3 * c] * s[0] + Cb[3 * c + 1] * s[1] + Cb[3 * c + 2] * s[2];   // (C_b s)_c
      double CtX = Cb[c] * X[0] + Cb[3 + c] * X[1] + Cb[6 + c] * X[2];           // (C_b^T x)_c
      dx[c] = cb[c] / n - qb[c] + Cs - CtX;
      dg[c] = qb[c] + CtX;
    }
    for (int c = 0; c < 3; c++) {
      atomicAdd(&xb[3 * p + c], dx[c]);
      atomicAdd(&gib[3 * p + c], dg[c]);
    }
  }
}

// Ghost adjoint: gi_i = x_infront(i), gb_i = x_behind(i), gii_i = x_infront(infront(i)),
// gbb_i = x_behind(behind(i)) (shifts by +-L are constants).
__global__ void k_ghost_vjp(int n, const int *__restrict__ inf, const int *__restrict__ beh,
                            const double *__restrict__ xb, const double *__restrict__ gib,
                            const double *__restrict__ gbb_, const double *__restrict__ giib,
                            const double *__restrict__ gbbb, double *out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (inf[p] == 0) {
    for (int c = 0; c < 3; c++) out[3 * p + c] = 0.;
    return;
  }
  int b = beh[p] - 1, f = inf[p] - 1, bb = beh[b] - 1, ff = inf[f] - 1;
  for (int c = 0; c < 3; c++)
    out[3 * p + c] = xb[3 * p + c] + gib[3 * b + c] + gbb_[3 * f + c] + giib[3 * bb + c] + gbbb[3 * ff + c];
}

// ------------------------------------------------------------------ energy
// W_q = u_q . (x_q x s'_q), l_q = |x_q - ghosti_q|.
template <typename T>
__device__ __forceinline__ T energy_w(int order, const T *X, const T *GI, const T *GB,
                                      const T *GII, const T *GBB, const double *u) {
  T s1[3], s2[3];
  lia_derivs(order, X, GI, GB, GII, GBB, s1, s2);
  T c0 = X[1] * s1[2] - X[2] * s1[1], c1 = X[2] * s1[0] - X[0] * s1[2], c2 = X[0] * s1[1] - X[1] * s1[0];
  return u[0] * c0 + u[1] * c1 + u[2] * c2;
}

__global__ void k_energy_w(int n, const double *__restrict__ x, const double *__restrict__ u,
                           const int *__restrict__ inf, const double *__restrict__ gi,
                           const double *__restrict__ gb, const double *__restrict__ gii,
                           const double *__restrict__ gbb, int order, double *W, double *ell) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n || inf[q] == 0) return;
  double X[3], GI[3], GB[3], GII[3], GBB[3], U[3];
  for (int c = 0; c < 3; c++) {
    X[c] = x[3 * q + c]; GI[c] = gi[3 * q + c]; GB[c] = gb[3 * q + c];
    GII[c] = gii[3 * q + c]; GBB[c] = gbb[3 * q + c]; U[c] = u[3 * q + c];
  }
  W[q] = energy_w(order, X, GI, GB, GII, GBB, U);
  ell[q] = lia_dist(X, GI);
}

// E = G sum_i 0.5 l_i (W_i + W_infront(i)); per point the term, the u
// gradient G 0.5 (l_q + l_behind(q)) x_q x s'_q, and the stencil gradients.
__global__ void k_energy_grad(int n, const double *__restrict__ x, const double *__restrict__ u,
                              const int *__restrict__ inf, const int *__restrict__ beh,
                              const double *__restrict__ gi, const double *__restrict__ gb,
                              const double *__restrict__ gii, const double *__restrict__ gbb,
                              const double *__restrict__ W, const double *__restrict__ ell,
                              int order, double G, double *eterm, double *ub, double *xb,
                              double *gib, double *gbb_, double *giib, double *gbbb) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  for (int c = 0; c < 3; c++) {
    ub[3 * q + c] = 0.; xb[3 * q + c] = 0.; gib[3 * q + c] = 0.; gbb_[3 * q + c] = 0.;
    giib[3 * q + c] = 0.; gbbb[3 * q + c] = 0.;
  }
  eterm[q] = 0.;
  if (inf[q] == 0) return;
  int a = inf[q] - 1, b = beh[q] - 1;
  double X[3], GI[3], GB[3], GII[3], GBB[3], U[3];
  for (int c = 0; c < 3; c++) {
    X[c] = x[3 * q + c]; GI[c] = gi[3 * q + c]; GB[c] = gb[3 * q + c];
    GII[c] = gii[3 * q + c]; GBB[c] = gbb[3 * q + c]; U[c] = u[3 * q + c];
  }
  eterm[q] = 0.5 * ell[q] * (W[q] + W[a]);
  double cW = G * 0.5 * (ell[q] + ell[b]);
  double cL = G * 0.5 * (W[q] + W[a]);
  // dE/du_q = cW (x_q x s'_q)
  double s1[3], s2[3];
  lia_derivs(order, X, GI, GB, GII, GBB, s1, s2);
  ub[3 * q] = cW * (X[1] * s1[2] - X[2] * s1[1]);
  ub[3 * q + 1] = cW * (X[2] * s1[0] - X[0] * s1[2]);
  ub[3 * q + 2] = cW * (X[0] * s1[1] - X[1] * s1[0]);
  // dE/d(stencil) through W_q
  const int nin = order == 4 ? 15 : 9;
  double bar[15];
  for (int k = 0; k < 15; k++) bar[k] = 0.;
  for (int k = 0; k < nin; k++) {
    Dual in[15];
    const double *src[5] = {X, GI, GB, GII, GBB};
    for (int t = 0; t < 15; t++) in[t] = Dual(src[t / 3][t % 3], t == k ? 1. : 0.);
    bar[k] = cW * energy_w(order, in, in + 3, in + 6, in + 9, in + 12, U).d;
  }
  // dE/dl_q: l_q = |x_q - gi_q|
  for (int c = 0; c < 3; c++) {
    double dl = ell[q] > 0. ? (X[c] - GI[c]) / ell[q] : 0.;
    bar[c] += cL * dl;
    bar[3 + c] -= cL * dl;
  }
  for (int c = 0; c < 3; c++) {
    xb[3 * q + c] = bar[c]; gib[3 * q + c] = bar[3 + c]; gbb_[3 * q + c] = bar[6 + c];
    giib[3 * q + c] = bar[9 + c]; gbbb[3 * q + c] = bar[12 + c];
  }
}

// ------------------------------------------------------------- field points
// biot_savart_general(_shift) at point x (src/timestep.f90:516-563): every
// active segment, no skip; and the exact gradient du_i/dx_k of the unshifted
// sum (what velocity_quasip differentiates) or of the full periodic sum.
template <int BC>
__global__ void k_field(int m, const double *__restrict__ pts, int grad_images, int na,
                        const double *__restrict__ src, double G, double L, double *u,
                        double *dudx) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  double X[3] = {pts[3 * t], pts[3 * t + 1], pts[3 * t + 2]};
  double acc[3] = {0., 0., 0.}, J[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  for (int j = 0; j < na; j++) {
    const double *s = src + 8 * j;
    for (int im = -1; im < NIMG; im++) {
      int ma = 0, mb = 0, mc = 0;
      if (im >= 0) qv_img_shift(BC, im, &ma, &mb, &mc);
      double d[3] = {shiftv(s[0], ma, L) - X[0], shiftv(s[1], mb, L) - X[1], shiftv(s[2], mc, L) - X[2]};
      double a = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      double b = 2. * (d[0] * s[3] + d[1] * s[4] + d[2] * s[5]);
      double c = s[6];
      double disc = 4. * a * c - b * b;
      if (disc == 0.) continue;  // src/timestep.f90:531
      double fac = (2. * c + b) / sqrt(a + b + c) - b / sqrt(a);
      double sc = G / (2. * QV_PI) / disc * fac;
      acc[0] += (d[1] * s[5] - d[2] * s[4]) * sc;
      acc[1] += (d[2] * s[3] - d[0] * s[5]) * sc;
      acc[2] += (d[0] * s[4] - d[1] * s[3]) * sc;
      if (im < 0 || grad_images) {
        double R2[3] = {d[0] + s[3], d[1] + s[4], d[2] + s[5]};
        for (int r = 0; r < 3; r++) {  // row r of the Jacobian: g = e_r
          double g[3] = {r == 0 ? G / (4. * QV_PI) : 0., r == 1 ? G / (4. * QV_PI) : 0.,
                         r == 2 ? G / (4. * QV_PI) : 0.};
          double g1[3], g2[3];
          seg_grad(d, R2, g, g1, g2);
          for (int k = 0; k < 3; k++) J[3 * r + k] -= g1[k] + g2[k];
        }
      }
    }
  }
  for (int c = 0; c < 3; c++) u[3 * t + c] = acc[c];
  for (int k = 0; k < 9; k++) dudx[9 * t + k] = J[k];
}

// ------------------------------------------------------------------ host side
static int adj_reserve(qv_ctx *c) {
  size_t v = sizeof(double) * 3 * (size_t)std::max(c->n, 1);
  if (c->adj_n >= c->n && c->adj_xb) return QV_OK;
  int rc;
  double **bufs[] = {&c->adj_xb, &c->adj_gib, &c->adj_gbb, &c->adj_giib, &c->adj_gbbb};
  for (double **b : bufs)
    if ((rc = qv_grow(c, (void **)b, v))) return rc;
  c->adj_n = c->n;
  return QV_OK;
}

// ------------------------------------------------------ Adams-Bashforth step
// The position update of pmotion (src/timestep.f90:48-71) followed by the wrap
// of enforce_periodic (src/periodic.f90:188-214), from device arrays, and its
// adjoint.  The forward takes the update kernel's operations (qv_ab.cuh), so a
// differentiable trajectory is bitwise the trajectory qv_step would make from
// the same velocities.  The rung is chosen by exact-zero tests of the history,
// piecewise constant in every input, and the wrap moves a point by a constant:
// the adjoint is x_bar = x_out_bar and (u, u1, u2, u3)_bar = the rung's
// coefficients times x_out_bar.  Empty slots (infront = 0) do not move.
__global__ void k_ab_fwd(int n, double dt, const double *__restrict__ x,
                         const double *__restrict__ u, const double *__restrict__ u1,
                         const double *__restrict__ u2, const double *__restrict__ u3,
                         const int *__restrict__ inf, int lo_axis, double L, double *xo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (inf[i] == 0) {
    for (int c = 0; c < 3; c++) xo[3 * i + c] = x[3 * i + c];
    return;
  }
  double U1[3], U2[3], U3[3];
  for (int c = 0; c < 3; c++) {
    U1[c] = u1[3 * i + c]; U2[c] = u2[3 * i + c]; U3[c] = u3[3 * i + c];
  }
  const int rung = ab_rung(U1, U2, U3);
  for (int c = 0; c < 3; c++) {
    const double r = ab_update(rung, dt, x[3 * i + c], u[3 * i + c], U1[c], U2[c], U3[c]);
    xo[3 * i + c] = c >= lo_axis ? wrap_coord(r, L) : r;
  }
}

__global__ void k_ab_vjp(int n, double dt, const double *__restrict__ u1,
                         const double *__restrict__ u2, const double *__restrict__ u3,
                         const int *__restrict__ inf, const double *__restrict__ xob, double *xb,
                         double *ub, double *u1b, double *u2b, double *u3b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double k[4] = {0., 0., 0., 0.};
  if (inf[i] != 0) {
    double U1[3], U2[3], U3[3];
    for (int c = 0; c < 3; c++) {
      U1[c] = u1[3 * i + c]; U2[c] = u2[3 * i + c]; U3[c] = u3[3 * i + c];
    }
    ab_coef(ab_rung(U1, U2, U3), dt, k);
  }
  for (int c = 0; c < 3; c++) {
    const double g = xob[3 * i + c];
    xb[3 * i + c] = g;
    ub[3 * i + c] = k[0] * g;
    u1b[3 * i + c] = k[1] * g;
    u2b[3 * i + c] = k[2] * g;
    u3b[3 * i + c] = k[3] * g;
  }
}

static int ab_lo_axis(int bc) {
  return bc == QV_BC_PERIODIC ? 0 : bc == QV_BC_OPENX ? 1 : bc == QV_BC_OPENXY ? 2 : 3;
}

extern "C" int qv_ab_step_device(qv_ctx *c, int n, const double *x, const double *u,
                                 const double *u1, const double *u2, const double *u3,
                                 double *x_out) {
  if (!c) return QV_ERR_ARG;
  if (n != c->n) return qv_fail(c, QV_ERR_STATE, "qv_ab_step_device: %d slots, context holds %d", n, c->n);
  if (n == 0) return QV_OK;
  if (!x || !u || !u1 || !u2 || !u3 || !x_out) return qv_fail(c, QV_ERR_ARG, "null array");
  k_ab_fwd<<<nblk(n, 256), 256, 0, c->stream>>>(n, c->p.dt, x, u, u1, u2, u3, c->infront,
                                                ab_lo_axis(c->p.boundary), c->p.box_size, x_out);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

extern "C" int qv_ab_vjp_device(qv_ctx *c, int n, const double *u1, const double *u2,
                                const double *u3, const double *xbar_out, double *xbar,
                                double *ubar, double *u1bar, double *u2bar, double *u3bar) {
  if (!c) return QV_ERR_ARG;
  if (n != c->n) return qv_fail(c, QV_ERR_STATE, "qv_ab_vjp_device: %d slots, context holds %d", n, c->n);
  if (n == 0) return QV_OK;
  if (!u1 || !u2 || !u3 || !xbar_out || !xbar || !ubar || !u1bar || !u2bar || !u3bar)
    return qv_fail(c, QV_ERR_ARG, "null array");
  k_ab_vjp<<<nblk(n, 256), 256, 0, c->stream>>>(n, c->p.dt, u1, u2, u3, c->infront, xbar_out,
                                                xbar, ubar, u1bar, u2bar, u3bar);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

extern "C" int qv_velocity_vjp(qv_ctx *c, const double *ubar, double *xbar) {
  if (!c || !ubar || !xbar) return QV_ERR_ARG;
  if (c->n == 0) return QV_OK;
  int rc;
  if (!c->ghosts_valid)
    if ((rc = qv_launch_ghosts(c))) return rc;
  if ((rc = adj_reserve(c))) return rc;
  const qv_params &p = c->p;
  k_lia_vjp<<<nblk(c->n, 128), 128, 0, c->stream>>>(
      c->n, c->x, c->infront, c->gi, c->gb, c->gii, c->gbb, ubar, p.velocity, p.deriv_order,
      p.fixed_lia_beta, p.quant_circ, p.corea, c->adj_xb, c->adj_gib, c->adj_gbb, c->adj_giib,
      c->adj_gbbb);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  double gfac = p.quant_circ / (4. * QV_PI);
  if (p.velocity == QV_VEL_BS) {
    if ((rc = qv_compact_active(c))) return rc;
    int na = c->n_act;
    if (na > 0) {
      int nb = nblk(na, VT);
      switch (p.boundary) {
#define QV_DVJP(BCV)                                                                              \
  case BCV:                                                                                       \
    k_dvjp_tgt<BCV><<<nb, VT, 0, c->stream>>>(na, c->act, c->x, c->gi, c->behind, ubar, gfac,     \
                                              p.box_size, c->adj_xb);                             \
    k_dvjp_src<BCV><<<nb, VT, 0, c->stream>>>(na, c->act, c->x, c->gi, c->behind, ubar, gfac,     \
                                              p.box_size, c->adj_xb, c->adj_gib);                 \
    break;
        QV_DVJP(QV_BC_OPEN)
        QV_DVJP(QV_BC_PERIODIC)
        QV_DVJP(QV_BC_OPENX)
        QV_DVJP(QV_BC_OPENXY)
#undef QV_DVJP
        default:
          return qv_fail(c, QV_ERR_UNSUPPORTED, "boundary %d", p.boundary);
      }
      QV_LAUNCH_CHECK(c);
      QV_COUNT(c, 2);
    }
  } else if (p.velocity == QV_VEL_TREE) {
    if (!c->tree.valid)
      if ((rc = qv_launch_tree_build(c))) return rc;
    if ((rc = qv_tree_finalize_root(c))) return rc;
    TreeBuf &t = c->tree;
    size_t nbytes = sizeof(double) * 15 * (size_t)t.n_nodes;
    if (nbytes > c->adj_nb_bytes) {
      if ((rc = qv_grow(c, (void **)&c->adj_nb, nbytes))) return rc;
      c->adj_nb_bytes = nbytes;
    }
    QV_CUDA(c, cudaMemsetAsync(c->adj_nb, 0, nbytes, c->stream));
    if (t.n_act > 0) {
      WalkVjpArgs a;
      a.n_act = t.n_act; a.ngroups = (t.n_act + 31) / 32; a.perm = t.perm; a.inf = c->infront;
      a.beh = c->behind; a.x = c->x; a.ubar = ubar; a.w64 = t.w64; a.p64 = t.p64; a.first = t.first;
      a.L = p.box_size; a.theta = p.tree_theta; a.gfac = gfac; a.extra = p.tree_extra_correction;
      a.xb = c->adj_xb; a.gib = c->adj_gib; a.nb = c->adj_nb;
      int nimg = qv_img_count(p.boundary);
      long items = (long)a.ngroups * (ANSPLIT + nimg);
      int nb = (int)std::min<long>((items + AW - 1) / AW, 64L * c->sm_count);
      switch (p.boundary) {
        case QV_BC_OPEN: k_walk_vjp<QV_BC_OPEN><<<nb, AW * 32, 0, c->stream>>>(a); break;
        case QV_BC_PERIODIC: k_walk_vjp<QV_BC_PERIODIC><<<nb, AW * 32, 0, c->stream>>>(a); break;
        case QV_BC_OPENX: k_walk_vjp<QV_BC_OPENX><<<nb, AW * 32, 0, c->stream>>>(a); break;
        case QV_BC_OPENXY: k_walk_vjp<QV_BC_OPENXY><<<nb, AW * 32, 0, c->stream>>>(a); break;
        default: return qv_fail(c, QV_ERR_UNSUPPORTED, "boundary %d", p.boundary);
      }
      QV_LAUNCH_CHECK(c);
      if (t.n_nodes > 1) {
        k_moment_vjp<<<nblk((long)(t.n_nodes - 1) * 32, 256), 256, 0, c->stream>>>(
            t.n_nodes, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, c->gi, t.cent, t.circ,
            c->adj_nb, c->adj_xb, c->adj_gib);
        QV_LAUNCH_CHECK(c);
      }
      QV_COUNT(c, 2);
    }
  }
  k_ghost_vjp<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->infront, c->behind, c->adj_xb,
                                                      c->adj_gib, c->adj_gbb, c->adj_giib,
                                                      c->adj_gbbb, xbar);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  return QV_OK;
}

extern "C" int qv_energy_grad(qv_ctx *c, const double *u, double *energy, double *xbar,
                              double *ubar) {
  if (!c || !u || !energy || !xbar || !ubar) return QV_ERR_ARG;
  if (c->n == 0) { *energy = 0.; return QV_OK; }
  int rc;
  if (!c->ghosts_valid)
    if ((rc = qv_launch_ghosts(c))) return rc;
  if ((rc = adj_reserve(c))) return rc;
  int n = c->n;
  double *W = nullptr;
  QV_CUDA(c, cudaMalloc((void **)&W, sizeof(double) * 3 * (size_t)n));
  double *ell = W + n, *eterm = W + 2 * (size_t)n;
  QV_CUDA(c, cudaMemsetAsync(W, 0, sizeof(double) * 3 * (size_t)n, c->stream));
  k_energy_w<<<nblk(n, 128), 128, 0, c->stream>>>(n, c->x, u, c->infront, c->gi, c->gb, c->gii,
                                                  c->gbb, c->p.deriv_order, W, ell);
  k_energy_grad<<<nblk(n, 128), 128, 0, c->stream>>>(
      n, c->x, u, c->infront, c->behind, c->gi, c->gb, c->gii, c->gbb, W, ell, c->p.deriv_order,
      c->p.quant_circ, eterm, ubar, c->adj_xb, c->adj_gib, c->adj_gbb, c->adj_giib, c->adj_gbbb);
  k_ghost_vjp<<<nblk(n, 256), 256, 0, c->stream>>>(n, c->infront, c->behind, c->adj_xb,
                                                   c->adj_gib, c->adj_gbb, c->adj_giib,
                                                   c->adj_gbbb, xbar);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 3);
  std::vector<double> h(n);
  QV_CUDA(c, cudaMemcpyAsync(h.data(), eterm, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  QV_CUDA(c, cudaFree(W));
  // Neumaier-compensated sum of the per-point terms: the energy of a loss is
  // differenced across nearby states, and a plain sequential sum's rounding
  // (up to n u sum|t|) would dominate a difference quotient at small steps;
  // qv_energy keeps the reference's sequential order
  double e = 0., comp = 0.;
  for (int i = 0; i < n; i++) {
    const double t = e + h[i];
    comp += fabs(e) >= fabs(h[i]) ? (e - t) + h[i] : (h[i] - t) + e;
    e = t;
  }
  *energy = (e + comp) * c->p.quant_circ;
  return QV_OK;
}

int qv_pack_sources64(qv_ctx *c);

extern "C" int qv_field_velocity(qv_ctx *c, int m, const double *pts, int grad_images, double *u,
                                 double *dudx) {
  if (!c || m < 0 || (m > 0 && (!pts || !u || !dudx))) return QV_ERR_ARG;
  if (m == 0) return QV_OK;
  int rc;
  if (!c->ghosts_valid)
    if ((rc = qv_launch_ghosts(c))) return rc;
  if ((rc = qv_compact_active(c))) return rc;
  if ((rc = qv_pack_sources64(c))) return rc;
  double *dp = nullptr;
  QV_CUDA(c, cudaMalloc((void **)&dp, sizeof(double) * 15 * (size_t)m));
  QV_CUDA(c, cudaMemcpyAsync(dp, pts, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, c->stream));
  double *du = dp + 3 * (size_t)m, *dj = dp + 6 * (size_t)m;
  int nb = nblk(m, 64);
  switch (c->p.boundary) {
    case QV_BC_OPEN: k_field<QV_BC_OPEN><<<nb, 64, 0, c->stream>>>(m, dp, grad_images, c->n_act, c->src64, c->p.quant_circ, c->p.box_size, du, dj); break;
    case QV_BC_PERIODIC: k_field<QV_BC_PERIODIC><<<nb, 64, 0, c->stream>>>(m, dp, grad_images, c->n_act, c->src64, c->p.quant_circ, c->p.box_size, du, dj); break;
    case QV_BC_OPENX: k_field<QV_BC_OPENX><<<nb, 64, 0, c->stream>>>(m, dp, grad_images, c->n_act, c->src64, c->p.quant_circ, c->p.box_size, du, dj); break;
    case QV_BC_OPENXY: k_field<QV_BC_OPENXY><<<nb, 64, 0, c->stream>>>(m, dp, grad_images, c->n_act, c->src64, c->p.quant_circ, c->p.box_size, du, dj); break;
    default: cudaFree(dp); return qv_fail(c, QV_ERR_UNSUPPORTED, "boundary %d", c->p.boundary);
  }
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  QV_CUDA(c, cudaMemcpyAsync(u, du, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaMemcpyAsync(dudx, dj, sizeof(double) * 9 * m, cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  QV_CUDA(c, cudaFree(dp));
  return QV_OK;
}

extern "C" int qv_velocity_device(qv_ctx *c, double *u_out) {
  if (!c || !u_out) return QV_ERR_ARG;
  int rc = qv_velocity(c, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  if (c->n)
    QV_CUDA(c, cudaMemcpyAsync(u_out, c->u, sizeof(double) * 3 * (size_t)c->n,
                               cudaMemcpyDeviceToDevice, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  return QV_OK;
}
