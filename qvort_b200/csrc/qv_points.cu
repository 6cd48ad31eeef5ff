// qv_points.cu -- per-point O(N) kernels: ghost gather, LIA local term, the
// Adams-Bashforth ladder, the RK3 stages, the periodic wrap and the energy.
// All HBM-bound; one thread per slot, interleaved xyz loads.
#include <cstdarg>
#include <cstdio>

#include "qv_internal.cuh"
#include "qv_ab.cuh"
#include "qv_lia.cuh"

int qv_fail(qv_ctx *c, int code, const char *fmt, ...) {
  if (c) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->err, sizeof(c->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

int qv_grow(qv_ctx *c, void **ptr, size_t bytes) {
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  if (bytes == 0) return QV_OK;
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    cudaGetLastError();
    return qv_fail(c, QV_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  return QV_OK;
}

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------- ghosts
// get_ghost_p, src/periodic.f90:23-165: positions of the +-1 and +-2
// neighbours, shifted by +-L on every periodic axis where they differ from
// x_i by more than L/2 (strict comparisons).
__global__ void k_ghosts(int n, const double *__restrict__ x, const int *__restrict__ inf,
                         const int *__restrict__ beh, double *gi, double *gb, double *gii,
                         double *gbb, int lo_axis, double L) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int a = inf[i];
  if (a == 0) return;
  int b = beh[i];
  int aa = inf[a - 1], bb = beh[b - 1];
  int src[4] = {a - 1, b - 1, aa - 1, bb - 1};
  double *dst[4] = {gi, gb, gii, gbb};
  double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  double h = L / 2.;
#pragma unroll
  for (int k = 0; k < 4; k++) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double g = x[3 * src[k] + c];
      if (c >= lo_axis) {
        if ((xi[c] - g) > h)
          g = g + L;
        else if ((xi[c] - g) < (-h))
          g = g - L;
      }
      dst[k][3 * i + c] = g;
    }
  }
}

static int lo_axis_of(int bc) {
  return bc == QV_BC_PERIODIC ? 0 : bc == QV_BC_OPENX ? 1 : bc == QV_BC_OPENXY ? 2 : 3;
}

int qv_launch_ghosts(qv_ctx *c) {
  if (c->n == 0) return QV_OK;
  k_ghosts<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->x, c->infront, c->behind, c->gi,
                                                   c->gb, c->gii, c->gbb,
                                                   lo_axis_of(c->p.boundary), c->p.box_size);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  c->ghosts_valid = true;
  c->ghosts_stored = true;
  return QV_OK;
}

// ---------------------------------------------------------------- LIA
__device__ __forceinline__ double ddist(const double *a, const double *b) { return lia_dist(a, b); }

__device__ __forceinline__ void derivs(int order, const double *x, const double *gi,
                                       const double *gb, const double *gii, const double *gbb,
                                       double *s1, double *s2) {
  lia_derivs(order, x, gi, gb, gii, gbb, s1, s2);
}

// Local term of calc_velocity: LIA arm (src/timestep.f90:196-217) or the
// local part of the BS/Tree arms (src/timestep.f90:221-225, 270-274).  The
// log term stays FP64.  Writes u_li; for velocity LIA/Off also u.
__global__ void k_lia(int n, const double *__restrict__ x, const int *__restrict__ inf,
                      const double *__restrict__ gi, const double *__restrict__ gb,
                      const double *__restrict__ gii, const double *__restrict__ gbb,
                      double *u_li, double *u, int velocity, int order, int fixed_beta,
                      double quant_circ, double corea) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (inf[i] == 0) return;
  double X[3], GI[3], GB[3], GII[3], GBB[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    X[c] = x[3 * i + c]; GI[c] = gi[3 * i + c]; GB[c] = gb[3 * i + c];
    GII[c] = gii[3 * i + c]; GBB[c] = gbb[3 * i + c];
  }
  double out[3];
  lia_term(velocity, order, fixed_beta, quant_circ, corea, X, GI, GB, GII, GBB, out);
#pragma unroll
  for (int c = 0; c < 3; c++) u_li[3 * i + c] = out[c];
  if (velocity == QV_VEL_LIA || velocity == QV_VEL_OFF)
#pragma unroll
    for (int c = 0; c < 3; c++) u[3 * i + c] = out[c];
}

int qv_launch_lia(qv_ctx *c) {
  if (c->n == 0) return QV_OK;
  k_lia<<<nblk(c->n, 128), 128, 0, c->stream>>>(
      c->n, c->x, c->infront, c->gi, c->gb, c->gii, c->gbb, c->u_li, c->u, c->p.velocity,
      c->p.deriv_order, c->p.fixed_lia_beta, c->p.quant_circ, c->p.corea);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

// ---------------------------------------------------------------- AB ladder
// pmotion, src/timestep.f90:48-71.  The rung is picked per point by exact
// zero tests on the history; products and sums are rounded one at a time
// (no FMA) in the reference's evaluation order, so given the same velocities
// the positions agree bit for bit with the reference arithmetic.
__global__ void k_ab(int n, double dt, double *x, const double *__restrict__ u, double *u1,
                     double *u2, double *u3, const int *__restrict__ inf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (inf[i] == 0) return;
  double X[3], U[3], U1[3], U2[3], U3[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    X[c] = x[3 * i + c]; U[c] = u[3 * i + c]; U1[c] = u1[3 * i + c];
    U2[c] = u2[3 * i + c]; U3[c] = u3[3 * i + c];
  }
  const int rung = ab_rung(U1, U2, U3);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    x[3 * i + c] = ab_update(rung, dt, X[c], U[c], U1[c], U2[c], U3[c]);
    u3[3 * i + c] = U2[c];
    u2[3 * i + c] = U1[c];
    u1[3 * i + c] = U[c];
  }
}

int qv_launch_ab(qv_ctx *c) {
  if (c->n == 0) return QV_OK;
  k_ab<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->p.dt, c->x, c->u, c->u1, c->u2,
                                               c->u3, c->infront);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

// ---------------------------------------------------------------- RK3
// pmotion_RK3 stage updates, src/timestep.f90:105-175 (u1 is the RK register).
__global__ void k_rk3(int n, int stage, double dt, double *x, const double *__restrict__ u,
                      double *u1, const int *__restrict__ inf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (inf[i] == 0) return;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double uu = u[3 * i + c], q = u1[3 * i + c], xx = x[3 * i + c];
    if (stage == 0) {
      q = __dmul_rn(uu, dt);
      xx = __dadd_rn(xx, __ddiv_rn(q, 3.));
    } else if (stage == 1) {
      q = __dadd_rn(__dmul_rn(-(2. / 3.), q), __dmul_rn(uu, dt));
      xx = __dadd_rn(xx, q);
    } else {
      q = __dadd_rn(-q, __dmul_rn(uu, dt));
      xx = __dadd_rn(xx, __dmul_rn(0.5, q));
    }
    u1[3 * i + c] = q;
    x[3 * i + c] = xx;
  }
}

int qv_launch_rk3_stage(qv_ctx *c, int stage) {
  if (c->n == 0) return QV_OK;
  k_rk3<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, stage, c->p.dt, c->x, c->u, c->u1,
                                                c->infront);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

// ---------------------------------------------------------------- wrap
// enforce_periodic, src/periodic.f90:188-214 (and its yz / z variants).
// enforce_periodic (src/periodic.f90:188-214) on the axes lo_axis..2, and the
// end-of-step NaN test of NAN_finder (src/general.f90:253-280, called at
// src/run.f90:168): a NaN in any coordinate of any slot below n, empty slots
// included, sets QV_STAT_NAN.  lo_axis = 3 (open boundaries): the test only.
__global__ void k_wrap(int n, double *x, const int *__restrict__ inf, int lo_axis, double L,
                       int *status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool nan = i < n && (isnan(x[3 * i]) || isnan(x[3 * i + 1]) || isnan(x[3 * i + 2]));
  if (__any_sync(0xffffffffu, nan) && (threadIdx.x & 31) == 0) atomicOr(status, QV_STAT_NAN);
  if (i >= n) return;
  if (inf[i] == 0) return;
  double h = L / 2.;
  for (int c = lo_axis; c < 3; c++) {
    double v = x[3 * i + c];
    if (v > h)
      x[3 * i + c] = v - L;
    else if (v < (-h))
      x[3 * i + c] = v + L;
  }
}

int qv_launch_wrap(qv_ctx *c) {
  int lo = lo_axis_of(c->p.boundary);
  if (c->n == 0) return QV_OK;
  k_wrap<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->x, c->infront, std::min(lo, 3),
                                                 c->p.box_size, c->dstatus);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

// ---------------------------------------------------------------- energy
// energy_info, src/diagnostic.f90:259-280.  Per-point terms in parallel, then
// a fixed-order two-level sum (deterministic).
__global__ void k_energy_terms(int n, const double *__restrict__ x, const double *__restrict__ u,
                               const int *__restrict__ inf, const double *__restrict__ gi,
                               const double *__restrict__ gb, const double *__restrict__ gii,
                               const double *__restrict__ gbb, int order, double *blk_out) {
  __shared__ double red[256];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.;
  if (i < n && inf[i] != 0) {
    int a = inf[i] - 1;
    double s1[3], s2[3], t1[3], t2[3];
    const int idx[2] = {i, a};
    double dots[2];
    for (int q = 0; q < 2; q++) {
      int k = idx[q];
      double X[3], GI[3], GB[3], GII[3], GBB[3];
      for (int c = 0; c < 3; c++) {
        X[c] = x[3 * k + c]; GI[c] = gi[3 * k + c]; GB[c] = gb[3 * k + c];
        GII[c] = gii[3 * k + c]; GBB[c] = gbb[3 * k + c];
      }
      derivs(order, X, GI, GB, GII, GBB, s1, s2);
      t1[0] = X[1] * s1[2] - X[2] * s1[1];
      t1[1] = X[2] * s1[0] - X[0] * s1[2];
      t1[2] = X[0] * s1[1] - X[1] * s1[0];
      dots[q] = u[3 * k] * t1[0] + u[3 * k + 1] * t1[1] + u[3 * k + 2] * t1[2];
      (void)t2;
    }
    double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    double g[3] = {gi[3 * i], gi[3 * i + 1], gi[3 * i + 2]};
    e = 0.5 * ddist(xi, g) * (dots[0] + dots[1]);
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) blk_out[blockIdx.x] = red[0];
}

__global__ void k_energy_final(int nb, const double *blk, double *out, double quant_circ) {
  __shared__ double red[256];
  double s = 0.;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) s += blk[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int t = blockDim.x / 2; t > 0; t >>= 1) {
    if (threadIdx.x < t) red[threadIdx.x] += red[threadIdx.x + t];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] * quant_circ;
}

int qv_launch_energy(qv_ctx *c, double *out_host) {
  int nb = nblk(c->n, 256);
  double *blk = nullptr;  // energy is a diagnostic, off the step path
  QV_CUDA(c, cudaMalloc((void **)&blk, sizeof(double) * (nb + 1)));
  k_energy_terms<<<nb, 256, 0, c->stream>>>(c->n, c->x, c->u, c->infront, c->gi, c->gb, c->gii,
                                            c->gbb, c->p.deriv_order, blk);
  k_energy_final<<<1, 256, 0, c->stream>>>(nb, blk, blk + nb, c->p.quant_circ);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 2);
  QV_CUDA(c, cudaMemcpyAsync(out_host, blk + nb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  QV_CUDA(c, cudaFree(blk));
  return QV_OK;
}
