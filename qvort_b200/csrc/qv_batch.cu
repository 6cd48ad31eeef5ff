// qv_batch.cu -- many independent filament systems advanced together.
//
// Each system is what one run of the reference's time loop would hold (its own
// f(:), links, dt, velocity method; open boundaries, box of side box_size
// centred on the origin of its own coordinates): calc_velocity
// (src/timestep.f90:180-309, BS arm = direct sum, Tree arm = Barnes-Hut walk
// of its own octree, src/tree.f90:44-186, 336-421) then pmotion's
// Adams-Bashforth ladder (src/timestep.f90:48-71).  The reference runs one
// system per process; this file runs all of them in one pass per step:
//
//   ghosts + LIA over all points (one launch each)
//   the octrees of all Barnes-Hut systems as one forest (qv_forest_build)
//   the FP32 source pack of the direct systems
//   ONE persistent work kernel over a cost-ordered list of warp items:
//     walk items   (32 targets of a Barnes-Hut system x one root child)
//     direct items (32 targets of a direct system x one source chunk)
//   one kernel that adds each point's partial sums in a fixed order and
//   applies the AB update with the system's own dt
//
// The step contains no host synchronisation, so it is captured once as a CUDA
// graph and replayed.  Every target's arithmetic is the same sequence of
// operations as in a single-system context (the walk visits the same nodes in
// the same order, the direct sum uses the same source chunks, the partial
// sums are added in the same order), so a batched step reproduces per-system
// runs bit for bit; how items are scheduled changes nothing but time, which
// is what the autotuner (qv_batch_tune) searches over.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "qv_walk.cuh"

namespace cg = cooperative_groups;

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

#define BSPLIT 8   // walk items per target group: the root's children
#define BDT 128    // source tile of the single-system direct kernel (chunk rounding)

// status bits
#define BST_SINGULAR 1
#define BST_STACK 2
#define BST_TREE 4

struct BatchArgs {
  int ntot, nitems, nroots, cap_pts, stk_cap;
  const int4 *items;    // (x: sub-item, y: group or system, z: first target slot, w: unused)
  const int4 *groups;   // walk group: (first perm position, targets, root node, system)
  const int4 *sys;      // (first slot, slots, method, chunks)
  const int2 *dsrc;     // direct system: (first pack position, chunk length)
  const int *ctl, *perm;
  const double *x;
  const int *inf, *beh;
  const WNode64 *w64;
  const WNode32 *w32;
  const WPay32 *p32;
  const float *src32;
  double theta;
  int extra;
  double *partw, *partd;
  int *counter, *status;
  unsigned long long *evals, *evals_far;
};

// ---------------------------------------------------------------- walk item
// One warp, 32 targets of one system (adjacent in its tree's depth-first
// order), the unshifted image restricted to root child sl: the same task as
// the single-system mixed walk (its main image, without periodic images).
__device__ __forceinline__ void walk_item(const BatchArgs &a, StkEnt *st, int g, int sl,
                                          const int *perm, unsigned &ev, unsigned &evf,
                                          bool &bad) {
  const int lane = threadIdx.x & 31;
  const int4 G = a.groups[g];
  const int q = G.x + lane;
  const bool live = lane < G.y;
  const int i = live ? perm[q] : 0;
  double xi[3] = {0., 0., 0.};
  int bi = -1, fi = -1, ii = -1;
  if (live) {
    xi[0] = a.x[3 * i]; xi[1] = a.x[3 * i + 1]; xi[2] = a.x[3 * i + 2];
    bi = a.beh[i]; fi = a.inf[i]; ii = i + 1;
  }
  Kahan3w k0;
  k0.zero();
  const double s[3] = {0., 0., 0.};
  float th[3], tl[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double t = xi[c] - s[c];
    th[c] = __double2float_rn(t);
    tl[c] = __double2float_rn(t - (double)th[c]);
  }
  int top = 0;
  {
    const int root = G.z;
    const WNode64 r = a.w64[root];
    bool ropen = false;
    if (r.count == 1) {
      const unsigned live_mask = __ballot_sync(0xffffffffu, live);
      if (sl == 0 && lane == 0) {
        st[0].h = a.w32[root];
        st[0].node = root;
        st[0].mask = live_mask;
      }
      top = (sl == 0 && live_mask) ? 1 : 0;
    } else {
      if (live) {
        ropen = exact_open(exact_dist(xi, r, s), r, a.theta, a.extra);
        if (!ropen && sl == 0) { ev++; evf++; }  // root far field: zero moments
      }
      const unsigned om = __ballot_sync(0xffffffffu, ropen);
      if (om && sl < r.nchild) {
        if (lane == 0) {
          st[0].h = a.w32[r.child_first + sl];
          st[0].node = r.child_first + sl;
          st[0].mask = om;
        }
        top = 1;
      }
    }
  }
  __syncwarp();
  while (top > 0) {
    top--;
    const WNode32 h = st[top].h;
    const int node = st[top].node;
    const bool in = (st[top].mask >> lane) & 1u;
    __syncwarp();
    float v0 = (th[0] - h.ch[0]) + (tl[0] - h.cl[0]);
    float v1 = (th[1] - h.ch[1]) + (tl[1] - h.cl[1]);
    float v2 = (th[2] - h.ch[2]) + (tl[2] - h.cl[2]);
    float d2 = fmaf(v0, v0, fmaf(v1, v1, v2 * v2));
    if (h.count == 1) {
      if (in) {
        int j = h.jb;
        if (j != ii && j != bi && j != fi) {
          bool sing = false;
          if (d2 < 1e-20f) {
            double dist = exact_dist(xi, a.w64[node], s);
            sing = dist < QV_DEPS;
          }
          if (sing) {
            bad = true;
          } else {
            const WPay32 &P = a.p32[node];
            float r2x = (P.a[0] - th[0]) + (P.b[0] - tl[0]);
            float r2y = (P.a[1] - th[1]) + (P.b[1] - tl[1]);
            float r2z = (P.a[2] - th[2]) + (P.b[2] - tl[2]);
            float ox, oy, oz;
            qv_seg32(-v0, -v1, -v2, r2x, r2y, r2z, P.C[0], P.C[1], P.C[2], d2, ox, oy, oz);
            k0.add(ox, oy, oz);
            ev++;
          }
        }
      }
    } else {
      // one predicate (far) guards the far-field term, as in the single walk
      const bool amb = in && !(h.rhi > 0.f && (d2 > h.rhi || d2 < h.rlo));
      bool open = in && d2 < h.rlo;
      if (amb) {
        const WNode64 h64 = a.w64[node];
        open = exact_open(exact_dist(xi, h64, s), h64, a.theta, a.extra);
      }
      const bool far = in && !open;
      ev += far ? 1u : 0u;
      evf += far ? 1u : 0u;
      if (far && node >= a.nroots) {  // a root's moments are zero
        const WPay32 &P = a.p32[node];
        float rd = rsqrtf(d2);
        float rd2 = rd * rd, rd3 = rd2 * rd, rd5 = rd3 * rd2;
        float z0 = fmaf(v0, P.C[0], fmaf(v1, P.C[3], v2 * P.C[6]));
        float z1 = fmaf(v0, P.C[1], fmaf(v1, P.C[4], v2 * P.C[7]));
        float z2 = fmaf(v0, P.C[2], fmaf(v1, P.C[5], v2 * P.C[8]));
        float cx = fmaf(P.a[1], v2, -P.a[2] * v1) - P.b[0];
        float cy = fmaf(P.a[2], v0, -P.a[0] * v2) - P.b[1];
        float cz = fmaf(P.a[0], v1, -P.a[1] * v0) - P.b[2];
        float wx = fmaf(v1, z2, -v2 * z1);
        float wy = fmaf(v2, z0, -v0 * z2);
        float wz = fmaf(v0, z1, -v1 * z0);
        float t5 = 3.f * rd5;
        k0.add(fmaf(cx, rd3, wx * t5), fmaf(cy, rd3, wy * t5), fmaf(cz, rd3, wz * t5));
      }
      unsigned om = __ballot_sync(0xffffffffu, open);
      if (om) {
        int nc = h.nchild;
        if (top + nc > a.stk_cap) {  // deeper than the captured stack: flagged, step skipped
          if (lane == 0) atomicOr(a.status, BST_STACK);
          nc = 0;
        }
        if (lane < nc) {
          int ch = h.child_first + nc - 1 - lane;
          StkEnt &E = st[top + lane];
          E.h = a.w32[ch];
          E.node = ch;
          E.mask = om;
        }
        top += nc;
      }
      __syncwarp();
    }
  }
  if (live) {
    double *o = a.partw + ((size_t)sl * a.ntot + i) * 3;
    o[0] = k0.get(0); o[1] = k0.get(1); o[2] = k0.get(2);
  }
}

// -------------------------------------------------------------- direct item
// One warp, 32 consecutive targets of one system, the sources of one chunk
// (the chunking of the single-system direct kernel), staged 32 at a time in
// the warp's shared memory; per target the same sequence of pair terms and
// compensated sums as the single-system kernel's unshifted sum.
__device__ __forceinline__ void direct_item(const BatchArgs &a, float4 *tile, int s, int chunk,
                                            int t0) {
  const int lane = threadIdx.x & 31;
  const int4 S = a.sys[s];
  const int2 D = a.dsrc[s];
  const int i = t0 + lane;
  const bool live = i < S.x + S.y;
  double xi[3] = {0., 0., 0.};
  int bi = -1, ii = -1;
  if (live) {
    xi[0] = a.x[3 * i]; xi[1] = a.x[3 * i + 1]; xi[2] = a.x[3 * i + 2];
    bi = a.beh[i]; ii = i + 1;
  }
  float th[3], tl[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    th[c] = __double2float_rn(xi[c]);
    tl[c] = __double2float_rn(xi[c] - (double)th[c]);
  }
  Kahan3w k0;
  k0.zero();
  const int j0 = chunk * D.y, j1 = min(S.y, j0 + D.y);
  const float4 *src4 = reinterpret_cast<const float4 *>(a.src32) + 4 * (size_t)D.x;
  for (int t = j0; t < j1; t += 32) {
    const int m = min(32, j1 - t);
    __syncwarp();
    if (lane < m) {
      const float4 *g = src4 + 4 * (size_t)(t + lane);
      tile[4 * lane] = g[0];
      tile[4 * lane + 1] = g[1];
      tile[4 * lane + 2] = g[2];
      tile[4 * lane + 3] = g[3];
    }
    __syncwarp();
    if (live) {
      for (int k = 0; k < m; k++) {
        float4 A = tile[4 * k], B = tile[4 * k + 1], Cc = tile[4 * k + 2], Dd = tile[4 * k + 3];
        int jj = __float_as_int(Dd.x);
        if (jj == bi || jj == ii) continue;
        float r1x = (A.x - th[0]) + (A.w - tl[0]);
        float r1y = (A.y - th[1]) + (B.x - tl[1]);
        float r1z = (A.z - th[2]) + (B.y - tl[2]);
        float r2x = (B.z - th[0]) + (Cc.y - tl[0]);
        float r2y = (B.w - th[1]) + (Cc.z - tl[1]);
        float r2z = (Cc.x - th[2]) + (Cc.w - tl[2]);
        float ox, oy, oz;
        float r1s = fmaf(r1x, r1x, fmaf(r1y, r1y, r1z * r1z));
        qv_seg32(r1x, r1y, r1z, r2x, r2y, r2z, Dd.y, Dd.z, Dd.w, r1s, ox, oy, oz);
        k0.add(ox, oy, oz);
      }
    }
  }
  if (live) {
    double *o = a.partd + ((size_t)chunk * a.ntot + i) * 3;
    o[0] = k0.get(0); o[1] = k0.get(1); o[2] = k0.get(2);
  }
}

// ---------------------------------------------------------- work items
// Each warp takes the next item from a global counter until the list is
// exhausted; the list is ordered by estimated cost, largest first.
__device__ __forceinline__ void batch_items(const BatchArgs &a) {
  extern __shared__ __align__(16) unsigned char bsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const size_t per_warp = (size_t)max(a.stk_cap * (int)sizeof(StkEnt), 32 * 4 * (int)sizeof(float4));
  unsigned char *mine = bsm + per_warp * wid;
  const int *perm = a.nroots > 0 ? a.perm : nullptr;
  unsigned ev = 0, evf = 0;  // per warp: far below 2^32
  bool bad = false;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(a.counter, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= a.nitems) break;
    const int4 W = a.items[it];
    if (W.x < BSPLIT)
      walk_item(a, reinterpret_cast<StkEnt *>(mine), W.y, W.x, perm, ev, evf, bad);
    else
      direct_item(a, reinterpret_cast<float4 *>(mine), W.y, W.x - BSPLIT, W.z);
  }
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_down_sync(0xffffffffu, ev, o);
    evf += __shfl_down_sync(0xffffffffu, evf, o);
  }
  if (lane == 0 && ev) atomicAdd(a.evals, (unsigned long long)ev);
  if (lane == 0 && evf) atomicAdd(a.evals_far, (unsigned long long)evf);
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.status, BST_SINGULAR);
}

// ------------------------------------------------------------ update kernel
// Per point: the non-local velocity from its partial sums in the
// single-system reduce order (walk: root children 0..7; direct: chunks in
// order; no images under open boundaries), u = u_LI + u_BS, then, when
// do_ab, the AB ladder of pmotion with the system's dt (the arithmetic of
// k_ab: exact-zero rung tests, products and sums rounded one at a time).
struct UpdateArgs {
  int ntot, do_ab;
  const int *sysof;
  const double *dts, *u_li;
  double gfac_w, gfac_d;
  double *x, *u, *u_bs, *u1, *u2, *u3;
  int *done;  // steps applied (counted on the device)
};

__device__ __forceinline__ void batch_update_point(const BatchArgs &a, const UpdateArgs &b, int i) {
  const int ntot = b.ntot, do_ab = b.do_ab;
  const int *__restrict__ sysof = b.sysof;
  const int4 *__restrict__ sys = a.sys;
  const double *__restrict__ dts = b.dts, *__restrict__ u_li = b.u_li;
  const double *__restrict__ partw = a.partw, *__restrict__ partd = a.partd;
  const double gfac_w = b.gfac_w, gfac_d = b.gfac_d;
  double *x = b.x, *u = b.u, *u_bs = b.u_bs, *u1 = b.u1, *u2 = b.u2, *u3 = b.u3;
  if (a.inf[i] == 0) return;
  const int s = sysof[i];
  const int4 S = sys[s];
  double s0[3] = {0., 0., 0.}, s1[3] = {0., 0., 0.};
  double scale;
  if (S.z == QV_VEL_TREE) {
    for (int m = 0; m < BSPLIT; m++)
      for (int c = 0; c < 3; c++) s0[c] += partw[((size_t)m * ntot + i) * 3 + c];
    scale = gfac_w;
  } else {
    for (int k = 0; k < S.w; k++)
      for (int c = 0; c < 3; c++) s0[c] += partd[((size_t)k * ntot + i) * 3 + c];
    scale = gfac_d;
  }
  double U[3];
  for (int c = 0; c < 3; c++) {
    double b0 = s0[c] * scale, b1 = s1[c] * scale;
    u_bs[3 * i + c] = b0 + b1;
    U[c] = (u_li[3 * i + c] + b0) + b1;
    u[3 * i + c] = U[c];
  }
  if (!do_ab) return;
  const double dt = dts[s];
  double X[3], U1[3], U2[3], U3[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    X[c] = x[3 * i + c]; U1[c] = u1[3 * i + c]; U2[c] = u2[3 * i + c]; U3[c] = u3[3 * i + c];
  }
  bool z1 = fabs(U1[0]) == 0 && fabs(U1[1]) == 0 && fabs(U1[2]) == 0;
  bool z2 = fabs(U2[0]) == 0 && fabs(U2[1]) == 0 && fabs(U2[2]) == 0;
  bool z3 = fabs(U3[0]) == 0 && fabs(U3[1]) == 0 && fabs(U3[2]) == 0;
  const double three_twos = 3. / 2., one_half = 1. / 2., c23_12 = 23. / 12.,
               c4_3 = 4. / 3., c5_12 = 5. / 12.;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double r;
    if (z1) {
      r = __dadd_rn(X[c], __dmul_rn(dt, U[c]));
    } else if (z2) {
      r = __dadd_rn(X[c], __dmul_rn(__dmul_rn(three_twos, dt), U[c]));
      r = __dsub_rn(r, __dmul_rn(__dmul_rn(one_half, dt), U1[c]));
    } else if (z3) {
      r = __dadd_rn(X[c], __dmul_rn(__dmul_rn(c23_12, dt), U[c]));
      r = __dsub_rn(r, __dmul_rn(__dmul_rn(c4_3, dt), U1[c]));
      r = __dadd_rn(r, __dmul_rn(__dmul_rn(c5_12, dt), U2[c]));
    } else {
      double sm = __dsub_rn(__dmul_rn(55., U[c]), __dmul_rn(59., U1[c]));
      sm = __dadd_rn(sm, __dmul_rn(37., U2[c]));
      sm = __dsub_rn(sm, __dmul_rn(9., U3[c]));
      r = __dadd_rn(X[c], __ddiv_rn(__dmul_rn(dt, sm), 24.));
    }
    x[3 * i + c] = r;
    u3[3 * i + c] = U2[c];
    u2[3 * i + c] = U1[c];
    u1[3 * i + c] = U[c];
  }
}

// FP32 source pack of the direct systems' slots (k_pack_sources' FP32 half):
// x hi/lo, ghosti hi/lo, slot, s = ghosti - x.
__device__ __forceinline__ void batch_pack_point(int q, const int *__restrict__ dact,
                                                 const double *__restrict__ x,
                                                 const double *__restrict__ gi, float *s32) {
  int j = dact[q];
  double X[3], G[3];
#pragma unroll
  for (int k = 0; k < 3; k++) { X[k] = x[3 * j + k]; G[k] = gi[3 * j + k]; }
  double e0 = G[0] - X[0], e1 = G[1] - X[1], e2 = G[2] - X[2];
  float *f = s32 + 16 * (size_t)q;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float h = __double2float_rn(X[k]);
    f[k] = h;
    f[3 + k] = __double2float_rn(X[k] - (double)h);
    float g = __double2float_rn(G[k]);
    f[6 + k] = g;
    f[9 + k] = __double2float_rn(G[k] - (double)g);
  }
  f[12] = __int_as_float(j + 1);
  f[13] = __double2float_rn(e0);
  f[14] = __double2float_rn(e1);
  f[15] = __double2float_rn(e2);
}

struct PackArgsB {
  int nd;
  const int *dact;
  const double *gi;
  float *s32;
};

// ------------------------------------------------------------ the step
// One cooperative launch after the forest build: the FP32 source pack of the
// direct systems; a grid barrier; the work items; a grid barrier; per point the
// non-local velocity from its partial sums and, when do_ab, the AB update, and
// the count of applied steps.  The barriers replace three kernel boundaries
// (the pack, the items and the update used to be separate launches with the
// same order).  Nothing is updated when any status bit is set (a forest or
// stack overflow makes the host resize and run the step again).  Ghosts and
// LIA stay separate launches before the forest build: the forest's moments
// need the ghosts, and LIA keeps the single-system kernel's arithmetic (its
// file is compiled without FMA contraction).
__global__ void k_batch_step(BatchArgs a, UpdateArgs ub, PackArgsB pb) {
  cg::grid_group grid = cg::this_grid();
  const int nthreads = gridDim.x * blockDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const bool overflow = a.nroots > 0 && a.ctl[QV_CTL_OVERFLOW];
  if (gt == 0) {
    *a.evals = 0;
    *a.evals_far = 0;
    if (overflow) atomicOr(a.status, BST_TREE);
  }
  for (int q = gt; q < pb.nd; q += nthreads) batch_pack_point(q, pb.dact, a.x, pb.gi, pb.s32);
  grid.sync();
  if (*a.status == 0) batch_items(a);
  grid.sync();
  if (gt == 0) *a.counter = 0;  // every fetch is done: ready for the next step
  if (*a.status) return;
  for (int i = gt; i < ub.ntot; i += nthreads) batch_update_point(a, ub, i);
  if (gt == 0 && ub.do_ab) atomicAdd(ub.done, 1);
}

// ================================================================ host side
struct qv_batch {
  qv_ctx *c = nullptr;
  int nsys = 0, ntot = 0;
  std::vector<int> off, meth, nchunk, clen;
  std::vector<double> dt;
  int nroots = 0, n_fact = 0, nd = 0, max_chunks = 1, ngroups = 0;
  // device tables
  int *d_sysof = nullptr, *d_dact = nullptr, *d_fact = nullptr, *d_froot = nullptr;
  int *d_nfact = nullptr, *d_counter = nullptr, *d_status = nullptr, *d_done = nullptr;
  int4 *d_sys = nullptr, *d_roots = nullptr, *d_groups = nullptr, *d_items = nullptr;
  int2 *d_dsrc = nullptr;
  double *d_dt = nullptr, *d_part = nullptr;
  float *d_src32 = nullptr;
  size_t part_slots = 0;
  std::vector<int4> items, items_cost;  // natural and cost-descending orders
  int cap_nodes = 0, stk_cap = 0, depth = 0;
  bool points_set = false;
  // launch configuration of the work kernel (qv_batch_tune)
  int wpb = 4, bps = 2, order = 1;
  cudaGraphExec_t gexec = nullptr;
  bool graph_tried = false, graph_ok = false;
  long long steps_done = 0;
};

static void free_batch_tables(qv_batch *b) {
  void *ptrs[] = {b->d_sysof, b->d_dact, b->d_fact, b->d_froot, b->d_nfact, b->d_counter,
                  b->d_status, b->d_done, b->d_sys, b->d_roots, b->d_groups, b->d_items,
                  b->d_dsrc, b->d_dt, b->d_part, b->d_src32};
  for (void *p : ptrs)
    if (p) cudaFree(p);
}

template <typename T>
static int upload(qv_ctx *c, T **dst, const std::vector<T> &v) {
  size_t bytes = sizeof(T) * std::max<size_t>(v.size(), 1);
  QV_CUDA(c, cudaMalloc((void **)dst, bytes));
  if (!v.empty())
    QV_CUDA(c, cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return QV_OK;
}

static size_t work_smem_per_warp(const qv_batch *b) {
  return std::max(b->stk_cap * sizeof(StkEnt), (size_t)(32 * 4 * sizeof(float4)));
}

static void drop_graph(qv_batch *b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->graph_tried = false;
  b->graph_ok = false;
}

static BatchArgs work_args(qv_batch *b) {
  qv_ctx *c = b->c;
  TreeBuf &t = c->tree;
  BatchArgs a;
  a.ntot = b->ntot;
  a.nitems = (int)b->items.size();
  a.nroots = b->nroots;
  a.cap_pts = t.cap_pts;
  a.stk_cap = b->stk_cap;
  a.items = b->d_items;
  a.groups = b->d_groups;
  a.sys = b->d_sys;
  a.dsrc = b->d_dsrc;
  a.ctl = t.ctl;
  a.perm = t.permb;
  a.x = c->x;
  a.inf = c->infront;
  a.beh = c->behind;
  a.w64 = t.w64;
  a.w32 = t.w32;
  a.p32 = t.p32;
  a.src32 = b->d_src32;
  a.theta = c->p.tree_theta;
  a.extra = c->p.tree_extra_correction;
  a.partw = b->d_part;
  a.partd = b->d_part;
  a.counter = b->d_counter;
  a.status = b->d_status;
  a.evals = c->evals;
  a.evals_far = c->evals_far;
  return a;
}

// The cooperative step kernel (pack, items, update) with the batch's launch
// shape; the tuner keeps that shape within what is resident at once.
static int launch_step(qv_batch *b, int do_ab) {
  qv_ctx *c = b->c;
  BatchArgs a = work_args(b);
  const qv_params &p = c->p;
  UpdateArgs ub;
  ub.ntot = b->ntot; ub.do_ab = do_ab; ub.sysof = b->d_sysof; ub.dts = b->d_dt; ub.u_li = c->u_li;
  ub.gfac_w = p.quant_circ / 4. / QV_PI; ub.gfac_d = p.quant_circ / (4. * QV_PI);
  ub.x = c->x; ub.u = c->u; ub.u_bs = c->u_bs; ub.u1 = c->u1; ub.u2 = c->u2; ub.u3 = c->u3;
  ub.done = b->d_done;
  PackArgsB pb;
  pb.nd = b->nd; pb.dact = b->d_dact; pb.gi = c->gi; pb.s32 = b->d_src32;
  size_t smem = work_smem_per_warp(b) * b->wpb;
  void *args[] = {&a, &ub, &pb};
  QV_CUDA(c, cudaLaunchCooperativeKernel((const void *)k_batch_step, dim3(b->bps * c->sm_count),
                                         dim3(b->wpb * 32), args, smem, c->stream));
  QV_COUNT(c, 1);
  return QV_OK;
}

// One step (or one velocity evaluation when do_ab is 0) on the context stream,
// with no host synchronisation: ghosts, LIA, the forest build, the step kernel.
static int enqueue_step(qv_batch *b, int do_ab) {
  qv_ctx *c = b->c;
  int rc;
  if ((rc = qv_launch_ghosts(c))) return rc;
  if ((rc = qv_launch_lia(c))) return rc;
  if (b->nroots > 0) {
    ForestArgs f;
    f.nroots = b->nroots; f.n_fact = b->n_fact; f.roots = b->d_roots; f.fact = b->d_fact;
    f.froot = b->d_froot; f.d_nfact = b->d_nfact;
    if ((rc = qv_forest_build(c, f))) return rc;
  }
  return launch_step(b, do_ab);
}

// Chunking of the single-system direct kernel for na active sources
// (qv_launch_direct): the batch reuses it so that every target sums the same
// source ranges in the same order.
static void direct_chunks(int na, int sm_count, int *nchunk, int *chunk_len) {
  int bx = nblk(na, BDT);
  int want = (4 * sm_count + bx - 1) / bx;
  int maxch = std::max(1, na / (4 * BDT));
  int nc = std::max(1, std::min(want, maxch));
  int cl = ((nblk(na, nc) + BDT - 1) / BDT) * BDT;
  *chunk_len = cl;
  *nchunk = nblk(na, cl);
}

extern "C" int qv_batch_create(const qv_params *p, int nsys, const int *offsets, const int *method,
                               const double *dt, void *stream, qv_batch **out) {
  if (!p || !out || nsys < 1 || !offsets || !method || !dt) return QV_ERR_ARG;
  *out = nullptr;
  if (p->boundary != QV_BC_OPEN || p->precision != QV_PREC_MIXED) return QV_ERR_UNSUPPORTED;
  if (offsets[0] != 0) return QV_ERR_ARG;
  for (int s = 0; s < nsys; s++) {
    if (offsets[s + 1] <= offsets[s]) return QV_ERR_ARG;
    if (method[s] != QV_VEL_BS && method[s] != QV_VEL_TREE) return QV_ERR_UNSUPPORTED;
    if (!(dt[s] > 0.)) return QV_ERR_ARG;
  }
  qv_params q = *p;
  q.velocity = QV_VEL_TREE;  // the local term of the BS and Tree arms (src/timestep.f90:223, 272)
  qv_ctx *c = nullptr;
  int rc = qv_create(&q, stream, &c);
  if (rc) return rc;
  qv_batch *b = new qv_batch();
  b->c = c;
  b->nsys = nsys;
  b->ntot = offsets[nsys];
  b->off.assign(offsets, offsets + nsys + 1);
  b->meth.assign(method, method + nsys);
  b->dt.assign(dt, dt + nsys);
  b->nchunk.assign(nsys, 0);
  b->clen.assign(nsys, 0);
  std::vector<int> sysof(b->ntot), dact, fact, froot;
  std::vector<int4> sys(nsys), roots, groups;
  std::vector<int2> dsrc(nsys, make_int2(0, 0));
  std::vector<double> cost;
  for (int s = 0; s < nsys; s++) {
    const int o = offsets[s], n = offsets[s + 1] - offsets[s];
    for (int i = o; i < o + n; i++) sysof[i] = s;
    if (method[s] == QV_VEL_BS) {
      int nc, cl;
      direct_chunks(n, c->sm_count, &nc, &cl);
      b->nchunk[s] = nc;
      b->clen[s] = cl;
      b->max_chunks = std::max(b->max_chunks, nc);
      dsrc[s] = make_int2((int)dact.size(), cl);
      for (int i = o; i < o + n; i++) dact.push_back(i);
      sys[s] = make_int4(o, n, QV_VEL_BS, nc);
      for (int k = 0; k < nc; k++)
        for (int t0 = o; t0 < o + n; t0 += 32) {
          b->items.push_back(make_int4(BSPLIT + k, s, t0, 0));
          int len = std::min(n, (k + 1) * cl) - k * cl;
          cost.push_back((double)std::min(32, o + n - t0) * len);
        }
    } else {
      const int r = (int)roots.size();
      roots.push_back(make_int4(o, n, (int)fact.size(), n));
      for (int q0 = 0; q0 < n; q0 += 32) {
        const int g = (int)groups.size();
        groups.push_back(make_int4((int)fact.size() + q0, std::min(32, n - q0), r, s));
        for (int sl = 0; sl < BSPLIT; sl++) {
          b->items.push_back(make_int4(sl, g, 0, 0));
          // a rough per-target walk cost: a few dozen cells per octave of N,
          // spread over the root's children
          cost.push_back((double)std::min(32, n - q0) * 40. * std::log2((double)n + 1.) / 4.);
        }
      }
      for (int i = o; i < o + n; i++) {
        fact.push_back(i);
        froot.push_back(r);
      }
      sys[s] = make_int4(o, n, QV_VEL_TREE, 0);
    }
  }
  b->nroots = (int)roots.size();
  b->n_fact = (int)fact.size();
  b->nd = (int)dact.size();
  b->ngroups = (int)groups.size();
  std::vector<int> idx(b->items.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int u, int v) { return cost[u] > cost[v]; });
  for (int k : idx) b->items_cost.push_back(b->items[k]);
  b->part_slots = (size_t)std::max(BSPLIT, b->max_chunks);
  std::vector<int> one(1, b->n_fact);
  if ((rc = upload(c, &b->d_sysof, sysof)) || (rc = upload(c, &b->d_sys, sys)) ||
      (rc = upload(c, &b->d_dsrc, dsrc)) || (rc = upload(c, &b->d_dt, b->dt)) ||
      (rc = upload(c, &b->d_dact, dact)) || (rc = upload(c, &b->d_fact, fact)) ||
      (rc = upload(c, &b->d_froot, froot)) || (rc = upload(c, &b->d_roots, roots)) ||
      (rc = upload(c, &b->d_groups, groups)) || (rc = upload(c, &b->d_items, b->items_cost)) ||
      (rc = upload(c, &b->d_nfact, one))) {
    free_batch_tables(b);
    qv_destroy(c);
    delete b;
    return rc;
  }
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_counter, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_done, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMalloc((void **)&b->d_part, sizeof(double) * 3 * b->part_slots * (size_t)b->ntot);
  if (e == cudaSuccess && b->nd > 0) e = cudaMalloc((void **)&b->d_src32, sizeof(float) * 16 * (size_t)b->nd);
  if (e == cudaSuccess) e = cudaMemset(b->d_status, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_done, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_counter, 0, sizeof(int));  // the step kernel resets it after use
  if (e != cudaSuccess) {
    cudaGetLastError();
    free_batch_tables(b);
    qv_destroy(c);
    delete b;
    return QV_ERR_NOMEM;
  }
  b->cap_nodes = 4 * std::max(b->n_fact, 1) + 64 * std::max(b->nroots, 1);
  *out = b;
  return QV_OK;
}

extern "C" void qv_batch_destroy(qv_batch *b) {
  if (!b) return;
  drop_graph(b);
  free_batch_tables(b);
  qv_destroy(b->c);
  delete b;
}

extern "C" const char *qv_batch_last_error(qv_batch *b) { return b ? b->c->err : "null batch"; }

// Tree depth of the current positions (an eager build read back on the host)
// and the walk stack that covers it with four levels to spare.
static int size_stack(qv_batch *b) {
  qv_ctx *c = b->c;
  if (b->nroots == 0) {
    b->stk_cap = 8;
    return QV_OK;
  }
  int rc;
  for (int attempt = 0; attempt < 8; attempt++) {
    if ((rc = qv_forest_reserve(c, b->n_fact, b->cap_nodes))) return rc;
    if ((rc = qv_launch_ghosts(c))) return rc;
    ForestArgs f;
    f.nroots = b->nroots; f.n_fact = b->n_fact; f.roots = b->d_roots; f.fact = b->d_fact;
    f.froot = b->d_froot; f.d_nfact = b->d_nfact;
    if ((rc = qv_forest_build(c, f))) return rc;
    int ctl[8];
    QV_CUDA(c, cudaMemcpyAsync(ctl, c->tree.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, c->stream));
    QV_CUDA(c, cudaStreamSynchronize(c->stream));
    if (ctl[QV_CTL_OVERFLOW] == 1) {
      b->cap_nodes *= 2;
      continue;
    }
    if (ctl[QV_CTL_OVERFLOW])
      return qv_fail(c, QV_ERR_TREE_DEPTH,
                     "octree deeper than %d levels (coincident or nearly coincident points)",
                     QV_MAX_DEPTH);
    b->depth = ctl[QV_CTL_DEPTH];
    int need = 7 * (b->depth + 5) + 8;
    if (need != b->stk_cap) {
      b->stk_cap = need;
      drop_graph(b);
    }
    size_t smem = work_smem_per_warp(b) * 8;
    QV_CUDA(c, cudaFuncSetAttribute(k_batch_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)std::min<size_t>(smem, 227 * 1024)));
    return QV_OK;
  }
  return qv_fail(c, QV_ERR_NOMEM, "forest did not fit after repeated growth");
}

extern "C" int qv_batch_set_points(qv_batch *b, const double *x, const int *infront,
                                   const int *behind) {
  if (!b || !x || !infront || !behind) return QV_ERR_ARG;
  qv_ctx *c = b->c;
  std::vector<int> inf(b->ntot), beh(b->ntot);
  for (int s = 0; s < b->nsys; s++) {
    const int o = b->off[s], n = b->off[s + 1] - o;
    for (int i = o; i < o + n; i++) {
      if (infront[i] < 1 || infront[i] > n || behind[i] < 1 || behind[i] > n)
        return qv_fail(c, QV_ERR_ARG, "system %d slot %d: links must be 1..%d (no empty slots)",
                       s, i - o + 1, n);
      inf[i] = infront[i] + o;
      beh[i] = behind[i] + o;
    }
  }
  int rc = qv_set_points(c, b->ntot, x, inf.data(), beh.data());
  if (rc) return rc;
  QV_CUDA(c, cudaMemset(b->d_status, 0, sizeof(int)));
  if ((rc = size_stack(b))) return rc;
  b->points_set = true;
  return QV_OK;
}

static int check_status(qv_batch *b, int *st) {
  qv_ctx *c = b->c;
  QV_CUDA(c, cudaMemcpyAsync(st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  return QV_OK;
}

extern "C" int qv_batch_velocity(qv_batch *b, double *u) {
  if (!b) return QV_ERR_ARG;
  qv_ctx *c = b->c;
  if (!b->points_set) return qv_fail(c, QV_ERR_STATE, "batch velocity before qv_batch_set_points");
  int rc, st = 0;
  for (int attempt = 0; attempt < 4; attempt++) {
    if ((rc = enqueue_step(b, 0))) return rc;
    if ((rc = check_status(b, &st))) return rc;
    if (st & BST_SINGULAR) return qv_fail(c, QV_ERR_SINGULAR, "singularity in BS (tree) velocity field");
    if (!st) break;
    QV_CUDA(c, cudaMemset(b->d_status, 0, sizeof(int)));
    if ((rc = size_stack(b))) return rc;
  }
  if (st) return qv_fail(c, QV_ERR_STATE, "batch velocity did not complete (status %d)", st);
  if (u)
    QV_CUDA(c, cudaMemcpy(u, c->u, sizeof(double) * 3 * (size_t)b->ntot, cudaMemcpyDeviceToHost));
  return QV_OK;
}

static void try_capture(qv_batch *b) {
  qv_ctx *c = b->c;
  b->graph_tried = true;
  b->graph_ok = false;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  int rc = enqueue_step(b, 1);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc != QV_OK || e != cudaSuccess || !g) {
    cudaGetLastError();
    c->err[0] = 0;
    if (g) cudaGraphDestroy(g);
    return;
  }
  e = cudaGraphInstantiate(&b->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b->gexec = nullptr;
    return;
  }
  b->graph_ok = true;
}

extern "C" int qv_batch_step(qv_batch *b, int nsteps) {
  if (!b || nsteps < 0) return QV_ERR_ARG;
  qv_ctx *c = b->c;
  if (!b->points_set) return qv_fail(c, QV_ERR_STATE, "batch step before qv_batch_set_points");
  int rc;
  int left = nsteps;
  for (int attempt = 0; left > 0 && attempt < 4; attempt++) {
    if (!b->graph_tried) try_capture(b);
    int done0 = 0, done1 = 0;
    QV_CUDA(c, cudaMemcpyAsync(&done0, b->d_done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    for (int k = 0; k < left; k++) {
      if (b->graph_ok) {
        QV_CUDA(c, cudaGraphLaunch(b->gexec, c->stream));
      } else if ((rc = enqueue_step(b, 1))) {
        return rc;
      }
    }
    int st = 0;
    QV_CUDA(c, cudaMemcpyAsync(&done1, b->d_done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    if ((rc = check_status(b, &st))) return rc;
    left -= done1 - done0;
    b->steps_done += done1 - done0;
    if (!st) break;
    if (st & BST_SINGULAR)
      return qv_fail(c, QV_ERR_SINGULAR, "singularity in BS (tree) velocity field");
    // a deeper tree or a larger forest than the capture was sized for: resize,
    // capture again and run the steps that were skipped
    QV_CUDA(c, cudaMemset(b->d_status, 0, sizeof(int)));
    if ((rc = size_stack(b))) return rc;
    drop_graph(b);
  }
  if (left > 0) return qv_fail(c, QV_ERR_STATE, "batch step did not complete (%d left)", left);
  return QV_OK;
}

extern "C" int qv_batch_get_points(qv_batch *b, double *x, double *u) {
  if (!b) return QV_ERR_ARG;
  qv_ctx *c = b->c;
  size_t v = sizeof(double) * 3 * (size_t)b->ntot;
  if (x) QV_CUDA(c, cudaMemcpyAsync(x, c->x, v, cudaMemcpyDeviceToHost, c->stream));
  if (u) QV_CUDA(c, cudaMemcpyAsync(u, c->u, v, cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  return QV_OK;
}

extern "C" int qv_batch_stats(qv_batch *b, long long *evals_leaf_far, int *graph_used,
                              int *config) {
  if (!b) return QV_ERR_ARG;
  qv_ctx *c = b->c;
  unsigned long long ev = 0, evf = 0;
  QV_CUDA(c, cudaMemcpyAsync(&ev, c->evals, sizeof(ev), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaMemcpyAsync(&evf, c->evals_far, sizeof(evf), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  if (evals_leaf_far) {
    evals_leaf_far[0] = (long long)(ev - evf);
    evals_leaf_far[1] = (long long)evf;
  }
  if (graph_used) *graph_used = b->graph_ok ? 1 : 0;
  if (config) {
    config[0] = b->wpb; config[1] = b->bps; config[2] = b->order; config[3] = b->stk_cap;
    config[4] = (int)b->items.size(); config[5] = b->nroots; config[6] = b->depth;
    config[7] = (int)c->launches;
  }
  return QV_OK;
}

// Autotuner: times the work kernel alone (tree, pack and LIA of the current
// positions in place) for each launch shape -- warps per block, resident
// blocks per SM, item order (natural or largest-first) -- and keeps the
// fastest.  None of these changes a result bit: each target's sums are fixed
// by the items' contents, not by which warp runs them or when.
extern "C" int qv_batch_tune(qv_batch *b, int reps, int *best_cfg, float *best_ms) {
  if (!b) return QV_ERR_ARG;
  qv_ctx *c = b->c;
  if (!b->points_set) return qv_fail(c, QV_ERR_STATE, "tune before qv_batch_set_points");
  int rc = qv_batch_velocity(b, nullptr);
  if (rc) return rc;
  reps = std::max(1, reps);
  cudaEvent_t e0, e1;
  QV_CUDA(c, cudaEventCreate(&e0));
  QV_CUDA(c, cudaEventCreate(&e1));
  const int wpbs[] = {2, 4, 8}, bpss[] = {1, 2, 3, 4, 6, 8};
  float best = 1e30f;
  int bw = b->wpb, bb = b->bps, bo = b->order, cur_order = b->order;
  for (int order = 0; order < 2; order++) {
    const std::vector<int4> &it = order ? b->items_cost : b->items;
    QV_CUDA(c, cudaMemcpy(b->d_items, it.data(), sizeof(int4) * it.size(), cudaMemcpyHostToDevice));
    cur_order = order;
    for (int w : wpbs)
      for (int s : bpss) {
        size_t smem = work_smem_per_warp(b) * w;
        if (smem > 227 * 1024) continue;
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_step, w * 32, smem) !=
            cudaSuccess) {
          cudaGetLastError();
          continue;
        }
        if (per < s) continue;
        b->wpb = w;
        b->bps = s;
        float tmin = 1e30f;
        for (int r = 0; r < reps + 1; r++) {
          QV_CUDA(c, cudaEventRecord(e0, c->stream));
          if ((rc = launch_step(b, 0))) return rc;  // velocity only: the state does not move
          QV_CUDA(c, cudaEventRecord(e1, c->stream));
          QV_CUDA(c, cudaEventSynchronize(e1));
          float ms = 0.f;
          QV_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
          if (r > 0) tmin = std::min(tmin, ms);  // the first run warms caches
        }
        if (tmin < best) {
          best = tmin;
          bw = w; bb = s; bo = order;
        }
      }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->wpb = bw;
  b->bps = bb;
  b->order = bo;
  if (cur_order != bo) {
    const std::vector<int4> &it = bo ? b->items_cost : b->items;
    QV_CUDA(c, cudaMemcpy(b->d_items, it.data(), sizeof(int4) * it.size(), cudaMemcpyHostToDevice));
  }
  drop_graph(b);
  if (best_cfg) { best_cfg[0] = bw; best_cfg[1] = bb; best_cfg[2] = bo; }
  if (best_ms) *best_ms = best;
  return QV_OK;
}

// Fix the launch shape without tuning (order: 0 natural, 1 largest first).
extern "C" int qv_batch_set_config(qv_batch *b, int warps_per_block, int blocks_per_sm, int order) {
  if (!b || warps_per_block < 1 || warps_per_block > 32 || blocks_per_sm < 1 || order < 0 || order > 1)
    return QV_ERR_ARG;
  qv_ctx *c = b->c;
  // the step kernel is a cooperative launch: all its blocks must fit at once
  int per = 0;
  size_t smem = work_smem_per_warp(b) * warps_per_block;
  if (smem > 227 * 1024 ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_step, warps_per_block * 32, smem) !=
          cudaSuccess ||
      per < blocks_per_sm) {
    cudaGetLastError();
    return qv_fail(c, QV_ERR_ARG, "qv_batch_set_config: %d blocks of %d warps per SM do not fit (%d do)",
                   blocks_per_sm, warps_per_block, per);
  }
  b->wpb = warps_per_block;
  b->bps = blocks_per_sm;
  if (order != b->order) {
    const std::vector<int4> &it = order ? b->items_cost : b->items;
    QV_CUDA(c, cudaMemcpy(b->d_items, it.data(), sizeof(int4) * it.size(), cudaMemcpyHostToDevice));
    b->order = order;
  }
  drop_graph(b);
  return QV_OK;
}
