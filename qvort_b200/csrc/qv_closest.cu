// qv_closest.cu -- reconnection candidate search.
//
// pclose_tree / closest_tree (src/tree.f90:219-278): for every point, walk the
// tree of the last build -- built before the move, so centroids and the
// parray(1)%infront links are stale (src/run.f90:43-66) -- with the current
// positions and links.  Per point the walk is sequential and order dependent
// (closestd shrinks as it goes and prunes later cells), so the kernel keeps
// the reference's depth-first child order per lane, with the same
// warp-coherent (node, lane mask) stack as the velocity walk, and evaluates
// every distance and theta with round-to-nearest FP64 intrinsics.  The pair
// list (closest, closestd) is bit-identical to the reference arithmetic.
//
// pclose (src/line.f90:205-234): the N^2 scan used when tree_theta == 0.
#include "qv_internal.cuh"

#define CW 4
// Targets per warp: the search is latency-bound, so small systems run more,
// shorter warps (8 targets each: 22 us less per config-2 step than 32), while
// large ones fill the warp (32: 0.68 ms less per config-3 step than 8).
#define TPW_SMALL 8
#define TPW_LARGE 32
#define TPW_LARGE_MIN 65536

__device__ __forceinline__ double dist_exact(const double *a, double b0, double b1, double b2) {
  double d0 = __dsub_rn(a[0], b0), d1 = __dsub_rn(a[1], b1), d2 = __dsub_rn(a[2], b2);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
}

// Every comparison is first taken in FP32 on squared distances from (hi, lo)
// float pairs of the FP64 coordinates; only when it falls within a relative
// 4e-6 of its threshold (or a distance must be stored) is the FP64 expression
// of the reference evaluated, so the outcome is always the FP64 outcome.
// Children's headers are fetched when they are pushed (stack entries carry
// them), so popping a node costs a shared-memory read.
//
// Pruning.  The traversal visits every cell that the reference's walk visits
// until it can prove that a subtree holds nothing that changes the result.
// Per target the walk is a fold over the visited cells in depth-first order:
// a one-point cell with a valid partner j at distance d < closestd sets
// (closest, closestd) = (j, d); a cell that passes the theta test at distance
// d < closestd sets closest = 0.  So the result is fixed by the valid leaf of
// least distance (its first occurrence in that order) and by whether a passing
// cell after it lies closer than that distance.  Let T bound the least valid
// leaf distance from above: any subtree whose cell is farther than T from the
// target holds neither that leaf nor a passing cell closer than it, and
// skipping it leaves the result unchanged.  T is the running closestd, and,
// from the start, the distance to the leaf of the point two links ahead or
// behind when that leaf is itself a valid visited cell (every ancestor opens
// for the target, checked on the parent chain with the same tests), else the
// distance to the first valid visited cell of a near-first descent.  The box
// distance is a lower bound taken in FP32 with a relative 1e-5 and an absolute
// 2e-6 (|x| + L) margin, above every rounding of the operands.
struct __align__(16) CStkEnt {
  SNode32 h;
  int node;
  unsigned mask;
  int pad[2];
};

// The theta test of closest_tree (src/tree.f90:248-249) for a cell with more
// than one point: true when width/dist < 0.5 (the cell is taken whole).
// d2 is the FP32 squared distance of the target from the centroid; d64 is
// set to the FP64 distance when it had to be computed (else left alone).
__device__ __forceinline__ bool search_far(const SNode32 &h, const WNode64 *__restrict__ w64,
                                           int node, float d2, bool tiny, const double *xi,
                                           double &d64) {
  if (!tiny && (d2 > h.rhi || d2 < h.rlo)) return d2 > h.rhi;
  const WNode64 hh = w64[node];
  d64 = dist_exact(xi, hh.cx, hh.cy, hh.cz);
  return __ddiv_rn(hh.width, d64) < .5;
}

__device__ __forceinline__ float cent_d2(const SNode32 &h, const float *xh, const float *xl) {
  float v0 = (xh[0] - h.ch[0]) + (xl[0] - h.cl[0]);
  float v1 = (xh[1] - h.ch[1]) + (xl[1] - h.cl[1]);
  float v2 = (xh[2] - h.ch[2]) + (xl[2] - h.cl[2]);
  return fmaf(v0, v0, fmaf(v1, v1, v2 * v2));
}

// Lower bound on the distance from xh to anything in the cell's box.
__device__ __forceinline__ float box_dist(const SNode32 &h, const float *xh) {
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float a = fmaxf(0.f, fmaxf(h.lo[c] - xh[c], xh[c] - (h.lo[c] + h.w)));
    s = fmaf(a, a, s);
  }
  return sqrtf(s);
}

// Distance to the one-point leaf holding slot s when that leaf is a valid cell
// of target i's walk (partner not i or its neighbours; every ancestor opens);
// else 100, the reference's starting closestd.
__device__ double leaf_bound(int s, int n, int nn, int n_leaf, const int *__restrict__ leaf_of,
                             const int *__restrict__ parent, const int *__restrict__ beh,
                             const WNode64 *__restrict__ w64, const SNode32 *__restrict__ c32,
                             int ii, int fi, int bi, const double *xi, const float *xh,
                             const float *xl) {
  if (s < 0 || s >= n_leaf) return 100.;
  const int k = leaf_of[s];
  if (k < 0 || k >= nn) return 100.;
  const WNode64 hh = w64[k];
  if (hh.count != 1 || hh.first != s || hh.finf < 1 || hh.finf > n) return 100.;
  const int j = beh[hh.finf - 1];
  if (j == ii || j == fi || j == bi) return 100.;
  int a = parent[k];
  for (int it = 0; a >= 0; it++) {
    if (it > QV_MAX_DEPTH + 2 || a >= nn) return 100.;
    const SNode32 h = c32[a];
    if (h.count <= 1) return 100.;
    const float d2 = cent_d2(h, xh, xl);
    double d64 = -1.;
    if (search_far(h, w64, a, d2, d2 < 1e-20f, xi, d64)) return 100.;
    a = parent[a];
  }
  return dist_exact(xi, hh.cx, hh.cy, hh.cz);
}

#define NFCAP 128  // per-lane stack of the near-first bound search
#define NFMAX 512  // its node visits before it gives up (no bound)

// A bound for a target whose link candidates gave none: the first valid cell
// of the target's walk met by a depth-first descent that takes the children
// of every opened cell nearest octant first (the target's own octant, then
// those differing in one, two, three axes).  It only enters cells that open
// for the target, so the leaf it returns is one the walk visits.
__device__ double near_bound(const SNode32 *__restrict__ c32, const WNode64 *__restrict__ w64,
                             const int *__restrict__ beh, int n, int ii, int fi, int bi,
                             const double *xi, const float *xh, const float *xl) {
  int stk[NFCAP];
  int top = 0;
  stk[top++] = 0;
  for (int it = 0; it < NFMAX && top > 0; it++) {
    const int node = stk[--top];
    const SNode32 h = c32[node];
    if (h.count <= 0) continue;
    const float d2 = cent_d2(h, xh, xl);
    if (h.count == 1) {
      const WNode64 hh = w64[node];
      if (hh.finf < 1 || hh.finf > n) continue;
      const int j = beh[hh.finf - 1];
      if (j == ii || j == fi || j == bi) continue;
      return dist_exact(xi, hh.cx, hh.cy, hh.cz);
    }
    double d64 = -1.;
    if (search_far(h, w64, node, d2, d2 < 1e-20f, xi, d64)) continue;  // taken whole
    if (top + h.nchild > NFCAP) return 100.;
    const float hw = 0.5f * h.w;
    const int gx = (xh[0] >= h.lo[0] + hw ? 1 : 0) + (xh[2] >= h.lo[2] + hw ? 2 : 0) +
                   (xh[1] >= h.lo[1] + hw ? 4 : 0);
    const unsigned cm = (unsigned)h.cmask;
    for (int r = 7; r >= 0; r--) {  // XOR masks by rising popcount: 0 1 2 4 3 5 6 7
      const int g = gx ^ ((0x76534210u >> (4 * r)) & 0xFu);
      if ((cm >> g) & 1u) stk[top++] = h.child_first + __popc(cm & ((1u << g) - 1u));
    }
  }
  return 100.;
}

__global__ void __launch_bounds__(CW * 32) k_closest_tree(int n_host, const int *d_n,
                                                         const int *d_skip,
                                                         const double *__restrict__ x,
                                                         const int *__restrict__ inf,
                                                         const int *__restrict__ beh,
                                                         const WNode64 *__restrict__ w64,
                                                         const SNode32 *__restrict__ c32,
                                                         const int *__restrict__ parent,
                                                         const int *__restrict__ leaf_of,
                                                         int n_leaf, int nn, float box,
                                                         int stk_cap, int tpw,
                                                         int *closest, double *closestd,
                                                         int *status) {
  extern __shared__ CStkEnt cstk[];
  if (d_skip && *d_skip) return;
  const int n = d_n ? *d_n : n_host;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  CStkEnt *st = cstk + wid * stk_cap;
  const int nwarps = (n + tpw - 1) / tpw;
  for (int w = blockIdx.x * CW + wid; w < nwarps; w += gridDim.x * CW) {
    int i = w * tpw + lane;
    bool live = lane < tpw && i < n && inf[i] != 0;
    double xi[3] = {0., 0., 0.};
    int ii = i + 1, fi = -1, bi = -1, cl = 0;
    double cd = 100.;
    float cd2 = 1e4f;
    float xh[3] = {0.f, 0.f, 0.f}, xl[3] = {0.f, 0.f, 0.f};
    float thr = 0.f, slack = 0.f;
    double ub = 100.;
    if (live) {
      xi[0] = x[3 * i]; xi[1] = x[3 * i + 1]; xi[2] = x[3 * i + 2];
      fi = inf[i]; bi = beh[i]; cl = closest[i];
      float amax = 0.f;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        xh[c] = __double2float_rn(xi[c]);
        xl[c] = __double2float_rn(xi[c] - (double)xh[c]);
        amax = fmaxf(amax, fabsf(xh[c]));
      }
      slack = 2e-6f * (amax + box);
      // the points two links ahead and behind
      int s1 = (fi >= 1 && fi <= n) ? inf[fi - 1] - 1 : -1;
      int s2 = (bi >= 1 && bi <= n) ? beh[bi - 1] - 1 : -1;
      ub = leaf_bound(s1, n, nn, n_leaf, leaf_of, parent, beh, w64, c32, ii, fi, bi, xi, xh, xl);
      if (s2 != s1)
        ub = fmin(ub, leaf_bound(s2, n, nn, n_leaf, leaf_of, parent, beh, w64, c32, ii, fi, bi, xi,
                                 xh, xl));
      if (ub >= 100.) ub = near_bound(c32, w64, beh, n, ii, fi, bi, xi, xh, xl);
      thr = __double2float_ru(ub) * 1.00001f + slack;
    }
    const unsigned live_mask = __ballot_sync(0xffffffffu, live);
    bool bad = false;
    int top = 0;
    if (lane == 0) {
      st[0].h = c32[0];
      st[0].node = 0;
      st[0].mask = live_mask;
    }
    top = live_mask ? 1 : 0;
    __syncwarp();
    while (top > 0) {
      top--;
      const SNode32 h = st[top].h;
      const int node = st[top].node;
      bool in = (st[top].mask >> lane) & 1u;
      __syncwarp();
      bool open = false;
      if (in && h.count > 0 && box_dist(h, xh) > thr) in = false;
      if (in && h.count > 0) {
        float d2 = cent_d2(h, xh, xl);
        bool tiny = d2 < 1e-20f;
        double d64 = -1.;  // exact distance, computed on demand
        bool pass = h.count == 1 || search_far(h, w64, node, d2, tiny, xi, d64);
        if (pass) {
          // dist < closestd
          bool closer;
          float dc = d2 - cd2;
          if (!tiny && d64 < 0. && fabsf(dc) > 4e-6f * cd2) {
            closer = dc < 0.f;
          } else {
            if (d64 < 0.) {
              const WNode64 hh = w64[node];
              d64 = dist_exact(xi, hh.cx, hh.cy, hh.cz);
            }
            closer = d64 < cd;
          }
          if (closer) {
            if (h.count > 1) {
              cl = 0;
            } else {
              const WNode64 hh = w64[node];
              int j = beh[hh.finf - 1];  // f(parray(1)%infront)%behind with current links
              if (ii != j && fi != j && bi != j) {
                if (d64 < 0.) d64 = dist_exact(xi, hh.cx, hh.cy, hh.cz);
                cl = j;
                cd = d64;
                float c32f = __double2float_rn(cd);
                cd2 = c32f * c32f;
                thr = __double2float_ru(fmin(cd, ub)) * 1.00001f + slack;
              }
            }
          }
        } else {
          open = true;
        }
      }
      unsigned om = __ballot_sync(0xffffffffu, open);
      if (om) {
        int nc = h.nchild;
        if (top + nc > stk_cap) {  // unreachable: the cap follows the tree depth
          bad = true;
          nc = 0;
        }
        if (lane < nc) {
          int ch = h.child_first + nc - 1 - lane;
          CStkEnt &E = st[top + lane];
          E.h = c32[ch];
          E.node = ch;
          E.mask = om;
        }
        top += nc;
      }
      __syncwarp();
    }
    if (lane < tpw && i < n) {
      closestd[i] = cd;  // 100 for empty slots too (src/tree.f90:225)
      if (live) closest[i] = cl;
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, QV_STAT_STACK);
  }
}

#define PT 128
__global__ void __launch_bounds__(PT) k_pclose(int n_host, const int *d_n, const int *d_skip,
                                              const double *__restrict__ x,
                                              const int *__restrict__ inf,
                                              const int *__restrict__ beh, int *closest,
                                              double *closestd) {
  __shared__ double sx[PT][3];
  __shared__ int sa[PT];
  if (d_skip && *d_skip) return;
  const int n = d_n ? *d_n : n_host;
  if (blockIdx.x * PT >= n) return;  // grid sized for the capacity
  int i = blockIdx.x * PT + threadIdx.x;
  bool live = i < n && inf[i] != 0;
  double xi[3] = {0., 0., 0.};
  int fi = -1, bi = -1, cl = 0;
  double cd = 100.;
  if (live) {
    xi[0] = x[3 * i]; xi[1] = x[3 * i + 1]; xi[2] = x[3 * i + 2];
    fi = inf[i]; bi = beh[i]; cl = closest[i];
  }
  for (int t0 = 0; t0 < n; t0 += PT) {
    __syncthreads();
    int j = t0 + threadIdx.x;
    if (j < n) {
      sa[threadIdx.x] = inf[j];
      for (int c = 0; c < 3; c++) sx[threadIdx.x][c] = x[3 * j + c];
    }
    __syncthreads();
    int m = min(PT, n - t0);
    if (live) {
      for (int k = 0; k < m; k++) {
        int jj = t0 + k;
        if (sa[k] == 0) continue;
        if (i != jj && fi != jj + 1 && bi != jj + 1) {
          double d = dist_exact(xi, sx[k][0], sx[k][1], sx[k][2]);
          if (d < cd) {
            cl = jj + 1;
            cd = d;
          }
        }
      }
    }
  }
  if (live) {
    closest[i] = cl;
    closestd[i] = cd;
  }
}

// The candidate search over the slots [0, n).  d_n / d_skip: when given, the
// slot count and a skip flag are read on the device when the kernel starts
// (the search queued behind pinsert, whose new count the host has not read
// yet), and the grid covers n_grid slots, an upper bound on that count.
int qv_launch_closest_ex(qv_ctx *c, const int *d_n, const int *d_skip, int n_grid) {
  if (n_grid == 0) return QV_OK;
  if (c->p.tree_theta > 0) {
    if (!c->tree.valid) return qv_fail(c, QV_ERR_STATE, "pclose_tree without a built tree");
    int rc = qv_tree_finalize_root(c);
    if (rc) return rc;
    const int tpw = n_grid >= TPW_LARGE_MIN ? TPW_LARGE : TPW_SMALL;
    int nwarps = (n_grid + tpw - 1) / tpw;
    int cap = 7 * (c->tree.depth + 1) + 8;
    size_t smem = sizeof(CStkEnt) * cap * CW;
    if (smem > 48 * 1024 && smem > c->smem_search) {  // per context: attributes are per device
      QV_CUDA(c, cudaFuncSetAttribute(k_closest_tree, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
      c->smem_search = smem;
    }
    const TreeBuf &t = c->tree;
    k_closest_tree<<<(nwarps + CW - 1) / CW, CW * 32, smem, c->stream>>>(
        c->n, d_n, d_skip, c->x, c->infront, c->behind, t.w64, t.c32, t.parent, t.leaf_of,
        t.n_leaf, std::min(t.n_nodes, t.cap_nodes), (float)c->p.box_size, cap, tpw, c->closest,
        c->closestd, c->dstatus);
  } else {
    k_pclose<<<(n_grid + PT - 1) / PT, PT, 0, c->stream>>>(c->n, d_n, d_skip, c->x, c->infront,
                                                           c->behind, c->closest, c->closestd);
  }
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

int qv_launch_closest(qv_ctx *c) { return qv_launch_closest_ex(c, nullptr, nullptr, c->n); }
