// qv_walk.cu -- Barnes-Hut tree walk of calc_velocity's Tree arm
// (tree_walk, src/tree.f90:336-421; image loop src/timestep.f90:276-307).
//
// Execution model: a warp task is (32 or 64 targets adjacent in the tree's
// depth-first point order, one periodic image, and for the unshifted image one
// of the root's children); these walks are independent, so the split gives
// the GPU enough warps to hide latency with and keeps the longest task short.
// The mixed walk's lanes carry two targets each in most tasks (see
// walk_task2): one node pop then serves 64 targets, and their FP32 arithmetic
// runs as packed pairs.
// Each task writes per-target partial sums; a second kernel adds them in the
// reference's order (main image by root child, then images peri,perj,perk =
// -1..1), so results do not depend on scheduling.  The
// warp keeps one explicit stack of (node, lane mask) in shared memory: at each
// node every lane in the mask takes its own decision exactly as the reference
// does (leaf -> exact segment, theta < tree_theta -> far-field multipole,
// else open), and children are pushed with the mask of the lanes that opened
// the node.  Each lane therefore visits exactly the nodes its own recursive
// walk would visit, in the same depth-first child order, while node headers
// are fetched once per warp (broadcast loads) instead of once per target.
//
// Opening decisions are always the reference's FP64 decisions: the FP64 walk
// computes them with round-to-nearest intrinsics; the mixed walk evaluates
// them in FP32 with a rigorous margin and falls back to the FP64 expression
// when a decision is within that margin, so both walks visit identical nodes.
//
// The root counts every slot and carries zero circ/Cij (src/tree.f90:51-58):
// when an image's root passes the opening test the image adds nothing, as in
// the reference.
#include <algorithm>
#include <climits>

#include "qv_walk.cuh"

#define WW 4                           // warps per block
#define STK (7 * QV_MAX_DEPTH + 16)    // stack entries per warp (FP64 walk)
#define NSPLIT 8                       // tasks per target group for the main image
// Active points from which the mixed walk's unshifted-image tasks carry 64
// targets, not 32.
#define QV_WALK_PAIR_NEAR 65536
// Active points from which the mixed walk hands out its tasks dynamically.
#define QV_WALK_DYNAMIC 65536

struct WalkArgs {
  int n_act;
  const int *perm;
  const double *x;
  const int *inf, *beh;
  const WNode64 *w64;
  const WPay64 *p64;
  const WNode32 *w32;
  const WPay32 *p32;
  const double *u_li;
  double *u, *u_bs;
  double *part;  // (NSPLIT+NIMG) x n_act x 3 partial sums, slot-major
  double L, theta, gfac;
  int extra, ngroups, stk_cap;
  // mixed walk: groups of 64 targets, and whether the unshifted image's tasks
  // carry 64 targets (else 32 per task, ngroups of them per slot)
  int ng64, pair_near;
  int *next;  // mixed walk, large systems: task counters, [0] the walk, [1] its gated relaunch
  unsigned long long *evals, *evals_far;
  int *status;
  // Root header speculation (see root_open): root_est[3] bounds the distance
  // of the header's centroid from the exact one (nullptr: the header is
  // exact); undecided root tests go to unc (capacity unc_cap, count in
  // *unc_count).  gate non-null: the launch does nothing unless *gate != 0.
  const double *root_est;
  int4 *unc;
  int *unc_count;
  int unc_cap;
  const int *gate;
  // Late level-1 moments (mixed walk): in the unshifted image's tasks, the
  // far-field term of a late root child (node < l1_end, qv_l1_late) is not
  // taken here; bit node - 1 of the task's byte in defer
  // (NSPLIT x n_act, slot major like part) records it for k_walk_l1_fix.  The
  // periodic images' tasks, where those cells are far for most targets, run
  // once the payloads are in and take every term.  l1_end = 0: no deferral.
  int l1_end;
  unsigned char *defer;
  // Mixed walk, dynamic mode: the task counter next[ctr]; or (split != 0) the
  // two launches of a late level-1 build (walk32_body), with l1_ready the flag
  // that k_l1_ready sets once the late payloads are packed.
  int ctr, split;
  const int *l1_ready;
};

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The one cell of an unshifted-image task whose far-field term the walk may
// leave to k_walk_l1_fix: the task's root child k, its first cell, when late.
// That first pop is taken before the task's loop (the loop itself is the
// inline walk's): the targets that find the cell far set its bit in their
// task's byte of defer (zeroed before the launch), the others open it.
__device__ __forceinline__ bool late_cell(const WalkArgs &a, int k) {
  if (!(k > 0 && k < a.l1_end)) return false;
  const int j = qv_l1_pair(k);
  return qv_l1_late(k, a.l1_end, a.w32[k].count, j < a.l1_end ? a.w32[j].count : 0);
}

// Record a lane whose root test the bound left undecided, with the
// evaluations its walk of this task counted.
__device__ __forceinline__ void note_undecided(const WalkArgs &a, int q, int sl, unsigned ev,
                                               unsigned evf) {
  const int k = atomicAdd(a.unc_count, 1);
  if (k < a.unc_cap) a.unc[k] = make_int4(q, sl, (int)ev, (int)evf);
}

// Task slot s: s < NSPLIT -> unshifted image, root child s; else image s-NSPLIT.
__device__ __forceinline__ void slot_image(int bc, int s, int &ma, int &mb, int &mc) {
  ma = mb = mc = 0;
  if (s >= NSPLIT) qv_img_shift(bc, s - NSPLIT, &ma, &mb, &mc);
}

// ---------------------------------------------------------------- FP64 walk
template <int BC>
__device__ __forceinline__ void walk64_body(const WalkArgs &a) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  __shared__ int2 stk[WW][STK];
  if (a.gate && *a.gate == 0) return;
  const double rdelta = a.root_est ? a.root_est[3] : 0.;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int2 *st = stk[wid];
  const int items = a.ngroups * (NSPLIT + NIMG);
  for (int item = blockIdx.x * WW + wid; item < items; item += gridDim.x * WW) {
    const int sl = item / a.ngroups, g = item - sl * a.ngroups;
    int q = g * 32 + lane;
    bool live = q < a.n_act;
    int i = live ? a.perm[q] : 0;
    double xi[3] = {0., 0., 0.};
    int bi = -1, fi = -1, ii = -1;
    if (live) {
      xi[0] = a.x[3 * i]; xi[1] = a.x[3 * i + 1]; xi[2] = a.x[3 * i + 2];
      bi = a.beh[i]; fi = a.inf[i]; ii = i + 1;
    }
    double acc[3] = {0., 0., 0.};
    unsigned long long ev = 0, evf = 0;
    bool bad = false, runc = false;
    int ma, mb, mc;
    slot_image(BC, sl, ma, mb, mc);
    const double s[3] = {shift_of(ma, a.L), shift_of(mb, a.L), shift_of(mc, a.L)};
    int top = 0;
    if (sl >= NSPLIT) {
      const unsigned live_mask = __ballot_sync(0xffffffffu, live);
      if (lane == 0) st[0] = make_int2(0, (int)live_mask);
      top = live_mask ? 1 : 0;
    } else {
      // unshifted image: the root's own decision, then only root child sl
      const WNode64 r = a.w64[0];
      bool ropen = false;
      if (r.count == 1) {
        const unsigned live_mask = __ballot_sync(0xffffffffu, live);
        if (sl == 0 && lane == 0) st[0] = make_int2(0, (int)live_mask);
        top = (sl == 0 && live_mask) ? 1 : 0;
      } else {
        if (live) {
          ropen = root_open(xi, r, s, a.theta, a.extra, rdelta, runc);
          if (!ropen && sl == 0) { ev++; evf++; }  // root far field: zero moments
        }
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
        if (in) {
          int j = h.jb;
          if (j != ii && j != bi && j != fi) {
            double dist = exact_dist(xi, h, s);
            if (dist < QV_DEPS) {
              bad = true;
            } else {
              const WPay64 &P = a.p64[node];
              double R1[3], R2[3], cr[3];
#pragma unroll
              for (int c = 0; c < 3; c++) {
                R1[c] = P.a[c] + s[c] - xi[c];
                R2[c] = P.b[c] + s[c] - xi[c];
              }
              double ra = sqrt(R1[0] * R1[0] + R1[1] * R1[1] + R1[2] * R1[2]);
              double rb = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
              double cc = ra * rb * (ra * rb + (R1[0] * R2[0] + R1[1] * R2[1] + R1[2] * R2[2]));
              cross3(R1, R2, cr);
              double f = (ra + rb) / cc;
#pragma unroll
              for (int c = 0; c < 3; c++) acc[c] += f * cr[c];
              ev++;
            }
          }
        }
      } else {
        bool open = false;
        if (in) {
          double dist = exact_dist(xi, h, s);
          if (node == 0 ? root_open(xi, h, s, a.theta, a.extra, rdelta, runc)
                        : exact_open(dist, h, a.theta, a.extra)) {
            open = true;
          } else {
            ev++;
            evf++;
            if (node != 0) {
              const WPay64 &P = a.p64[node];
              double v[3] = {__dsub_rn(xi[0], __dadd_rn(h.cx, s[0])),
                             __dsub_rn(xi[1], __dadd_rn(h.cy, s[1])),
                             __dsub_rn(xi[2], __dadd_rn(h.cz, s[2]))};
              double d2 = dist * dist, d3 = d2 * dist, d5 = d2 * d2 * dist;
              double cv[3], z[3], vz[3];
              cross3(P.a, v, cv);
#pragma unroll
              for (int l = 0; l < 3; l++) z[l] = v[0] * P.C[l] + v[1] * P.C[3 + l] + v[2] * P.C[6 + l];
              cross3(v, z, vz);
#pragma unroll
              for (int c = 0; c < 3; c++) acc[c] += (cv[c] - P.b[c]) / d3 + 3. * vz[c] / d5;
            }
          }
        }
        unsigned om = __ballot_sync(0xffffffffu, open);
        if (om) {
          int nc = h.nchild;
          if (top + nc > STK) {  // unreachable for trees within QV_MAX_DEPTH
            bad = true;
            nc = 0;
          }
          if (lane < nc) st[top + lane] = make_int2(h.child_first + nc - 1 - lane, (int)om);
          top += nc;
        }
        __syncwarp();
      }
    }
    if (live) {
      double *o = a.part + ((size_t)sl * a.n_act + q) * 3;
      o[0] = acc[0]; o[1] = acc[1]; o[2] = acc[2];
    }
    if (runc) note_undecided(a, q, sl, (unsigned)ev, (unsigned)evf);
    for (int o = 16; o > 0; o >>= 1) {
      ev += __shfl_down_sync(0xffffffffu, ev, o);
      evf += __shfl_down_sync(0xffffffffu, evf, o);
    }
    if (lane == 0 && ev) atomicAdd(a.evals, ev);
    if (lane == 0 && evf) atomicAdd(a.evals_far, evf);
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.status, QV_STAT_SINGULAR);
  }
}

// ---------------------------------------------------------------- mixed walk
// Image shift of task slot sl (FP64), for the rare exact tests.
__device__ __forceinline__ void slot_shift(int bc, int sl, double L, double *s) {
  int ma, mb, mc;
  slot_image(bc, sl, ma, mb, mc);
  s[0] = shift_of(ma, L); s[1] = shift_of(mb, L); s[2] = shift_of(mc, L);
}

// One target of a lane's pair: its point index and links.
struct PairTarget {
  int i, bi, fi;  // point index (0-based), behind, infront; bi = fi = -1 if not live
};

// Leaf pair (src/tree.f90:371-391) of half H of a lane's two targets.
template <int H>
__device__ __forceinline__ void leaf_half(const WalkArgs &a, int bc, int sl, int node,
                                          const WNode32 &h, const PairTarget &t,
                                          const float2 *th, const float2 *tl, float2 v0,
                                          float2 v1, float2 v2, float2 d2, Kahan3x2 &k,
                                          unsigned &ev, bool &bad) {
  const int j = h.jb;
  if (j == t.i + 1 || j == t.bi || j == t.fi) return;
  const float d2h = pick(d2, H);
  bool sing = false;
  if (d2h < 1e-20f) {
    double s[3];
    slot_shift(bc, sl, a.L, s);
    const double xi[3] = {a.x[3 * t.i], a.x[3 * t.i + 1], a.x[3 * t.i + 2]};
    sing = exact_dist(xi, a.w64[node], s) < QV_DEPS;
  }
  if (sing) {
    bad = true;
    return;
  }
  const WPay32 &P = a.p32[node];
  const float r2x = (P.a[0] - pick(th[0], H)) + (P.b[0] - pick(tl[0], H));
  const float r2y = (P.a[1] - pick(th[1], H)) + (P.b[1] - pick(tl[1], H));
  const float r2z = (P.a[2] - pick(th[2], H)) + (P.b[2] - pick(tl[2], H));
  float ox, oy, oz;
  qv_seg32(-pick(v0, H), -pick(v1, H), -pick(v2, H), r2x, r2y, r2z, P.C[0], P.C[1], P.C[2], d2h,
           ox, oy, oz);
  k.add1<H>(ox, oy, oz);
  ev++;
}

// The reference's FP64 opening test on an internal node for one target whose
// FP32 test fell inside the margin.
__device__ __forceinline__ bool exact_test(const WalkArgs &a, int bc, int sl, int node, int i,
                                           double rdelta, bool &runc) {
  double s[3];
  slot_shift(bc, sl, a.L, s);
  const double xi[3] = {a.x[3 * i], a.x[3 * i + 1], a.x[3 * i + 2]};
  const WNode64 h64 = a.w64[node];
  return node == 0 ? root_open(xi, h64, s, a.theta, a.extra, rdelta, runc)
                   : exact_open(exact_dist(xi, h64, s), h64, a.theta, a.extra);
}

// One task of one target per lane: 32 targets (group g of 32), task slot sl.
template <int BC>
__device__ __forceinline__ void walk_task1(const WalkArgs &a, StkEnt *st, int lane, int sl,
                                           int g, double rdelta) {
  int q = g * 32 + lane;
  bool live = q < a.n_act;
  int i = live ? a.perm[q] : 0;
  double xi[3] = {0., 0., 0.};
  int bi = -1, fi = -1, ii = -1;
  if (live) {
    xi[0] = a.x[3 * i]; xi[1] = a.x[3 * i + 1]; xi[2] = a.x[3 * i + 2];
    bi = a.beh[i]; fi = a.inf[i]; ii = i + 1;
  }
  // the gated redo rewrites every task: its bytes of defer start from zero
  if (a.gate && a.defer && sl < NSPLIT && live) a.defer[(size_t)sl * a.n_act + q] = 0;
  bool late_first = false;  // the first cell is a late root child (late_cell)
  Kahan3w k0;
  k0.zero();
  unsigned ev = 0, evf = 0;  // per task: far below 2^32
  bool bad = false, runc = false;
  int ma, mb, mc;
  slot_image(BC, sl, ma, mb, mc);
  const double s[3] = {shift_of(ma, a.L), shift_of(mb, a.L), shift_of(mc, a.L)};
  // target recentred for this image, t = x_i - shift as (hi, lo) floats
  float th[3], tl[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double t = xi[c] - s[c];
    th[c] = __double2float_rn(t);
    tl[c] = __double2float_rn(t - (double)th[c]);
  }
  int top = 0;
  if (sl >= NSPLIT) {
    const unsigned live_mask = __ballot_sync(0xffffffffu, live);
    if (lane == 0) {
      st[0].h = a.w32[0];
      st[0].node = 0;
      st[0].mask = live_mask;
    }
    top = live_mask ? 1 : 0;
  } else {
    // unshifted image: the root's own decision, then only root child sl
    const WNode64 r = a.w64[0];
    bool ropen = false;
    if (r.count == 1) {
      const unsigned live_mask = __ballot_sync(0xffffffffu, live);
      if (sl == 0 && lane == 0) {
        st[0].h = a.w32[0];
        st[0].node = 0;
        st[0].mask = live_mask;
      }
      top = (sl == 0 && live_mask) ? 1 : 0;
    } else {
      if (live) {
        ropen = root_open(xi, r, s, a.theta, a.extra, rdelta, runc);
        if (!ropen && sl == 0) { ev++; evf++; }  // root far field: zero moments
      }
      const unsigned om = __ballot_sync(0xffffffffu, ropen);
      if (om && sl < r.nchild) {
        if (lane == 0) {
          st[0].h = a.w32[r.child_first + sl];
          st[0].node = r.child_first + sl;
          st[0].mask = om;
        }
        late_first = late_cell(a, r.child_first + sl);
        top = 1;
      }
    }
  }
  __syncwarp();
  if (late_first) {
    // the late root child: the loop's decisions for it, its far-field term
    // deferred, its children pushed for the targets that open it
    top = 0;
    const WNode32 h = st[0].h;
    const int node = st[0].node;
    const bool in = (st[0].mask >> lane) & 1u;
    __syncwarp();
    float v0 = (th[0] - h.ch[0]) + (tl[0] - h.cl[0]);
    float v1 = (th[1] - h.ch[1]) + (tl[1] - h.cl[1]);
    float v2 = (th[2] - h.ch[2]) + (tl[2] - h.cl[2]);
    float d2 = fmaf(v0, v0, fmaf(v1, v1, v2 * v2));
    const bool amb = in && !(h.rhi > 0.f && (d2 > h.rhi || d2 < h.rlo));
    bool open = in && d2 < h.rlo;
    if (amb) {
      const WNode64 h64 = a.w64[node];
      open = exact_open(exact_dist(xi, h64, s), h64, a.theta, a.extra);
    }
    const bool far = in && !open;
    ev += far ? 1u : 0u;
    evf += far ? 1u : 0u;
    if (far) a.defer[(size_t)sl * a.n_act + q] = (unsigned char)(1u << (node - 1));
    const unsigned om = __ballot_sync(0xffffffffu, open);
    if (om) {
      const int nc = h.nchild;  // at most 8: the stack holds at least 15
      if (lane < nc) {
        int ch = h.child_first + nc - 1 - lane;
        StkEnt &E = st[lane];
        E.h = a.w32[ch];
        E.node = ch;
        E.mask = om;
      }
      top = nc;
    }
    __syncwarp();
  }
  while (top > 0) {
    top--;
    const WNode32 h = st[top].h;
    const int node = st[top].node;
    const bool in = (st[top].mask >> lane) & 1u;
    __syncwarp();
    // v = t - cent  (= x_i - (cent + shift))
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
      // accept (far field) iff d^2 > rc2, decided in FP32 outside a
      // relative margin of 4e-6 and by the reference's FP64 test inside it.
      // One predicate (far) guards the far-field term: nested per-lane
      // branches cost a reconvergence each on every node pop.
      const bool amb = in && !(h.rhi > 0.f && (d2 > h.rhi || d2 < h.rlo));
      bool open = in && d2 < h.rlo;
      if (amb) {
        const WNode64 h64 = a.w64[node];
        open = node == 0 ? root_open(xi, h64, s, a.theta, a.extra, rdelta, runc)
                         : exact_open(exact_dist(xi, h64, s), h64, a.theta, a.extra);
      }
      const bool far = in && !open;
      ev += far ? 1u : 0u;
      evf += far ? 1u : 0u;
      if (far && node != 0) {  // the root's moments are zero
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
        if (top + nc > a.stk_cap) {  // unreachable: the cap follows the tree depth
          bad = true;
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
    double *o = a.part + ((size_t)sl * a.n_act + q) * 3;
    o[0] = k0.get(0); o[1] = k0.get(1); o[2] = k0.get(2);
  }
  if (runc) note_undecided(a, q, sl, ev, evf);
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_down_sync(0xffffffffu, ev, o);
    evf += __shfl_down_sync(0xffffffffu, evf, o);
  }
  if (lane == 0 && ev) atomicAdd(a.evals, (unsigned long long)ev);
  if (lane == 0 && evf) atomicAdd(a.evals_far, (unsigned long long)evf);
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.status, QV_STAT_SINGULAR);
}

// Each lane carries two targets of a 64-target group (q and q + 32), their
// FP32 state as float2 pairs: one node pop serves 64 targets, and the
// far-field term and the recentring run on the packed FP32 pipe for both.
// Per target, every operation and its order are those of a one-target lane:
// the warp's pops follow the depth-first order of the union of the targets'
// walks, in which each target meets its own nodes in its own walk's order.
template <int BC>
__device__ __forceinline__ void walk_task2(const WalkArgs &a, StkEnt *st, int lane, int sl,
                                           int g, double rdelta) {
  const int qa = g * 64 + lane, qb = qa + 32;
  const bool la = qa < a.n_act, lb = qb < a.n_act;
  PairTarget ta = {0, -1, -1}, tb = {0, -1, -1};
  float2 th[3], tl[3];
  {
    double s[3];
    slot_shift(BC, sl, a.L, s);
    double xa[3] = {0., 0., 0.}, xb[3] = {0., 0., 0.};
    if (la) {
      ta.i = a.perm[qa];
      ta.bi = a.beh[ta.i]; ta.fi = a.inf[ta.i];
      xa[0] = a.x[3 * ta.i]; xa[1] = a.x[3 * ta.i + 1]; xa[2] = a.x[3 * ta.i + 2];
    }
    if (lb) {
      tb.i = a.perm[qb];
      tb.bi = a.beh[tb.i]; tb.fi = a.inf[tb.i];
      xb[0] = a.x[3 * tb.i]; xb[1] = a.x[3 * tb.i + 1]; xb[2] = a.x[3 * tb.i + 2];
    }
    // target recentred for this image, t = x_i - shift as (hi, lo) floats
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double ua = xa[c] - s[c], ub = xb[c] - s[c];
      th[c].x = __double2float_rn(ua);
      tl[c].x = __double2float_rn(ua - (double)th[c].x);
      th[c].y = __double2float_rn(ub);
      tl[c].y = __double2float_rn(ub - (double)th[c].y);
    }
  }
  // the gated redo rewrites every task: its bytes of defer start from zero
  if (a.gate && a.defer && sl < NSPLIT) {
    if (la) a.defer[(size_t)sl * a.n_act + qa] = 0;
    if (lb) a.defer[(size_t)sl * a.n_act + qb] = 0;
  }
  bool late_first = false;  // the first cell is a late root child (late_cell)
  Kahan3x2 k0;
  k0.zero();
  unsigned eva = 0, evfa = 0, evb = 0, evfb = 0;  // per task: far below 2^32
  bool bad = false, runa = false, runb = false;
  int top = 0;
  if (sl >= NSPLIT) {
    const unsigned ma = __ballot_sync(0xffffffffu, la), mb = __ballot_sync(0xffffffffu, lb);
    if (lane == 0) {
      st[0].h = a.w32[0];
      st[0].node = 0;
      st[0].mask = ma;
      st[0].mask2 = mb;
    }
    top = (ma | mb) ? 1 : 0;
  } else {
    // unshifted image: the root's own decision, then only root child sl
    const WNode64 r = a.w64[0];
    if (r.count == 1) {
      const unsigned ma = __ballot_sync(0xffffffffu, la), mb = __ballot_sync(0xffffffffu, lb);
      if (sl == 0 && lane == 0) {
        st[0].h = a.w32[0];
        st[0].node = 0;
        st[0].mask = ma;
        st[0].mask2 = mb;
      }
      top = (sl == 0 && (ma | mb)) ? 1 : 0;
    } else {
      bool oa = false, ob = false;
      if (la) {
        oa = exact_test(a, BC, sl, 0, ta.i, rdelta, runa);
        if (!oa && sl == 0) { eva++; evfa++; }  // root far field: zero moments
      }
      if (lb) {
        ob = exact_test(a, BC, sl, 0, tb.i, rdelta, runb);
        if (!ob && sl == 0) { evb++; evfb++; }
      }
      const unsigned ma = __ballot_sync(0xffffffffu, oa), mb = __ballot_sync(0xffffffffu, ob);
      if ((ma | mb) && sl < r.nchild) {
        if (lane == 0) {
          st[0].h = a.w32[r.child_first + sl];
          st[0].node = r.child_first + sl;
          st[0].mask = ma;
          st[0].mask2 = mb;
        }
        late_first = late_cell(a, r.child_first + sl);
        top = 1;
      }
    }
  }
  __syncwarp();
  if (late_first) {
    // the late root child: the loop's decisions for it, its far-field term
    // deferred, its children pushed for the targets that open it
    top = 0;
    const WNode32 h = st[0].h;
    const int node = st[0].node;
    const bool ina = (st[0].mask >> lane) & 1u, inb = (st[0].mask2 >> lane) & 1u;
    __syncwarp();
    const float2 v0 = add2(sub2(th[0], bc2(h.ch[0])), sub2(tl[0], bc2(h.cl[0])));
    const float2 v1 = add2(sub2(th[1], bc2(h.ch[1])), sub2(tl[1], bc2(h.cl[1])));
    const float2 v2 = add2(sub2(th[2], bc2(h.ch[2])), sub2(tl[2], bc2(h.cl[2])));
    const float2 d2 = fma2(v0, v0, fma2(v1, v1, mul2(v2, v2)));
    const bool sure = h.rhi > 0.f;
    const bool amba = ina && !(sure && (d2.x > h.rhi || d2.x < h.rlo));
    const bool ambb = inb && !(sure && (d2.y > h.rhi || d2.y < h.rlo));
    bool opa = ina && d2.x < h.rlo, opb = inb && d2.y < h.rlo;
    if (amba) opa = exact_test(a, BC, sl, node, ta.i, rdelta, runa);
    if (ambb) opb = exact_test(a, BC, sl, node, tb.i, rdelta, runb);
    const bool fa = ina && !opa, fb = inb && !opb;
    eva += fa ? 1u : 0u;
    evfa += fa ? 1u : 0u;
    evb += fb ? 1u : 0u;
    evfb += fb ? 1u : 0u;
    const unsigned char bit = (unsigned char)(1u << (node - 1));
    if (fa) a.defer[(size_t)sl * a.n_act + qa] = bit;
    if (fb) a.defer[(size_t)sl * a.n_act + qb] = bit;
    const unsigned ma = __ballot_sync(0xffffffffu, opa), mb = __ballot_sync(0xffffffffu, opb);
    if (ma | mb) {
      const int nc = h.nchild;  // at most 8: the stack holds at least 15
      if (lane < nc) {
        const int ch = h.child_first + nc - 1 - lane;
        StkEnt &E = st[lane];
        E.h = a.w32[ch];
        E.node = ch;
        E.mask = ma;
        E.mask2 = mb;
      }
      top = nc;
    }
    __syncwarp();
  }
  while (top > 0) {
    top--;
    const WNode32 h = st[top].h;
    const int node = st[top].node;
    const bool ina = (st[top].mask >> lane) & 1u, inb = (st[top].mask2 >> lane) & 1u;
    __syncwarp();
    // v = t - cent  (= x_i - (cent + shift))
    const float2 v0 = add2(sub2(th[0], bc2(h.ch[0])), sub2(tl[0], bc2(h.cl[0])));
    const float2 v1 = add2(sub2(th[1], bc2(h.ch[1])), sub2(tl[1], bc2(h.cl[1])));
    const float2 v2 = add2(sub2(th[2], bc2(h.ch[2])), sub2(tl[2], bc2(h.cl[2])));
    const float2 d2 = fma2(v0, v0, fma2(v1, v1, mul2(v2, v2)));
    if (h.count == 1) {
      if (ina) leaf_half<0>(a, BC, sl, node, h, ta, th, tl, v0, v1, v2, d2, k0, eva, bad);
      if (inb) leaf_half<1>(a, BC, sl, node, h, tb, th, tl, v0, v1, v2, d2, k0, evb, bad);
    } else {
      // accept (far field) iff d^2 > rc2, decided in FP32 outside a
      // relative margin of 4e-6 and by the reference's FP64 test inside it.
      // One predicate per target (far) guards the far-field term: nested
      // per-lane branches cost a reconvergence each on every node pop.
      const bool sure = h.rhi > 0.f;
      const bool amba = ina && !(sure && (d2.x > h.rhi || d2.x < h.rlo));
      const bool ambb = inb && !(sure && (d2.y > h.rhi || d2.y < h.rlo));
      bool opa = ina && d2.x < h.rlo, opb = inb && d2.y < h.rlo;
      if (amba) opa = exact_test(a, BC, sl, node, ta.i, rdelta, runa);
      if (ambb) opb = exact_test(a, BC, sl, node, tb.i, rdelta, runb);
      const bool fa = ina && !opa, fb = inb && !opb;
      eva += fa ? 1u : 0u;
      evfa += fa ? 1u : 0u;
      evb += fb ? 1u : 0u;
      evfb += fb ? 1u : 0u;
      if ((fa || fb) && node != 0) {  // the root's moments are zero
        const WPay32 &P = a.p32[node];
        const float2 rd = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
        const float2 rd2 = mul2(rd, rd), rd3 = mul2(rd2, rd), rd5 = mul2(rd3, rd2);
        const float2 z0 = fma2(v0, bc2(P.C[0]), fma2(v1, bc2(P.C[3]), mul2(v2, bc2(P.C[6]))));
        const float2 z1 = fma2(v0, bc2(P.C[1]), fma2(v1, bc2(P.C[4]), mul2(v2, bc2(P.C[7]))));
        const float2 z2 = fma2(v0, bc2(P.C[2]), fma2(v1, bc2(P.C[5]), mul2(v2, bc2(P.C[8]))));
        const float2 cx = sub2(fma2(bc2(P.a[1]), v2, mul2(bc2(-P.a[2]), v1)), bc2(P.b[0]));
        const float2 cy = sub2(fma2(bc2(P.a[2]), v0, mul2(bc2(-P.a[0]), v2)), bc2(P.b[1]));
        const float2 cz = sub2(fma2(bc2(P.a[0]), v1, mul2(bc2(-P.a[1]), v0)), bc2(P.b[2]));
        const float2 wx = fma2(v1, z2, mul2(neg2(v2), z1));
        const float2 wy = fma2(v2, z0, mul2(neg2(v0), z2));
        const float2 wz = fma2(v0, z1, mul2(neg2(v1), z0));
        const float2 t5 = mul2(bc2(3.f), rd5);
        k0.add(fma2(cx, rd3, mul2(wx, t5)), fma2(cy, rd3, mul2(wy, t5)),
               fma2(cz, rd3, mul2(wz, t5)), fa, fb);
      }
      const unsigned ma = __ballot_sync(0xffffffffu, opa), mb = __ballot_sync(0xffffffffu, opb);
      if (ma | mb) {
        int nc = h.nchild;
        if (top + nc > a.stk_cap) {  // unreachable: the cap follows the tree depth
          bad = true;
          nc = 0;
        }
        if (lane < nc) {
          const int ch = h.child_first + nc - 1 - lane;
          StkEnt &E = st[top + lane];
          E.h = a.w32[ch];
          E.node = ch;
          E.mask = ma;
          E.mask2 = mb;
        }
        top += nc;
      }
      __syncwarp();
    }
  }
  if (la) {
    double *o = a.part + ((size_t)sl * a.n_act + qa) * 3;
    o[0] = k0.get(0, 0); o[1] = k0.get(0, 1); o[2] = k0.get(0, 2);
  }
  if (lb) {
    double *o = a.part + ((size_t)sl * a.n_act + qb) * 3;
    o[0] = k0.get(1, 0); o[1] = k0.get(1, 1); o[2] = k0.get(1, 2);
  }
  if (runa) note_undecided(a, qa, sl, eva, evfa);
  if (runb) note_undecided(a, qb, sl, evb, evfb);
  unsigned ev = eva + evb, evf = evfa + evfb;
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_down_sync(0xffffffffu, ev, o);
    evf += __shfl_down_sync(0xffffffffu, evf, o);
  }
  if (lane == 0 && ev) atomicAdd(a.evals, (unsigned long long)ev);
  if (lane == 0 && evf) atomicAdd(a.evals_far, (unsigned long long)evf);
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.status, QV_STAT_SINGULAR);
}

// Task order: the unshifted image's tasks (the heaviest: they carry the near
// field), slot by slot, then the periodic images'.  Large systems hand the
// tasks out one at a time from a counter, so that a warp which finishes early
// takes the next task instead of idling until its block's slowest warp is
// done.  Small ones (a few tasks per warp) keep a fixed task per warp, whose
// block's four warps walk neighbouring target groups and share their nodes in
// L1: handed out dynamically, or longest first by the last walk's task times,
// they ran slower (the walk's length is then its longest near-field task).
// Image tasks carry 64 targets (two per lane); the unshifted image's carry 64
// when the system is large and 32 (one per lane) otherwise, which halves the
// longest task when there are few tasks per warp.  Each (group, slot) task
// writes its own partial sums, so neither the order nor the kind changes a
// result: per target, both kinds compute the same sums bit for bit.
template <int BC>
__device__ __forceinline__ void walk32_body(const WalkArgs &a) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  extern __shared__ StkEnt stk_dyn[];
  if (a.gate && *a.gate == 0) return;
  const double rdelta = a.root_est ? a.root_est[3] : 0.;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  StkEnt *st = stk_dyn + wid * a.stk_cap;
  const int gn = a.pair_near ? a.ng64 : a.ngroups;  // groups of the unshifted image's tasks
  const int nnear = NSPLIT * gn;
  const int items = nnear + NIMG * a.ng64;
  // Late level-1 split: the unshifted image's tasks come from next[0], the
  // images' (which read the late payloads) from next[2].  Launch 1 (split 1)
  // takes the unshifted ones, then the images' if the payloads are in by then
  // (the flag is read, never waited for: otherwise it stops); launch 2
  // (split 2), queued behind the payloads, takes the images' and then helps
  // with the unshifted ones.
  // split launches, per warp: bit 0 = on its second pool, bit 1 = the ready
  // flag was seen set (read once: the acquire load is a round trip to L2)
  __shared__ int wphase[WW];
  if (lane == 0) wphase[wid] = 0;
  int item = blockIdx.x * WW + wid;
  for (;;) {
    if (a.next) {
      if (lane == 0) {
        if (!a.split) {
          item = atomicAdd(a.next + a.ctr, 1);
        } else {
          for (;;) {
            const int phase = wphase[wid] & 1;
            const bool img = (phase == 0) == (a.split == 2);
            if (img && a.split == 1 && !(wphase[wid] & 2)) {
              if (ld_acquire(a.l1_ready) == 0) {
                item = items;
                break;
              }
              wphase[wid] |= 2;
            }
            const int t = atomicAdd(a.next + (img ? 2 : 0), 1);
            if (t < (img ? items - nnear : nnear)) {
              item = img ? nnear + t : t;
              break;
            }
            if (phase == 1) {
              item = items;
              break;
            }
            wphase[wid] |= 1;
          }
        }
      }
      item = __shfl_sync(0xffffffffu, item, 0);
    }
    if (item >= items) break;
    if (item < nnear) {
      const int sl = item / gn, g = item - sl * gn;
      if (a.pair_near) walk_task2<BC>(a, st, lane, sl, g, rdelta);
      else walk_task1<BC>(a, st, lane, sl, g, rdelta);
    } else {
      const int j = item - nnear, k = j / a.ng64;
      walk_task2<BC>(a, st, lane, NSPLIT + k, j - k * a.ng64, rdelta);
    }
    item += gridDim.x * WW;
  }
}

// The walks, and the same walks under a second name for the gated relaunch
// after an overflowing root fix-up (it returns at once unless flagged), so
// that a profile tells the two launches apart.
template <int BC>
__global__ void __launch_bounds__(WW * 32) k_walk64(WalkArgs a) { walk64_body<BC>(a); }
template <int BC>
__global__ void __launch_bounds__(WW * 32) k_walk64_redo(WalkArgs a) { walk64_body<BC>(a); }
// 5 blocks/SM (96 registers): faster than 4 (111 registers) on the paired tasks
#define WALK32_BLOCKS_PER_SM 5
template <int BC>
__global__ void __launch_bounds__(WW * 32, WALK32_BLOCKS_PER_SM) k_walk32(WalkArgs a) {
  walk32_body<BC>(a);
}
template <int BC>
__global__ void __launch_bounds__(WW * 32, WALK32_BLOCKS_PER_SM) k_walk32_redo(WalkArgs a) {
  walk32_body<BC>(a);
}

// u_bs = main + images, u = (u_li + main) + images, with the main image summed
// over the root's children in child order and the images in the reference's
// loop order (src/timestep.f90:276-288).
__global__ void k_walk_reduce(int n_act, int nimg, const int *__restrict__ perm,
                              const double *__restrict__ part, double gfac,
                              const double *__restrict__ u_li, double *u, double *u_bs) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_act) return;
  int i = perm[q];
  double s0[3] = {0., 0., 0.}, s1[3] = {0., 0., 0.};
  for (int m = 0; m < NSPLIT; m++)
    for (int c = 0; c < 3; c++) s0[c] += part[((size_t)m * n_act + q) * 3 + c];
  for (int m = NSPLIT; m < NSPLIT + nimg; m++)
    for (int c = 0; c < 3; c++) s1[c] += part[((size_t)m * n_act + q) * 3 + c];
  for (int c = 0; c < 3; c++) {
    double b0 = s0[c] * gfac, b1 = s1[c] * gfac;
    u_bs[3 * i + c] = b0 + b1;
    u[3 * i + c] = (u_li[3 * i + c] + b0) + b1;
  }
}

// Root tests the centroid bound left undecided (see root_open), once the
// exact root header is in: a lane that walked an image whose root is in fact
// far drops that image's sum (the root's moments are zero) and counts the one
// far-field evaluation the reference counts instead of its walk's.  More
// undecided tests than the list holds: zero the counters and raise the redo
// flag, and the gated second walk recomputes every task with the exact root.
__global__ void k_root_fix(WalkArgs a, int bc, const int4 *__restrict__ unc, int *ctl) {
  const int cnt = ctl[0];
  if (cnt > QV_ROOT_UNC_CAP) {
    if (threadIdx.x == 0) {
      *a.evals = 0;
      *a.evals_far = 0;
      ctl[2] = 1;
    }
    return;
  }
  if (threadIdx.x == 0) ctl[2] = 0;
  const WNode64 r = a.w64[0];
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int4 u = unc[e];
    const int q = u.x, sl = u.y, i = a.perm[q];
    const double xi[3] = {a.x[3 * i], a.x[3 * i + 1], a.x[3 * i + 2]};
    int ma, mb, mc;
    slot_image(bc, sl, ma, mb, mc);
    const double s[3] = {shift_of(ma, a.L), shift_of(mb, a.L), shift_of(mc, a.L)};
    if (exact_open(exact_dist(xi, r, s), r, a.theta, a.extra)) continue;
    double *o = a.part + ((size_t)sl * a.n_act + q) * 3;
    o[0] = o[1] = o[2] = 0.;
    if (a.defer && sl < NSPLIT) a.defer[(size_t)sl * a.n_act + q] = 0;
    const unsigned long long one = (sl == 0 || sl >= NSPLIT) ? 1ull : 0ull;
    atomicAdd(a.evals, one - (unsigned long long)(unsigned)u.z);
    atomicAdd(a.evals_far, one - (unsigned long long)(unsigned)u.w);
  }
}

// The root children's far-field terms that the mixed walk deferred (late_cell),
// once their moments and payloads are in: for each (task slot, target) whose
// byte is set, the reference's far-cell term (src/tree.f90:394-413) of each
// flagged child, in child order, in FP64 from the FP64 header and payload, as
// the FP64 walk takes it, added to that task's partial sum after the walk's
// compensated FP32 sum.
__global__ void k_walk_l1_fix(WalkArgs a, int bc, int ntask) {
  const size_t tot = (size_t)ntask * a.n_act;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    unsigned m = a.defer[e];
    if (!m) continue;
    const int sl = (int)(e / (size_t)a.n_act), q = (int)(e - (size_t)sl * a.n_act);
    const int i = a.perm[q];
    const double xi[3] = {a.x[3 * i], a.x[3 * i + 1], a.x[3 * i + 2]};
    double s[3];
    slot_shift(bc, sl, a.L, s);
    double acc[3] = {0., 0., 0.};
    for (; m; m &= m - 1) {
      const int node = __ffs(m);  // bit node - 1
      const WNode64 h = a.w64[node];
      const WPay64 &P = a.p64[node];
      const double dist = exact_dist(xi, h, s);
      double v[3] = {__dsub_rn(xi[0], __dadd_rn(h.cx, s[0])), __dsub_rn(xi[1], __dadd_rn(h.cy, s[1])),
                     __dsub_rn(xi[2], __dadd_rn(h.cz, s[2]))};
      double d2 = dist * dist, d3 = d2 * dist, d5 = d2 * d2 * dist;
      double cv[3], z[3], vz[3];
      cross3(P.a, v, cv);
#pragma unroll
      for (int l = 0; l < 3; l++) z[l] = v[0] * P.C[l] + v[1] * P.C[3 + l] + v[2] * P.C[6 + l];
      cross3(v, z, vz);
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] += (cv[c] - P.b[c]) / d3 + 3. * vz[c] / d5;
    }
    double *o = a.part + e * 3;
    o[0] += acc[0]; o[1] += acc[1]; o[2] += acc[2];
  }
}

int qv_launch_walk(qv_ctx *c) {
  TreeBuf &t = c->tree;
  if (!t.valid) return qv_fail(c, QV_ERR_STATE, "tree walk without a built tree");
  if (t.n_act == 0) return QV_OK;
  int nimg = qv_img_count(c->p.boundary);
  size_t need = sizeof(double) * 3 * (size_t)(NSPLIT + nimg) * t.n_act;
  if (need > c->walk_part_bytes) {
    int rc = qv_grow(c, (void **)&c->walk_part, need);
    if (rc) return rc;
    c->walk_part_bytes = need;
  }
  WalkArgs a;
  a.n_act = t.n_act; a.perm = t.perm; a.x = c->x; a.inf = c->infront; a.beh = c->behind;
  a.w64 = t.w64; a.p64 = t.p64; a.w32 = t.w32; a.p32 = t.p32;
  a.u_li = c->u_li; a.u = c->u; a.u_bs = c->u_bs; a.part = c->walk_part;
  a.L = c->p.box_size; a.theta = c->p.tree_theta; a.gfac = c->p.quant_circ / 4. / QV_PI;
  a.extra = c->p.tree_extra_correction; a.evals = c->evals; a.evals_far = c->evals_far;
  a.status = c->dstatus;
  a.root_est = nullptr; a.unc = nullptr; a.unc_count = nullptr; a.unc_cap = 0; a.gate = nullptr;
  const bool spec = t.root_pending;
  const bool mixed = c->p.precision == QV_PREC_MIXED;
  // Late level-1 payloads (qv_launch_tree_build): the mixed walk runs the
  // unshifted image's tasks at once, deferring those cells' rare far-field
  // terms, and the periodic images' tasks on a side stream once the payloads
  // are in; its blocks take the SMs as the first launch's blocks run out of
  // tasks.  The FP64 walk reads every payload, so it joins them first.
  const bool l1 = mixed && t.l1_pending && t.lvl_start.size() > 2;
  a.l1_end = 0;
  a.defer = nullptr;
  if (l1) {
    const size_t nbytes = (size_t)NSPLIT * t.n_act;
    if (nbytes > c->walk_defer_bytes) {
      int rc = qv_grow(c, (void **)&c->walk_defer, nbytes);
      if (rc) return rc;
      c->walk_defer_bytes = nbytes;
    }
    a.l1_end = t.lvl_start[2];
    a.defer = c->walk_defer;
  } else if (t.l1_pending) {
    QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_l1, 0));
    t.l1_pending = false;
  }
  if (spec) {
    a.root_est = t.root_est; a.unc = t.root_unc; a.unc_count = t.root_ctl;
    a.unc_cap = QV_ROOT_UNC_CAP;
  }
  a.ngroups = (t.n_act + 31) / 32;
  a.ng64 = (t.n_act + 63) / 64;
  a.pair_near = t.n_act >= QV_WALK_PAIR_NEAR;
  a.ctr = 0;
  a.split = 0;
  a.l1_ready = nullptr;
  // a depth-first stack over a tree of depth D never holds more than 7 D + 1
  // entries (each open pushes at most 8 and pops 1)
  a.stk_cap = 7 * (t.depth + 1) + 8;
  size_t smem = sizeof(StkEnt) * a.stk_cap * WW;
  const long nnear = (long)NSPLIT * (a.pair_near ? a.ng64 : a.ngroups);
  const long items = mixed ? nnear + (long)a.ng64 * nimg : (long)a.ngroups * (NSPLIT + nimg);
  const bool dynamic = mixed && (t.n_act >= QV_WALK_DYNAMIC || l1);
  // blocks of a launch of m tasks
  auto grid_for = [&](long m) -> int {
    const long cap = dynamic ? (long)WALK32_BLOCKS_PER_SM * c->sm_count  // one resident grid
                             : 64L * c->sm_count;
    return (int)std::max(1L, std::min<long>((m + WW - 1) / WW, cap));
  };
  int nb = grid_for(items);
  a.next = nullptr;
  if (dynamic) {
    // every warp stays until its task counters run out: next[0] the walk (the
    // unshifted image's tasks when level 1 is late), next[1] the gated redo,
    // next[2] the images' tasks when level 1 is late
    if (!c->walk_next) {
      int rc = qv_grow(c, (void **)&c->walk_next, 4 * sizeof(int));
      if (rc) return rc;
    }
    QV_CUDA(c, cudaMemsetAsync(c->walk_next, 0, 4 * sizeof(int), c->stream));
    a.next = c->walk_next;
  }
  if (mixed && smem > 48 * 1024) {
    if (smem > c->smem_walk) {  // per context: attributes are per device
      const void *fs[] = {(const void *)k_walk32<QV_BC_OPEN>, (const void *)k_walk32<QV_BC_PERIODIC>,
                          (const void *)k_walk32<QV_BC_OPENX>, (const void *)k_walk32<QV_BC_OPENXY>,
                          (const void *)k_walk32_redo<QV_BC_OPEN>,
                          (const void *)k_walk32_redo<QV_BC_PERIODIC>,
                          (const void *)k_walk32_redo<QV_BC_OPENX>,
                          (const void *)k_walk32_redo<QV_BC_OPENXY>};
      for (const void *f : fs)
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      c->smem_walk = smem;
    }
  }
  auto launch = [&](const WalkArgs &w, int grid, cudaStream_t st) -> int {
    const bool redo = w.gate != nullptr;
    switch (c->p.boundary) {
#define QV_WALK_CASE(BCV)                                                  \
  case BCV:                                                                \
    if (mixed && redo) k_walk32_redo<BCV><<<grid, WW * 32, smem, st>>>(w); \
    else if (mixed) k_walk32<BCV><<<grid, WW * 32, smem, st>>>(w);        \
    else if (redo) k_walk64_redo<BCV><<<grid, WW * 32, 0, st>>>(w);       \
    else k_walk64<BCV><<<grid, WW * 32, 0, st>>>(w);                      \
    break;
      QV_WALK_CASE(QV_BC_OPEN)
      QV_WALK_CASE(QV_BC_PERIODIC)
      QV_WALK_CASE(QV_BC_OPENX)
      QV_WALK_CASE(QV_BC_OPENXY)
#undef QV_WALK_CASE
      default:
        return qv_fail(c, QV_ERR_UNSUPPORTED, "boundary %d not supported", c->p.boundary);
    }
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    return QV_OK;
  };
  int rc;
  if (l1) {
    // launch 1 now; launch 2 behind the late payloads on aux[3] (the stream
    // that packs them).  In practice launch 1 finds the payloads in once the
    // unshifted tasks run out and takes every task; launch 2's blocks then
    // find both counters spent.
    QV_CUDA(c, cudaMemsetAsync(c->walk_defer, 0, (size_t)NSPLIT * t.n_act, c->stream));
    WalkArgs a1 = a;
    a1.split = 1;
    a1.l1_ready = t.l1list + 15;
    QV_CUDA(c, cudaEventRecord(c->ev_fork, c->stream));
    if (mixed) qv_phase_begin(c, PH_WALK);
    if ((rc = launch(a1, nb, c->stream))) return rc;
    if (mixed) qv_phase_end_async(c, PH_WALK);
    WalkArgs a2 = a;
    a2.split = 2;
    cudaStream_t s3 = c->aux[3];
    QV_CUDA(c, cudaStreamWaitEvent(s3, c->ev_fork, 0));
    if ((rc = launch(a2, nb, s3))) return rc;
    QV_CUDA(c, cudaEventRecord(c->ev_l1, s3));
    // the finalize below joins ev_l1: the payloads and launch 2
  } else {
    if (mixed) qv_phase_begin(c, PH_WALK);
    if ((rc = launch(a, nb, c->stream))) return rc;
    if (mixed) qv_phase_end_async(c, PH_WALK);
  }
  // joined now, long after they finished: the images' walk and the late
  // level-1 payloads, and the exact root centroid
  if (spec || l1)
    if ((rc = qv_tree_finalize_root(c))) return rc;
  if (spec) {
    // the fix-up of undecided root tests, and the second walk that runs only
    // if the fix-up's list overflowed (it defers the same cells)
    k_root_fix<<<1, 256, 0, c->stream>>>(a, c->p.boundary, t.root_unc, t.root_ctl);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    WalkArgs b = a;
    b.root_est = nullptr; b.unc = nullptr; b.unc_count = nullptr; b.unc_cap = 0;
    b.gate = t.root_ctl + 2;
    b.ctr = 1;
    if ((rc = launch(b, std::min(nb, 2 * c->sm_count), c->stream))) return rc;
  }
  if (l1) {
    k_walk_l1_fix<<<4 * c->sm_count, 256, 0, c->stream>>>(a, c->p.boundary, NSPLIT);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
  }
  k_walk_reduce<<<(t.n_act + 255) / 256, 256, 0, c->stream>>>(t.n_act, nimg, t.perm, c->walk_part,
                                                                a.gfac, c->u_li, c->u, c->u_bs);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

// ------------------------------------------------------- field points (tree)
// tree_walk_general (src/tree.f90:425-488) at m arbitrary points, as the Tree
// arm of mesh_velocity uses it (src/timestep.f90:374-452): per point the
// unshifted tree, then the boundary's images in the reference's loop order,
// all into one running FP64 sum, with the reference's operations: a node
// within epsilon of the point adds nothing (its subtree included), the
// opening test is width/dist < tree_theta, a leaf's segment runs from its
// centroid to centroid + circ, the leaf term is divided by 4 pi, the far term
// is not, and neither carries quant_circ.  One warp per 32 points with the
// warp-coherent (node, lane mask) stack of the velocity walk.
#define GW 4
template <int BC>
__global__ void __launch_bounds__(GW * 32) k_walk_general(int m, const double *__restrict__ pts,
                                                         const WNode64 *__restrict__ w64,
                                                         const WPay64 *__restrict__ p64,
                                                         const double *__restrict__ cent,
                                                         const double *__restrict__ circ,
                                                         double L, double theta, int nroots,
                                                         double *u, unsigned long long *evals,
                                                         int *status) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  __shared__ int2 stk[GW][STK];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int2 *st = stk[wid];
  const int ngroups = (m + 31) / 32;
  for (int g = blockIdx.x * GW + wid; g < ngroups; g += gridDim.x * GW) {
    const int q = g * 32 + lane;
    const bool live = q < m;
    double x[3] = {0., 0., 0.};
    if (live) { x[0] = pts[3 * q]; x[1] = pts[3 * q + 1]; x[2] = pts[3 * q + 2]; }
    double acc[3] = {0., 0., 0.};
    unsigned long long ev = 0;
    bool bad = false;
    const unsigned live_mask = __ballot_sync(0xffffffffu, live);
    for (int img = -1; img < NIMG; img++) {
      int ma = 0, mb = 0, mc = 0;
      if (img >= 0) qv_img_shift(BC, img, &ma, &mb, &mc);
      const double s[3] = {shift_of(ma, L), shift_of(mb, L), shift_of(mc, L)};
      int top = 0;
      if (lane == 0) st[0] = make_int2(0, (int)live_mask);
      top = live_mask ? 1 : 0;
      __syncwarp();
      while (top > 0) {
        top--;
        const int2 e = st[top];
        __syncwarp();
        const int node = e.x;
        const bool in = (((unsigned)e.y) >> lane) & 1u;
        const WNode64 h = w64[node];
        bool open = false;
        if (in && h.count > 0) {
          const double dist = exact_dist(x, h, s);
          if (!(dist < QV_DEPS)) {
            const double th = __ddiv_rn(h.width, dist);
            const double zero3[3] = {0., 0., 0.};
            const double *C0 = cent + 3 * node, *R = node < nroots ? zero3 : circ + 3 * node;
            if (h.count == 1) {
              double v1[3], v2[3];
#pragma unroll
              for (int c = 0; c < 3; c++) {
                v1[c] = __dsub_rn(__dadd_rn(C0[c], s[c]), x[c]);
                v2[c] = __dsub_rn(__dadd_rn(__dadd_rn(C0[c], R[c]), s[c]), x[c]);
              }
              const double a = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(v1[0], v1[0]), __dmul_rn(v1[1], v1[1])), __dmul_rn(v1[2], v1[2])));
              const double b = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(v2[0], v2[0]), __dmul_rn(v2[1], v2[1])), __dmul_rn(v2[2], v2[2])));
              const double dv = __dadd_rn(__dadd_rn(__dmul_rn(v1[0], v2[0]), __dmul_rn(v1[1], v2[1])), __dmul_rn(v1[2], v2[2]));
              const double ab = __dmul_rn(a, b);
              const double cc = __dmul_rn(ab, __dadd_rn(ab, dv));
              const double f = __ddiv_rn(__dadd_rn(a, b), cc);
              const double cr[3] = {__dsub_rn(__dmul_rn(v1[1], v2[2]), __dmul_rn(v1[2], v2[1])),
                                    __dsub_rn(__dmul_rn(v1[2], v2[0]), __dmul_rn(v1[0], v2[2])),
                                    __dsub_rn(__dmul_rn(v1[0], v2[1]), __dmul_rn(v1[1], v2[0]))};
#pragma unroll
              for (int c = 0; c < 3; c++)
                acc[c] = __dadd_rn(acc[c], __ddiv_rn(__ddiv_rn(__dmul_rn(f, cr[c]), 4.), QV_PI));
              ev++;
            } else if (th < theta) {
              const double v[3] = {__dsub_rn(x[0], __dadd_rn(C0[0], s[0])),
                                   __dsub_rn(x[1], __dadd_rn(C0[1], s[1])),
                                   __dsub_rn(x[2], __dadd_rn(C0[2], s[2]))};
              const double d2 = __dmul_rn(dist, dist);
              const double d3 = __dmul_rn(d2, dist);
              const double d5 = __dmul_rn(__dmul_rn(d2, d2), dist);
              const WPay64 &P = p64[node];
              double ci[3], Cm[9];
#pragma unroll
              for (int c = 0; c < 3; c++) ci[c] = node < nroots ? 0. : P.a[c];
#pragma unroll
              for (int c = 0; c < 9; c++) Cm[c] = node < nroots ? 0. : P.C[c];
              double ub[3] = {__ddiv_rn(__dsub_rn(__dmul_rn(ci[1], v[2]), __dmul_rn(ci[2], v[1])), d3),
                              __ddiv_rn(__dsub_rn(__dmul_rn(ci[2], v[0]), __dmul_rn(ci[0], v[2])), d3),
                              __ddiv_rn(__dsub_rn(__dmul_rn(ci[0], v[1]), __dmul_rn(ci[1], v[0])), d3)};
              for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) {
                  double vc = __dmul_rn(v[0], Cm[l]);
                  vc = __dadd_rn(vc, __dmul_rn(v[1], Cm[3 + l]));
                  vc = __dadd_rn(vc, __dmul_rn(v[2], Cm[6 + l]));
#pragma unroll
                  for (int mm = 0; mm < 3; mm++) {
                    const double e = (mm == k || k == l || l == mm) ? 0.
                                     : ((mm + 1) % 3 == k ? 1. : -1.);  // eps(m,k,l)
                    ub[mm] = __dsub_rn(ub[mm], __ddiv_rn(__dmul_rn(e, Cm[3 * k + l]), d3));
                  }
#pragma unroll
                  for (int mm = 0; mm < 3; mm++) {
                    const double e = (mm == k || k == l || l == mm) ? 0.
                                     : ((mm + 1) % 3 == k ? 1. : -1.);
                    ub[mm] = __dadd_rn(ub[mm], __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(3., e), v[k]), vc), d5));
                  }
                }
#pragma unroll
              for (int c = 0; c < 3; c++) acc[c] = __dadd_rn(acc[c], ub[c]);
              ev++;
            } else {
              open = true;
            }
          }
        }
        const unsigned om = __ballot_sync(0xffffffffu, open);
        if (om) {
          int nc = h.nchild;
          if (top + nc > STK) {  // unreachable for trees within QV_MAX_DEPTH
            bad = true;
            nc = 0;
          }
          if (lane < nc) st[top + lane] = make_int2(h.child_first + nc - 1 - lane, (int)om);
          top += nc;
        }
        __syncwarp();
      }
    }
    if (live) { u[3 * q] = acc[0]; u[3 * q + 1] = acc[1]; u[3 * q + 2] = acc[2]; }
    for (int o = 16; o > 0; o >>= 1) ev += __shfl_down_sync(0xffffffffu, ev, o);
    if (lane == 0 && ev) atomicAdd(evals, ev);
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, QV_STAT_STACK);
  }
}

extern "C" int qv_field_velocity_tree(qv_ctx *c, int m, const double *pts, double *u,
                                      long long *evals) {
  if (!c || m < 0 || (m > 0 && (!pts || !u))) return QV_ERR_ARG;
  if (!(c->p.tree_theta > 0) || !(c->p.box_size > 0))
    return qv_fail(c, QV_ERR_ARG, "tree_walk_general needs tree_theta > 0 and a box");
  if (m == 0 || c->n == 0) {
    for (int k = 0; k < 3 * m; k++) u[k] = 0.;
    if (evals) *evals = 0;
    return QV_OK;
  }
  int rc;
  if (!c->tree.valid)
    if ((rc = qv_launch_tree_build(c))) return rc;
  if ((rc = qv_tree_finalize_root(c))) return rc;
  TreeBuf &t = c->tree;
  double *dp = nullptr;
  QV_CUDA(c, cudaMalloc((void **)&dp, sizeof(double) * 6 * (size_t)m));
  struct Free {
    double *p;
    ~Free() { cudaFree(p); }
  } guard{dp};  // freed on every return path
  double *du = dp + 3 * (size_t)m;
  QV_CUDA(c, cudaMemcpyAsync(dp, pts, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, c->stream));
  QV_CUDA(c, cudaMemsetAsync(c->evals, 0, sizeof(unsigned long long), c->stream));
  QV_CUDA(c, cudaMemsetAsync(c->dstatus, 0, sizeof(int), c->stream));
  const int nb = std::max(1, std::min((m + 32 * GW - 1) / (32 * GW), 64 * c->sm_count));
  switch (c->p.boundary) {
#define QV_GW_CASE(BCV)                                                                          \
  case BCV:                                                                                      \
    k_walk_general<BCV><<<nb, GW * 32, 0, c->stream>>>(m, dp, t.w64, t.p64, t.cent, t.circ,     \
                                                       c->p.box_size, c->p.tree_theta, 1, du,   \
                                                       c->evals, c->dstatus);                   \
    break;
    QV_GW_CASE(QV_BC_OPEN)
    QV_GW_CASE(QV_BC_PERIODIC)
    QV_GW_CASE(QV_BC_OPENX)
    QV_GW_CASE(QV_BC_OPENXY)
#undef QV_GW_CASE
    default:
      return qv_fail(c, QV_ERR_UNSUPPORTED, "boundary %d not supported", c->p.boundary);
  }
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  unsigned long long ev = 0;
  int st = 0;
  QV_CUDA(c, cudaMemcpyAsync(u, du, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaMemcpyAsync(&ev, c->evals, sizeof(ev), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaMemcpyAsync(&st, c->dstatus, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  if (evals) *evals = (long long)ev;
  if (st & 2) return qv_fail(c, QV_ERR_TREE_DEPTH, "tree_walk_general stack overflow");
  return QV_OK;
}
