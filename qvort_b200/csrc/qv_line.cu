// qv_line.cu -- the line operations of the time loop: pinsert
// (src/line.f90:18-106), precon_original (src/reconnection.f90:145-254) and
// premove with loop_killer (src/line.f90:112-161, src/reconnection.f90:421-461).
//
// All three are sequential scans over the slots in ascending order whose effects
// feed later iterations: an insertion takes the first empty slot (or appends
// one), relinks, and refreshes the stored ghosts of three slots (the new
// point, i, and i's old infront), and a later test of a refreshed slot sees
// the new ghosts; a removal relinks i past its infront, which changes the test
// of i's behind.  Tests on unaffected slots only read state that nothing
// earlier changed.  So:
//   * one parallel pass evaluates every slot's test and compacts the
//     candidates (ascending), plus the empty slots for pinsert;
//   * one device thread then runs the reference's loop over the candidates
//     and the slots an earlier iteration touched (a small min-heap), each
//     re-tested on the current state, with the reference's arithmetic.
// Candidates are few per step (the resolution is maintained every step), so
// the sequential part is short; its state lives in device memory and a run
// that needs more slots than are allocated stops before the insertion that
// needs them, so that the host can grow the arrays and resume it.
//
// Compiled without FMA contraction: positions are computed in the reference's
// order of roundings (gfortran -O2 does not contract either).
#include <algorithm>

#include <cstring>

#include "qv_internal.cuh"
#include "qv_lia.cuh"

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

#define LHEAP 8192  // slots waiting for a re-test (min-heap)

struct LineState {
  int nc, ne;        // candidates, empty slots (written by the compaction)
  int pc, epos;      // next candidate, next empty slot
  int n_old, n_cur;  // slot count at the start (loop bound), current slot count
  int last;          // last slot processed
  int heap_n;
  int status;        // 1: more slots needed, 2: heap overflow
  int done;          // points inserted / removed so far
  int n_clr;         // entries of the cleared-slot log (may exceed its capacity)
  int pad[5];
  int heap[LHEAP];
};

// ------------------------------------------------------------- per slot
__device__ __forceinline__ void ghost_one(int i, const double *__restrict__ x, const int *inf,
                                          const int *beh, double *gi, double *gb, double *gii,
                                          double *gbb, int lo_axis, double L) {
  int a = inf[i], b = beh[i];
  int aa = inf[a - 1], bb = beh[b - 1];
  int src[4] = {a - 1, b - 1, aa - 1, bb - 1};
  double *dst[4] = {gi, gb, gii, gbb};
  double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  double h = L / 2.;
  for (int k = 0; k < 4; k++)
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

struct LineArgs {
  double *x, *u, *u1, *u2, *u3, *gi, *gb, *gii, *gbb, *u_li, *u_bs, *closestd;
  int *inf, *beh, *closest;
  int cap, lo_axis, order;
  double L, delta, thr;
  const int *cand, *empt;
  int *flag_a, *flag_b;
  LineState *st;
  int *dstatus;  // the context's status word (QV_STAT_HEAP: a scan's re-test heap overflowed)
  int *clr;      // cleared-slot log, QV_LINE_CLR_CAP entries
};

// clear_particle, src/general.f90:11-22 (u3 is kept)
__device__ __forceinline__ void clear_slot(const LineArgs &a, int i) {
  for (int c = 0; c < 3; c++) {
    a.x[3 * i + c] = 0.; a.u[3 * i + c] = 0.; a.u1[3 * i + c] = 0.; a.u2[3 * i + c] = 0.;
    a.gi[3 * i + c] = 0.; a.gb[3 * i + c] = 0.; a.gii[3 * i + c] = 0.; a.gbb[3 * i + c] = 0.;
    a.u_li[3 * i + c] = 0.; a.u_bs[3 * i + c] = 0.;
  }
  a.inf[i] = 0;
  a.beh[i] = 0;
  a.closest[i] = 0;
  a.closestd[i] = 0.;
  // the log lets a host copy taken before this scan be corrected afterwards
  const int k = atomicAdd(&a.st->n_clr, 1);
  if (k < QV_LINE_CLR_CAP) a.clr[k] = i;
}

__device__ __forceinline__ double seg_len(const double *a, const double *b) {
  return lia_dist(a, b);  // dist_gen, src/derivatives.f90:79-86
}

// ------------------------------------------------------------ detection
// Reset of the sequential state for a scan over n slots (done by the flag
// kernel that starts each scan; the compaction then writes nc / ne).
__device__ __forceinline__ void begin_state(LineState *s, int n) {
  s->pc = 0; s->epos = 0; s->n_old = n; s->n_cur = n; s->last = -1; s->heap_n = 0;
  s->status = 0; s->done = 0;
}

// pinsert's test on the stored ghosts (src/line.f90:41,49) and the empty slots.
__global__ void k_ins_flags(int n, LineArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    begin_state(a.st, n);
    a.st->n_clr = 0;  // a step's line operations start with pinsert: a fresh cleared-slot log
  }
  if (i >= n) return;
  int act = a.inf[i] != 0;
  a.flag_b[i] = !act;
  a.flag_a[i] = act && seg_len(a.x + 3 * i, a.gi + 3 * i) > 1. * a.delta;
}

// premove's test: |x_i - x_infront(infront(i))| on raw positions (src/line.f90:131-137).
__device__ __forceinline__ bool remove_test(const LineArgs &a, int i) {
  int j = a.inf[a.inf[i] - 1] - 1;
  const double *xi = a.x + 3 * i, *xj = a.x + 3 * j;
  double d0 = xi[0] - xj[0], d1 = xi[1] - xj[1], d2 = xi[2] - xj[2];
  return sqrt(d0 * d0 + d1 * d1 + d2 * d2) < a.thr;
}

__global__ void k_rem_flags(int n, LineArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) begin_state(a.st, n);
  if (i >= n) return;
  a.flag_a[i] = a.inf[i] != 0 && remove_test(a, i);
}

// ------------------------------------------------------------- worklist
__device__ void heap_push(LineState *s, int *dstatus, int v) {
  if (s->heap_n >= LHEAP) {
    s->status = 2;
    atomicOr(dstatus, QV_STAT_HEAP);
    return;
  }
  int k = s->heap_n++;
  s->heap[k] = v;
  while (k > 0) {
    int p = (k - 1) / 2;
    if (s->heap[p] <= s->heap[k]) break;
    int t = s->heap[p]; s->heap[p] = s->heap[k]; s->heap[k] = t;
    k = p;
  }
}

__device__ void heap_pop(LineState *s) {
  s->heap[0] = s->heap[--s->heap_n];
  int k = 0;
  for (;;) {
    int l = 2 * k + 1, r = l + 1, m = k;
    if (l < s->heap_n && s->heap[l] < s->heap[m]) m = l;
    if (r < s->heap_n && s->heap[r] < s->heap[m]) m = r;
    if (m == k) break;
    int t = s->heap[m]; s->heap[m] = s->heap[k]; s->heap[k] = t;
    k = m;
  }
}

// The next slot above `last` from the candidates and the heap (-1: none).
__device__ int next_slot(LineState *s, const int *cand) {
  while (s->pc < s->nc && cand[s->pc] <= s->last) s->pc++;
  while (s->heap_n > 0 && s->heap[0] <= s->last) heap_pop(s);
  int c = s->pc < s->nc ? cand[s->pc] : -1;
  int h = s->heap_n > 0 ? s->heap[0] : -1;
  if (c < 0) return h;
  if (h < 0) return c;
  return min(c, h);
}

// ------------------------------------------------------------- pinsert
__global__ void k_pinsert_seq(LineArgs a) {
  LineState *s = a.st;
  if (s->status) return;
  for (;;) {
    const int i = next_slot(s, a.cand);
    if (i < 0) break;
    if (a.inf[i] == 0) { s->last = i; continue; }
    const double disti = seg_len(a.x + 3 * i, a.gi + 3 * i);
    if (!(disti > 1. * a.delta)) { s->last = i; continue; }
    int par;
    if (s->epos < s->ne) {
      par = a.empt[s->epos];
    } else {
      if (s->n_cur >= a.cap) {  // stop before this insertion; the host grows and resumes
        s->status = 1;
        return;
      }
      par = s->n_cur;
      for (int c = 0; c < 3; c++) { a.u3[3 * par + c] = 0.; a.u_li[3 * par + c] = 0.; a.u_bs[3 * par + c] = 0.; }
      a.closest[par] = 0;
      a.closestd[par] = 0.;
    }
    s->last = i;
    if (s->epos < s->ne) s->epos++;
    else s->n_cur++;
    // new position: midpoint moved onto the circle of the local curvature
    // (src/line.f90:68-85)
    double X[3], GI[3], GB[3], GII[3], GBB[3], s1[3], fdd[3];
    for (int c = 0; c < 3; c++) {
      X[c] = a.x[3 * i + c]; GI[c] = a.gi[3 * i + c]; GB[c] = a.gb[3 * i + c];
      GII[c] = a.gii[3 * i + c]; GBB[c] = a.gbb[3 * i + c];
    }
    lia_derivs(a.order, X, GI, GB, GII, GBB, s1, fdd);  // get_deriv_2
    double curv = sqrt(fdd[0] * fdd[0] + fdd[1] * fdd[1] + fdd[2] * fdd[2]);
    double xn[3];
    if (curv > 1E-5) {
      curv = 1. / curv;
      if (curv * curv - 0.25 * (disti * disti) > 0.) {
        double f = (sqrt(curv * curv - 0.25 * (disti * disti)) - curv) * curv;
        for (int c = 0; c < 3; c++) xn[c] = 0.5 * (X[c] + GI[c]) + f * fdd[c];
      } else {
        for (int c = 0; c < 3; c++) xn[c] = 0.5 * (X[c] + GI[c]);
      }
    } else {
      for (int c = 0; c < 3; c++) xn[c] = 0.5 * (X[c] + GI[c]);
    }
    const int ao = a.inf[i] - 1;  // old infront
    for (int c = 0; c < 3; c++) {
      a.x[3 * par + c] = xn[c];
      a.u[3 * par + c] = 0.5 * (a.u[3 * i + c] + a.u[3 * ao + c]);
      a.u1[3 * par + c] = 0.;
      a.u2[3 * par + c] = 0.;
    }
    a.beh[par] = i + 1;
    a.inf[par] = a.inf[i];
    ghost_one(par, a.x, a.inf, a.beh, a.gi, a.gb, a.gii, a.gbb, a.lo_axis, a.L);
    a.beh[ao] = par + 1;
    ghost_one(ao, a.x, a.inf, a.beh, a.gi, a.gb, a.gii, a.gbb, a.lo_axis, a.L);
    a.inf[i] = par + 1;
    ghost_one(i, a.x, a.inf, a.beh, a.gi, a.gb, a.gii, a.gbb, a.lo_axis, a.L);
    s->done++;
    // slots whose stored ghosts changed and that the loop still visits
    if (ao > i && ao < s->n_old) heap_push(s, a.dstatus, ao);
    if (par > i && par < s->n_old) heap_push(s, a.dstatus, par);
    if (s->status) return;
  }
}

// ------------------------------------------------------------- premove
// loop_killer (src/reconnection.f90:421-461): only whether the loop has fewer
// than 5 points matters, so the count stops at 5.
__device__ int loop_killer(const LineArgs &a, int particle) {
  int counter = 1, next = particle;
  for (int k = 0; k < 5; k++) {
    next = a.inf[next] - 1;
    if (next == particle || next < 0) break;
    counter++;
  }
  if (counter >= 5) return 0;
  next = particle;
  for (int k = 0; k < 5; k++) {
    int store_next = a.inf[next] - 1;
    clear_slot(a, next);
    next = store_next;
    if (next == particle || next < 0) break;
  }
  return counter;
}

__global__ void k_premove_seq(LineArgs a) {
  LineState *s = a.st;
  if (s->status) return;
  for (;;) {
    const int i = next_slot(s, a.cand);
    if (i < 0) break;
    s->last = i;
    if (a.inf[i] == 0 || !remove_test(a, i)) continue;
    const int r = a.inf[i] - 1, t = a.inf[r] - 1;  // removed point, its infront
    a.beh[t] = i + 1;
    a.inf[i] = t + 1;
    clear_slot(a, r);
    s->done += 1 + loop_killer(a, i);
    // i's behind now reaches a different point two ahead
    if (a.inf[i] != 0) {
      const int b = a.beh[i] - 1;
      if (b > i && b < s->n_old) heap_push(s, a.dstatus, b);
    }
    if (s->status) return;
  }
}

// ------------------------------------------------------------- precon
// precon_original (src/reconnection.f90:145-254): its candidates are the
// active slots whose last search found a partner closer than delta/2 (and
// farther than epsilon) -- closestd is not changed by the scan, so the list is
// fixed before it runs; each candidate is then tested on the current links.
__global__ void k_rec_flags(int n, LineArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) begin_state(a.st, n);
  if (i >= n) return;
  double cd = a.closestd[i];
  a.flag_a[i] = a.inf[i] != 0 && (cd < a.delta / 2.) && (cd > QV_DEPS);
}

// norm_tanf, src/general.f90:94-107: get_deriv_1 on the stored ghosts, normalised.
__device__ void norm_tan(const LineArgs &a, int i, double *t) {
  double X[3], GI[3], GB[3], GII[3], GBB[3], s2[3];
  for (int c = 0; c < 3; c++) {
    X[c] = a.x[3 * i + c]; GI[c] = a.gi[3 * i + c]; GB[c] = a.gb[3 * i + c];
    GII[c] = a.gii[3 * i + c]; GBB[c] = a.gbb[3 * i + c];
  }
  lia_derivs(a.order, X, GI, GB, GII, GBB, t, s2);
  double length = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  for (int c = 0; c < 3; c++) t[c] = t[c] / length;
}

// What of a candidate's test does not depend on the links -- the tangents and
// their dot product, the length before, the first three terms of the length
// after (positions and stored ghosts, which precon does not change) -- is
// evaluated for all candidates in parallel; the ordered pass re-reads the
// links and recomputes only the last term when they have changed.
struct RecEval {
  int j, pari, parjb, parallel;
  double l_before, s3, l_after;
  int maybe;  // the test, on the links at the start of the pass, reconnects
  int pad;
};

__global__ void k_rec_eval(int n, LineArgs a, RecEval *rec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n || q >= a.st->nc) return;
  const int i = a.cand[q];
  RecEval r;
  r.j = a.closest[i] - 1;
  r.pari = a.inf[i] - 1;
  r.parjb = -1;
  r.parallel = 1;
  r.l_before = r.s3 = r.l_after = 0.;
  if (r.j >= 0 && a.inf[r.j] != 0) {
    const int j = r.j;
    r.parjb = a.beh[j] - 1;
    double t1[3], t2[3];
    norm_tan(a, i, t1);
    norm_tan(a, j, t2);
    const double dot_val = t1[0] * t2[0] + t1[1] * t2[1] + t1[2] * t2[2];
    r.parallel = dot_val > 0.9;
    const double *xi = a.x + 3 * i, *xj = a.x + 3 * j;
    r.l_before = seg_len(xi, a.gi + 3 * i) + seg_len(xi, a.gb + 3 * i) +
                 seg_len(xj, a.gi + 3 * j) + seg_len(xj, a.gb + 3 * j);
    r.s3 = seg_len(xi, a.gb + 3 * i) + seg_len(xi, xj) + seg_len(xj, a.gi + 3 * j);
    r.l_after = r.s3 + seg_len(a.x + 3 * r.pari, a.x + 3 * r.parjb);
  }
  // the ordered pass's test on the links as they are now (src/reconnection.f90:163-190)
  const int parb = a.beh[i] - 1;
  r.maybe = a.inf[i] != 0 && r.j >= 0 && r.j != r.pari && r.j != parb && a.inf[r.j] != 0 &&
            !r.parallel && r.l_after <= r.l_before;
  r.pad = 0;
  rec[q] = r;
}

// The ordered pass of precon_original.  A candidate's test reads the links of
// its own slot i and of its partner j (and positions, which the pass changes
// only in the slots loop_killer clears, whose links it clears too).  So while
// neither i's nor j's links have changed since the pass began, the test gives
// what it gave on the starting links, which k_rec_eval evaluated for every
// candidate (maybe).  The block therefore scans the candidates in order, a
// window of PC_T at a time, for the first that either reconnects on the
// starting links or has a slot whose links the pass has changed, and thread 0
// runs the reference's test on the current links for that one only: every
// candidate skipped would have done nothing.  The changed slots (the four
// relinked ones and those loop_killer clears, from the cleared-slot log) are
// listed in shared memory; past PC_CHG of them every candidate is tested.
#define PC_T 256
#define PC_CHG 1024
__device__ __forceinline__ bool pc_changed(const int *chg, int nchg, int slot) {
  for (int k = 0; k < nchg; k++)
    if (chg[k] == slot) return true;
  return false;
}

__global__ void __launch_bounds__(PC_T) k_precon_scan(LineArgs a, const RecEval *rec) {
  __shared__ int chg[PC_CHG];
  __shared__ int nchg, first;
  LineState *s = a.st;
  const int nc = s->nc, pc0 = s->pc;
  const int tid = threadIdx.x;
  if (tid == 0) nchg = 0;
  int done = 0;
  for (int pos = pc0; pos < nc;) {
    __syncthreads();
    if (tid == 0) first = PC_T;
    __syncthreads();
    const int q = pos + tid;
    if (q < nc) {
      const int n_c = nchg;
      bool hit = rec[q].maybe != 0 || n_c > PC_CHG;
      if (!hit && n_c > 0) {
        const int j = rec[q].j;
        hit = pc_changed(chg, n_c, a.cand[q]) || (j >= 0 && pc_changed(chg, n_c, j));
      }
      if (hit) atomicMin(&first, tid);
    }
    __syncthreads();
    const int f = first;
    if (f == PC_T) {
      pos += PC_T;
      continue;
    }
    if (tid == 0) {
      const int qq = pos + f, i = a.cand[qq];
      const RecEval r = rec[qq];
      const int infi = a.inf[i];
      const int pari = infi - 1, parb = a.beh[i] - 1, j = r.j;
      // src/reconnection.f90:163-190 on the current links
      if (infi != 0 && j >= 0 && j != pari && j != parb && a.inf[j] != 0 && !r.parallel) {
        const int parjb = a.beh[j] - 1;
        const double l_after = (pari == r.pari && parjb == r.parjb)
                                   ? r.l_after
                                   : r.s3 + seg_len(a.x + 3 * pari, a.x + 3 * parjb);
        if (l_after <= r.l_before) {
          a.inf[parjb] = pari + 1;
          a.beh[pari] = parjb + 1;
          a.inf[i] = j + 1;
          a.beh[j] = i + 1;
          const int c0 = s->n_clr;
          loop_killer(a, pari);
          loop_killer(a, i);
          const int c1 = s->n_clr;
          int m = nchg;
          const int mine[4] = {parjb, pari, i, j};
          for (int k = 0; k < 4; k++, m++)
            if (m < PC_CHG) chg[m] = mine[k];
          for (int k = c0; k < c1; k++, m++)
            if (m < PC_CHG) chg[m] = k < QV_LINE_CLR_CAP ? a.clr[k] : -1;
          if (c1 > QV_LINE_CLR_CAP) m = PC_CHG + 1;  // the log lost entries: test them all
          nchg = m;
          done++;
        }
      }
    }
    pos += f + 1;
  }
  if (tid == 0) {
    s->pc = max(nc, pc0);
    s->done += done;
  }
}

// --------------------------------------------------------------- host
// Flag and list arrays for n slots (the slot count at the start of a scan).
static int line_reserve(qv_ctx *c) {
  size_t n = (size_t)std::max(c->n, 1);
  if (c->line_cap >= n && c->line_st) return QV_OK;
  int rc;
  if ((rc = qv_grow(c, (void **)&c->line_flags, sizeof(int) * 4 * n))) return rc;
  if ((rc = qv_grow(c, (void **)&c->line_rec, sizeof(RecEval) * n))) return rc;
  if (!c->line_st) {
    if ((rc = qv_grow(c, (void **)&c->line_st, sizeof(LineState)))) return rc;
    QV_CUDA(c, cudaMemsetAsync(c->line_st, 0, sizeof(LineState), c->stream));
  }
  if (!c->line_clr)
    if ((rc = qv_grow(c, (void **)&c->line_clr, sizeof(int) * QV_LINE_CLR_CAP))) return rc;
  c->line_cap = n;
  return QV_OK;
}

static LineArgs line_args(qv_ctx *c) {
  LineArgs a;
  a.x = c->x; a.u = c->u; a.u1 = c->u1; a.u2 = c->u2; a.u3 = c->u3;
  a.gi = c->gi; a.gb = c->gb; a.gii = c->gii; a.gbb = c->gbb;
  a.u_li = c->u_li; a.u_bs = c->u_bs; a.closestd = c->closestd;
  a.inf = c->infront; a.beh = c->behind; a.closest = c->closest;
  a.cap = c->cap;
  a.lo_axis = c->p.boundary == QV_BC_PERIODIC ? 0 : c->p.boundary == QV_BC_OPENX ? 1
              : c->p.boundary == QV_BC_OPENXY ? 2 : 3;
  a.order = c->p.deriv_order;
  a.L = c->p.box_size;
  a.delta = c->p.delta;
  a.thr = .499 * c->p.delta * (1. + 1.);
  int *f = (int *)c->line_flags;
  size_t n = c->line_cap;
  a.flag_a = f;
  a.flag_b = f + n;
  a.cand = f + 2 * n;
  a.empt = f + 3 * n;
  a.st = (LineState *)c->line_st;
  a.dstatus = c->dstatus;
  a.clr = c->line_clr;
  return a;
}

// Ordered compaction of flag[0..n) into out (one block up to QV_COMPACT1_MAX
// slots, else count / scan / scatter); the count goes to *total on the device.
static int compact_flags(qv_ctx *c, int n, const int *flag, int *out, int *total) {
  if (n <= QV_COMPACT1_MAX) {
    k_compact1<<<1, 1024, 0, c->stream>>>(n, flag, out, total);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    return QV_OK;
  }
  int nb = nblk(n, 256);
  int *tmp = c->blkcnt;
  k_count_active<<<nb, 256, 0, c->stream>>>(n, flag, tmp);
  k_scan_small<<<1, 1024, 0, c->stream>>>(nb, tmp, total);
  k_scatter_active<<<nb, 256, 0, c->stream>>>(n, flag, tmp, out);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 3);
  return QV_OK;
}

static int read_state(qv_ctx *c, LineState *h) {
  QV_CUDA(c, cudaMemcpyAsync(h, c->line_st, offsetof(LineState, heap), cudaMemcpyDeviceToHost,
                             c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  return QV_OK;
}

// The state's copy to pinned host memory, queued now and waited for later
// (only for it, not for what is queued behind it).
static int queue_state_copy(qv_ctx *c) {
  if (!c->line_host) {
    QV_CUDA(c, cudaMallocHost(&c->line_host, offsetof(LineState, heap)));
    QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_line, cudaEventDisableTiming));
  }
  QV_CUDA(c, cudaMemcpyAsync(c->line_host, c->line_st, offsetof(LineState, heap),
                             cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaEventRecord(c->ev_line, c->stream));
  return QV_OK;
}

static int wait_state_copy(qv_ctx *c, LineState *h) {
  QV_CUDA(c, cudaEventSynchronize(c->ev_line));
  memcpy(h, c->line_host, offsetof(LineState, heap));
  return QV_OK;
}

static __global__ void k_line_clear_status(LineState *s) { s->status = 0; }

int qv_line_insert_queue(qv_ctx *c) {
  int rc;
  if (c->n == 0) return QV_OK;
  // pinsert reads the stored ghosts; compute them only if none exist yet
  if (!c->ghosts_stored)
    if ((rc = qv_launch_ghosts(c))) return rc;
  // room for insertions past the last slot: grow (keeping the points) so that
  // at least an eighth of the slots, or 4096, are free
  int want = c->n + std::max(4096, c->n / 8);
  if (c->cap < c->n + 1024)
    if ((rc = qv_grow_points(c, want))) return rc;
  if ((rc = line_reserve(c))) return rc;
  LineArgs a = line_args(c);
  const int n = c->n;
  k_ins_flags<<<nblk(n, 256), 256, 0, c->stream>>>(n, a);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  if ((rc = compact_flags(c, n, a.flag_a, (int *)a.cand, &a.st->nc))) return rc;
  if ((rc = compact_flags(c, n, a.flag_b, (int *)a.empt, &a.st->ne))) return rc;
  k_pinsert_seq<<<1, 1, 0, c->stream>>>(a);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  if (!c->ev_pins) QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_pins, cudaEventDisableTiming));
  QV_CUDA(c, cudaEventRecord(c->ev_pins, c->stream));
  return queue_state_copy(c);
}

int qv_line_insert_finish(qv_ctx *c, int *inserted, bool *resumed) {
  int rc;
  if (resumed) *resumed = false;
  if (c->n == 0) { if (inserted) *inserted = 0; return QV_OK; }
  LineArgs a = line_args(c);
  LineState h;
  for (int attempt = 0; attempt < 16; attempt++) {
    if ((rc = wait_state_copy(c, &h))) return rc;
    if (h.status != 1) break;
    // more slots than allocated: grow the point arrays, keeping every slot in
    // use including those appended so far (the candidate and empty-slot lists
    // keep their size), and resume where the scan stopped
    if (resumed) *resumed = true;
    QV_CUDA(c, cudaStreamSynchronize(c->stream));  // work queued behind pinsert is done
    c->n = h.n_cur;
    if ((rc = qv_grow_points(c, c->cap + std::max(4096, c->cap / 4)))) return rc;
    a = line_args(c);
    k_line_clear_status<<<1, 1, 0, c->stream>>>(a.st);
    k_pinsert_seq<<<1, 1, 0, c->stream>>>(a);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 2);
    if ((rc = queue_state_copy(c))) return rc;
  }
  if (h.status == 1) return qv_fail(c, QV_ERR_NOMEM, "pinsert: slot growth did not converge");
  if (h.status == 2) return qv_fail(c, QV_ERR_STATE, "pinsert: more than %d re-tests pending", LHEAP);
  c->n = h.n_cur;
  if (inserted) *inserted = h.done;
  return QV_OK;
}

int qv_line_insert(qv_ctx *c, int *inserted) {
  int rc;
  if ((rc = qv_line_insert_queue(c))) return rc;
  return qv_line_insert_finish(c, inserted, nullptr);
}

const int *qv_line_count_dev(qv_ctx *c) { return &((LineState *)c->line_st)->n_cur; }

int qv_line_clear_log_reset(qv_ctx *c) {
  int rc;
  if ((rc = line_reserve(c))) return rc;
  QV_CUDA(c, cudaMemsetAsync(&((LineState *)c->line_st)->n_clr, 0, sizeof(int), c->stream));
  return QV_OK;
}

int qv_line_clear_log_queue(qv_ctx *c) {
  if (!c->line_st || !c->line_clr) return qv_fail(c, QV_ERR_STATE, "no cleared-slot log");
  if (!c->h_clr)
    QV_CUDA(c, cudaHostAlloc((void **)&c->h_clr, sizeof(int) * (QV_LINE_CLR_HOST + 1),
                             cudaHostAllocDefault));
  const cudaMemcpyKind d2h = cudaMemcpyDeviceToHost;
  QV_CUDA(c, cudaMemcpyAsync(c->h_clr, &((LineState *)c->line_st)->n_clr, sizeof(int), d2h,
                             c->stream));
  QV_CUDA(c, cudaMemcpyAsync(c->h_clr + 1, c->line_clr, sizeof(int) * QV_LINE_CLR_HOST, d2h,
                             c->stream));
  return QV_OK;
}
const int *qv_line_status_dev(qv_ctx *c) { return &((LineState *)c->line_st)->status; }

int qv_line_reconnect(qv_ctx *c, int *count) {
  int rc;
  if (c->n == 0) { if (count) *count = 0; return QV_OK; }
  if ((rc = line_reserve(c))) return rc;
  LineArgs a = line_args(c);
  const int n = c->n;
  k_rec_flags<<<nblk(n, 256), 256, 0, c->stream>>>(n, a);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  if ((rc = compact_flags(c, n, a.flag_a, (int *)a.cand, &a.st->nc))) return rc;
  RecEval *rec = (RecEval *)c->line_rec;
  k_rec_eval<<<nblk(n, 128), 128, 0, c->stream>>>(n, a, rec);
  k_precon_scan<<<1, PC_T, 0, c->stream>>>(a, rec);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 2);
  if (count) {
    LineState h;
    if ((rc = read_state(c, &h))) return rc;
    *count = h.done;
  }
  return QV_OK;
}

int qv_line_remove(qv_ctx *c, int *removed) {
  int rc;
  if (c->n == 0) { if (removed) *removed = 0; return QV_OK; }
  if ((rc = line_reserve(c))) return rc;
  LineArgs a = line_args(c);
  const int n = c->n;
  k_rem_flags<<<nblk(n, 256), 256, 0, c->stream>>>(n, a);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  if ((rc = compact_flags(c, n, a.flag_a, (int *)a.cand, &a.st->nc))) return rc;
  k_premove_seq<<<1, 1, 0, c->stream>>>(a);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  // without a count to return, an overflow is reported through the status
  // word at the step's end instead of a wait here
  if (removed) {
    LineState h;
    if ((rc = read_state(c, &h))) return rc;
    if (h.status == 2) return qv_fail(c, QV_ERR_STATE, "premove: more than %d re-tests pending", LHEAP);
    *removed = h.done;
  }
  return QV_OK;
}
