// qv_tree.cu -- the octree of construct_tree / build_tree / new_tree
// (src/tree.f90:44-186), built bit-exactly on the GPU.
//
// What "bit-exact" has to reproduce:
//  * cell corners are formed by repeated FP64 additions pos + width/2 along
//    the path from the root (src/tree.f90:92-114), and membership is the
//    half-open test x >= pos, x < pos + width on every axis
//    (src/tree.f90:148-150).  Rounding in those additions can leave a point of
//    a parent in no child; such a point is counted by the parent only.
//  * the root counts every slot, empty ones included (src/tree.f90:51); its
//    centroid is the masked mean of all active points; its circ and Cij are 0.
//  * every other node's moments are sequential FP64 sums over its points in
//    ascending slot order (src/tree.f90:146-179): cent = sum x / n,
//    circ = (circ + ghosti) - x, Cij(:,k) += x (ghosti_k - x_k), then
//    Cij(i,k) -= cent_i circ_k.
//
// How: a level-synchronous build in one cooperative kernel.  Each point of a
// splitting node gets its child digit (0..7 in fbl..btr order, 8 = in no
// child) from the node's corner with __dadd_rn arithmetic; a stable segmented
// partition by digit then yields, for every level, an order array in which
// each node's points are contiguous and still in ascending slot order (the
// key (node prefix, slot) -- the Morton-style ordering, radix-partitioned one
// octal digit per level).  A separate kernel runs the moment chains of all
// nodes of all levels concurrently, one warp per node, with explicit
// round-to-nearest FP64 intrinsics so no FMA contraction changes a bit.
#include <climits>
#include <cooperative_groups.h>

#include "qv_internal.cuh"

namespace cg = cooperative_groups;

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

#define BT 256       // build threads per block
#define PPT 4        // positions per thread in a chunk
#define CH (BT * PPT)  // positions per chunk
#define NOD 0xFF     // digit marker: position not in a splitting node

// control block layout
#define CTL_NNODES 0
#define CTL_NGLOB 1     // nodes made by the grid-wide levels (all nodes of > LCH points)
#define CTL_LOCALD 2    // first block-local level, -1 if none
#define CTL_OVERFLOW 3  // 1 = node capacity, 2 = level capacity
#define CTL_NMID 7      // number of nodes handled by the second k_moments_big
#define CTL_DEPTH 4
#define CTL_NBIG 5      // number of nodes handled by k_moments_big
#define CTL_NACT 6      // active points of this build
#define CTL_LVL 8       // lvl_start[0..QV_MAX_DEPTH+2]
#define CTL_NS (CTL_LVL + QV_MAX_DEPTH + 4)  // splitting nodes per level
#define CTL_MAXC (CTL_NS + QV_MAX_DEPTH + 4) // largest splitting node per level
#define CTL_SIZE (CTL_MAXC + QV_MAX_DEPTH + 4)
#define LPT 4             // positions per thread in the block-local levels
#define LMAX (BT * LPT)   // positions per block-local range (whole nodes)
#define LCH (LMAX / 2)    // largest splitting node handed to the block-local levels

struct BuildArgs {
  const int *d_nact;  // active points (device-resident count of the compaction)
  int n_slots, cap_pts, cap_nodes, cap_levels, nchunks;
  const double *x, *gi;
  double *pos, *width;
  int *count, *start, *parent, *child_first, *nchild, *level;
  unsigned char *digit, *cmask;
  int *ord, *nodeA, *nodeB, *rnk, *cnt9A, *cnt9B, *rs9, *chunk9, *ctl;
  unsigned char *dig;
  int *perm;  // out: final (depth-first) order of the active points
};

// What pack_node needs.
struct PackArgs {
  int nroots;
  const double *pos, *width, *cent, *circ, *C;
  const int *count, *child_first, *nchild;
  const unsigned char *cmask;
  const int *first;
  const double *x, *gi;
  const int *inf, *beh;
  double theta;
  int extra;
  WNode64 *w64;
  WPay64 *p64;
  WNode32 *w32;
  SNode32 *c32;
  WPay32 *p32;
  int *leaf_of;
  int n_leaf;
  int full;  // also the FP64 walk payload and the search header (a forest needs neither)
};
__device__ void pack_one(const PackArgs &P, int k, int what);
static_assert(QV_L1_BIG == LCH, "the late level-1 nodes are the big-chain nodes of level 1");

// packed per-digit counters: digits 0..4 in lo (12-bit fields), 5..8 in hi
struct Pack2 {
  unsigned long long lo, hi;
};
__device__ __forceinline__ Pack2 pk_one(int g) {
  Pack2 r{0ull, 0ull};
  if (g < 5) r.lo = 1ull << (12 * g);
  else if (g < 9) r.hi = 1ull << (12 * (g - 5));
  return r;
}
__device__ __forceinline__ int pk_get(const Pack2 &p, int g) {
  return g < 5 ? (int)((p.lo >> (12 * g)) & 0xFFF) : (int)((p.hi >> (12 * (g - 5))) & 0xFFF);
}

// Block-wide exclusive scan of Pack2 (BT threads); returns exclusive prefix
// and writes the block total to *tot (all threads).
__device__ Pack2 block_scan_pack(Pack2 v, Pack2 *tot, Pack2 *sh) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Pack2 inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long a = __shfl_up_sync(0xffffffffu, inc.lo, o);
    unsigned long long b = __shfl_up_sync(0xffffffffu, inc.hi, o);
    if (lane >= o) { inc.lo += a; inc.hi += b; }
  }
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    Pack2 r{0ull, 0ull};
    for (int k = 0; k < BT / 32; k++) {
      Pack2 t = sh[k];
      sh[k] = r;
      r.lo += t.lo; r.hi += t.hi;
    }
    sh[BT / 32] = r;
  }
  __syncthreads();
  Pack2 ex;
  ex.lo = sh[wid].lo + inc.lo - v.lo;
  ex.hi = sh[wid].hi + inc.hi - v.hi;
  *tot = sh[BT / 32];
  __syncthreads();
  return ex;
}

// child digit of point X in the node with corner P and width W
// (src/tree.f90:92-114, 148-150).  8 = in no child.
__device__ __forceinline__ int child_digit(const double *X, const double *P, double W) {
  double w = W * 0.5;
  int b[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double cm = __dadd_rn(P[c], w);   // child corner (right) = upper bound (left)
    double up = __dadd_rn(cm, w);     // upper bound (right)
    if (X[c] >= P[c] && X[c] < cm) b[c] = 0;
    else if (X[c] >= cm && X[c] < up) b[c] = 1;
    else b[c] = -1;
  }
  if (b[0] < 0 || b[1] < 0 || b[2] < 0) return 8;
  return b[0] + 2 * b[2] + 4 * b[1];
}

// Block-local levels.  Once every splitting node of level d0 holds at most LCH
// points, the positions [0, n_act) are cut into ranges of whole nodes: range c
// runs from the start of the node holding position c*LCH (or that position, if
// its node does not split) to the same point of range c+1, so a range holds
// fewer than 2*LCH positions (bounds in chunk9[0..nch], written before a grid
// barrier).  A block then runs the remaining levels of its range with block
// barriers instead of grid barriers: the same child digits, the same stable
// partition (ranks from one block-wide scan of packed digit counts, a node's
// counts from the scan at its first and one-past-last positions) and the same
// node records; child ids are claimed with one atomic per block and level, and
// each child's record is written by its first point.  Each position's slot,
// node, node start and count travel with it in shared memory, so a level costs
// one batched gather of (x, corner, width) and one atomic; the order rows are
// written for the moment chains and the final order for the walks.  Node ids
// are not ordered by level in this part, which nothing downstream needs.
struct LocalSmem {
  Pack2 exs[LMAX + 1];  // exclusive digit-count prefix at each position
  int ordl[LMAX];       // slot at each position
  int nodl[LMAX];       // node at each position (-1: in no splitting node)
  int scl[LMAX];        // node start (relative) | node count << 16
  int cfl[LMAX];        // at a node's first position: its first child
  int cml[LMAX];        // at a node's first position: its child mask
};
#define LOCAL_SMEM ((int)sizeof(LocalSmem))

__device__ __forceinline__ int fld12(unsigned long long v, int f) {
  return (int)((v >> (12 * f)) & 0xFFF);
}
// Position offset of digit g's group inside a node whose packed per-digit
// counts are D: the exclusive prefix sum of D's fields, taken for all fields
// at once by multiplying with 1 + 2^12 + 2^24 + ... (no field exceeds 12 bits).
__device__ __forceinline__ int digit_offset(const Pack2 &D, int g) {
  const unsigned long long ilo = D.lo * 0x001001001001001ull;
  if (g < 5) return fld12(ilo, g) - fld12(D.lo, g);
  const unsigned long long ihi = D.hi * 0x001001001001ull;
  return fld12(ilo, 4) + fld12(ihi, g - 5) - fld12(D.hi, g - 5);
}

__device__ void build_local(const BuildArgs &a, const int d0, const int n_act, Pack2 *sh,
                            LocalSmem &L) {
  __shared__ int s_base, s_more, s_split, s_stop;
  __shared__ int wsum[BT / 32 + 1];
  volatile int *ctl = a.ctl;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nch = (n_act + LCH - 1) / LCH;
  const int *nod0 = (d0 & 1) ? a.nodeB : a.nodeA;
  const int *ord0 = a.ord + (size_t)d0 * a.cap_pts;
  int depth = d0;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int P0 = a.chunk9[c], P1 = a.chunk9[c + 1], m = P1 - P0;
    for (int q = tid; q < m; q += BT) {
      const int k = nod0[P0 + q];
      L.ordl[q] = ord0[P0 + q];
      L.nodl[q] = k;
      L.scl[q] = k >= 0 ? (a.start[k] - P0) | (a.count[k] << 16) : 0;
    }
    __syncthreads();
    int d = d0;
    for (;;) {
      int *ordn = a.ord + (size_t)(d + 1) * a.cap_pts;
      // digits of this thread's positions (one batched gather)
      int gs[LPT], ks[LPT], ss[LPT], sc[LPT];
      double X[LPT][3], P[LPT][3], Wd[LPT];
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        const int q = tid * LPT + j;
        ks[j] = q < m ? L.nodl[q] : -1;
        ss[j] = q < m ? L.ordl[q] : 0;
        sc[j] = q < m ? L.scl[q] : 0;
        gs[j] = NOD;
      }
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        const bool sp = ks[j] >= 0 && (sc[j] >> 16) >= 2;
        const int s = sp ? ss[j] : 0, k = sp ? ks[j] : 0;
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
          X[j][cc] = a.x[3 * s + cc];
          P[j][cc] = a.pos[3 * k + cc];
        }
        Wd[j] = a.width[k];
      }
      Pack2 loc{0ull, 0ull};
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        if (ks[j] >= 0 && (sc[j] >> 16) >= 2) {
          const int g = child_digit(X[j], P[j], Wd[j]);
          gs[j] = g;
          Pack2 o = pk_one(g);
          loc.lo += o.lo; loc.hi += o.hi;
        }
      }
      Pack2 tot;
      Pack2 run = block_scan_pack(loc, &tot, sh);
      Pack2 mine[LPT];
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        mine[j] = run;
        L.exs[tid * LPT + j] = run;
        if (gs[j] != NOD) {
          Pack2 o = pk_one(gs[j]);
          run.lo += o.lo; run.hi += o.hi;
        }
      }
      if (tid == 0) {
        L.exs[LMAX] = tot;
        s_more = 0;
        s_split = 0;
      }
      __syncthreads();
      // splitting nodes that start here: child count and mask (first position's thread)
      int nct = 0;
      unsigned msk[LPT];
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        const int q = tid * LPT + j, st = sc[j] & 0xFFFF;
        msk[j] = 0;
        if (gs[j] != NOD && q == st) {
          const Pack2 e = L.exs[q + (sc[j] >> 16)];
          const Pack2 D{e.lo - mine[j].lo, e.hi - mine[j].hi};
#pragma unroll
          for (int g = 0; g < 8; g++) {
            const int cg = g < 5 ? fld12(D.lo, g) : fld12(D.hi, g - 5);
            if (cg > 0) msk[j] |= 1u << g;
            if (cg >= 2) s_more = 1;
          }
          nct += __popc(msk[j]);
        }
      }
      int inc = nct;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      if (lane == 31) wsum[wid] = inc;
      __syncthreads();
      if (tid == 0) {
        int r = 0;
        for (int w = 0; w < BT / 32; w++) { int t = wsum[w]; wsum[w] = r; r += t; }
        s_base = r > 0 ? atomicAdd((int *)&ctl[CTL_NNODES], r) : 0;
        s_stop = (r > 0 && s_base + r > a.cap_nodes) ? 1 : 0;
        if (s_stop) ctl[CTL_OVERFLOW] = 1;
        if (r > 0) s_split = 1;
      }
      __syncthreads();
      if (s_stop) return;
      int id = s_base + wsum[wid] + inc - nct;
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        const int q = tid * LPT + j, st = sc[j] & 0xFFFF;
        if (gs[j] != NOD && q == st) {
          const int k = ks[j];
          L.cfl[q] = id;
          L.cml[q] = (int)msk[j];
          a.child_first[k] = id;
          a.nchild[k] = __popc(msk[j]);
          a.cmask[k] = (unsigned char)msk[j];
          id += __popc(msk[j]);
        }
      }
      __syncthreads();
      // stable scatter (next level's position, node, node start and count);
      // the first point of each child writes the child's record
      int nq[LPT], nk[LPT], nsc[LPT];
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        const int q = tid * LPT + j, g = gs[j];
        nq[j] = q;
        nk[j] = -1;
        nsc[j] = 0;
        if (g != NOD) {
          const int st = sc[j] & 0xFFFF;
          const Pack2 b = L.exs[st], e = L.exs[st + (sc[j] >> 16)];
          const Pack2 D{e.lo - b.lo, e.hi - b.hi};
          const int off = digit_offset(D, g);
          const int rank = (g < 5 ? fld12(mine[j].lo, g) - fld12(b.lo, g)
                                  : fld12(mine[j].hi, g - 5) - fld12(b.hi, g - 5));
          nq[j] = st + off + rank;
          ordn[P0 + nq[j]] = ss[j];
          if (g < 8) {
            const int cnt = g < 5 ? fld12(D.lo, g) : fld12(D.hi, g - 5);
            const int id2 = L.cfl[st] + __popc((unsigned)L.cml[st] & ((1u << g) - 1));
            nk[j] = id2;
            nsc[j] = (st + off) | (cnt << 16);
            if (rank == 0) {
              const int k = ks[j];
              const double W = Wd[j], w = W * 0.5;
              const int bx = g & 1, bz = (g >> 1) & 1, by = (g >> 2) & 1;
              a.pos[3 * id2] = bx ? __dadd_rn(P[j][0], W / 2) : P[j][0];
              a.pos[3 * id2 + 1] = by ? __dadd_rn(P[j][1], W / 2) : P[j][1];
              a.pos[3 * id2 + 2] = bz ? __dadd_rn(P[j][2], W / 2) : P[j][2];
              a.width[id2] = w;
              a.count[id2] = cnt;
              a.start[id2] = P0 + st + off;
              a.parent[id2] = k;
              a.level[id2] = d + 1;
              a.digit[id2] = (unsigned char)g;
              a.nchild[id2] = 0;
              a.cmask[id2] = 0;
              a.child_first[id2] = -1;
            }
          }
        }
      }
      const bool split = s_split, more = s_more;
      __syncthreads();
#pragma unroll
      for (int j = 0; j < LPT; j++) {
        if (tid * LPT + j < m) {
          L.ordl[nq[j]] = ss[j];
          L.nodl[nq[j]] = nk[j];
          L.scl[nq[j]] = nsc[j];
        }
      }
      __syncthreads();
      d++;
      if (split) depth = max(depth, d);
      if (!more) break;
      if (d + 1 >= a.cap_levels || d + 1 > QV_MAX_DEPTH) {
        if (tid == 0) ctl[CTL_OVERFLOW] = 2;
        return;
      }
    }
    for (int q = tid; q < m; q += BT) a.perm[P0 + q] = L.ordl[q];
    __syncthreads();
  }
  if (tid == 0) atomicMax((int *)&ctl[CTL_DEPTH], depth);
}

__global__ void __launch_bounds__(BT) k_build(BuildArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ Pack2 sh[BT / 32 + 1];
  __shared__ Pack2 ex1[CH + 1];  // P1: exclusive digit-count prefix at each position of a chunk
  __shared__ int s9[BT / 32][9];
  volatile int *ctl = a.ctl;
  const int n_act = *a.d_nact;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl[CTL_NACT] = n_act;
  int d = 0;
  bool local = false;
  for (;;) {
    int nsplit = ctl[CTL_NS + d];
    if (nsplit == 0 || n_act == 0) break;
    if (d + 1 >= a.cap_levels || d + 1 > QV_MAX_DEPTH) {
      if (blockIdx.x == 0 && threadIdx.x == 0) ctl[CTL_OVERFLOW] = 2;
      break;
    }
    // every splitting node of this level fits one block: finish block-locally
    if (d > 0 && ctl[CTL_MAXC + d] <= LCH) {
      local = true;
      break;
    }
    const int ls = ctl[CTL_LVL + d], le = ctl[CTL_LVL + d + 1];
    const int *ordc = a.ord + (size_t)d * a.cap_pts;
    int *ordn = a.ord + (size_t)(d + 1) * a.cap_pts;
    const int *nodc = (d & 1) ? a.nodeB : a.nodeA;
    int *nodn = (d & 1) ? a.nodeA : a.nodeB;
    int *cntc = (d & 1) ? a.cnt9B : a.cnt9A;
    int *cntn = (d & 1) ? a.cnt9A : a.cnt9B;

    // ---- P1: digits, node counts, chunk counts.  The loads of a thread's
    // positions are issued together; a node's digit counts in this chunk come
    // from the block scan (prefix at the end of its run of positions minus the
    // prefix at its start), added to the node's counters once per digit by the
    // thread holding the run's first position.
    for (int ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
      const int c0 = ch * CH;
      int ks[PPT], ss[PPT], cs[PPT], st[PPT], gs[PPT];
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        const int p = c0 + threadIdx.x * PPT + j;
        ks[j] = p < n_act ? nodc[p] : -1;
        ss[j] = p < n_act ? ordc[p] : 0;
      }
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        cs[j] = ks[j] >= 0 ? a.count[ks[j]] : 0;
        st[j] = ks[j] >= 0 ? a.start[ks[j]] : 0;
      }
      double X[PPT][3], P[PPT][3], Wd[PPT];
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        const bool sp = cs[j] >= 2;
        const int sl = sp ? ss[j] : 0, k = sp ? ks[j] : 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          X[j][c] = a.x[3 * sl + c];
          P[j][c] = a.pos[3 * k + c];
        }
        Wd[j] = a.width[k];
      }
      Pack2 loc{0ull, 0ull};
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        const int p = c0 + threadIdx.x * PPT + j;
        int g = NOD;
        if (cs[j] >= 2) {
          g = child_digit(X[j], P[j], Wd[j]);
          Pack2 o = pk_one(g);
          loc.lo += o.lo; loc.hi += o.hi;
        }
        gs[j] = g;
        if (p < n_act) a.dig[p] = (unsigned char)g;
      }
      Pack2 tot;
      Pack2 run = block_scan_pack(loc, &tot, sh);
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        ex1[threadIdx.x * PPT + j] = run;
        if (gs[j] != NOD) {
          Pack2 o = pk_one(gs[j]);
          run.lo += o.lo; run.hi += o.hi;
        }
      }
      if (threadIdx.x == 0) ex1[CH] = tot;
      __syncthreads();
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        const int q = threadIdx.x * PPT + j, p = c0 + q;
        if (gs[j] != NOD && p == max(st[j], c0)) {
          // a node's positions end at start + count, except for a root, whose
          // count includes its empty slots: its positions end where the next
          // root's begin
          const int k = ks[j];
          const int nend = d > 0 ? st[j] + cs[j] : (k + 1 < le ? a.start[k + 1] : n_act);
          const int e = min(min(nend, c0 + CH), n_act) - c0;
          const Pack2 b = ex1[q], f = ex1[e];
          int *cn = cntc + (k - ls) * 9;
          for (int g = 0; g < 9; g++) {
            const int v = pk_get(f, g) - pk_get(b, g);
            if (v > 0) atomicAdd(&cn[g], v);
          }
        }
      }
      if (threadIdx.x < 9) a.chunk9[ch * 9 + threadIdx.x] = pk_get(tot, threadIdx.x);
      __syncthreads();
    }
    grid.sync();

    // ---- P2: children (all blocks), chunk prefix scan (block 0)
    // Child slots are claimed with one atomic per warp (the warp's node counts
    // prefix-summed with shuffles); ids within a level carry no meaning beyond
    // contiguity, so their order does not matter.
    for (int kb = ls + blockIdx.x * BT; kb < le; kb += gridDim.x * BT) {
      const int k = kb + threadIdx.x;
      const int lane = threadIdx.x & 31;
      const bool split = k < le && a.count[k] >= 2;
      if (k < le && !split) { a.nchild[k] = 0; a.cmask[k] = 0; }
      int c9[9];
      int nc = 0, nsp = 0;
      unsigned mask = 0;
      if (split) {
        for (int g = 0; g < 9; g++) c9[g] = cntc[(k - ls) * 9 + g];
        for (int g = 0; g < 8; g++)
          if (c9[g] > 0) { nc++; mask |= 1u << g; if (c9[g] >= 2) nsp++; }
      }
      int inc = nc, isp = nsp;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        int u = __shfl_up_sync(0xffffffffu, isp, o);
        if (lane >= o) { inc += t; isp += u; }
      }
      int wbase = 0;
      if (lane == 31) {
        if (inc) wbase = atomicAdd((int *)&ctl[CTL_NNODES], inc);
        if (isp) atomicAdd((int *)&ctl[CTL_NS + d + 1], isp);
      }
      wbase = __shfl_sync(0xffffffffu, wbase, 31);
      if (!split) continue;
      const int base = wbase + inc - nc;
      if (base + nc > a.cap_nodes) {
        ctl[CTL_OVERFLOW] = 1;
        continue;
      }
      a.child_first[k] = base;
      a.nchild[k] = nc;
      a.cmask[k] = (unsigned char)mask;
      double W = a.width[k], w = W * 0.5;
      double P[3] = {a.pos[3 * k], a.pos[3 * k + 1], a.pos[3 * k + 2]};
      double M[3] = {__dadd_rn(P[0], W / 2), __dadd_rn(P[1], W / 2), __dadd_rn(P[2], W / 2)};
      int off = 0, id = base, cmax = 0;
      for (int g = 0; g < 8; g++) cmax = max(cmax, c9[g]);
      if (cmax >= 2) atomicMax((int *)&ctl[CTL_MAXC + d + 1], cmax);
      for (int g = 0; g < 8; g++) {
        if (c9[g] > 0) {
          int bx = g & 1, bz = (g >> 1) & 1, by = (g >> 2) & 1;
          a.pos[3 * id] = bx ? M[0] : P[0];
          a.pos[3 * id + 1] = by ? M[1] : P[1];
          a.pos[3 * id + 2] = bz ? M[2] : P[2];
          a.width[id] = w;
          a.count[id] = c9[g];
          a.start[id] = a.start[k] + off;
          a.parent[id] = k;
          a.level[id] = d + 1;
          a.digit[id] = (unsigned char)g;
          a.nchild[id] = 0;
          a.cmask[id] = 0;
          a.child_first[id] = -1;
          id++;
        }
        off += c9[g];
      }
    }
    if (blockIdx.x == 0) {
      // exclusive scan of chunk9 over chunks, 9 channels
      int per = (a.nchunks + BT - 1) / BT;
      int lo = threadIdx.x * per, hi = min(a.nchunks, lo + per);
      int sum[9];
#pragma unroll
      for (int g = 0; g < 9; g++) sum[g] = 0;
      for (int q = lo; q < hi; q++)
#pragma unroll
        for (int g = 0; g < 9; g++) sum[g] += a.chunk9[q * 9 + g];
      int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      int inc[9];
#pragma unroll
      for (int g = 0; g < 9; g++) {
        int v = sum[g];
        for (int o = 1; o < 32; o <<= 1) {
          int t = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += t;
        }
        inc[g] = v;
        if (lane == 31) s9[wid][g] = v;
      }
      __syncthreads();
      if (threadIdx.x < 9) {
        int r = 0;
        for (int w2 = 0; w2 < BT / 32; w2++) { int t = s9[w2][threadIdx.x]; s9[w2][threadIdx.x] = r; r += t; }
      }
      __syncthreads();
      int run[9];
#pragma unroll
      for (int g = 0; g < 9; g++) run[g] = s9[wid][g] + inc[g] - sum[g];
      for (int q = lo; q < hi; q++)
#pragma unroll
        for (int g = 0; g < 9; g++) {
          int t = a.chunk9[q * 9 + g];
          a.chunk9[q * 9 + g] = run[g];
          run[g] += t;
        }
    }
    grid.sync();
    if (ctl[CTL_OVERFLOW]) break;

    // ---- P3: stable ranks within digit channels; node-start snapshots
    for (int ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
      Pack2 loc{0ull, 0ull};
      int gs[PPT];
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        int p = ch * CH + threadIdx.x * PPT + j;
        gs[j] = p < n_act ? a.dig[p] : NOD;
        if (gs[j] != NOD) { Pack2 o = pk_one(gs[j]); loc.lo += o.lo; loc.hi += o.hi; }
      }
      Pack2 tot;
      Pack2 ex = block_scan_pack(loc, &tot, sh);
#pragma unroll
      for (int j = 0; j < PPT; j++) {
        int p = ch * CH + threadIdx.x * PPT + j;
        int g = gs[j];
        if (g != NOD) {
          int k = nodc[p];
          a.rnk[p] = a.chunk9[ch * 9 + g] + pk_get(ex, g);
          if (p == a.start[k]) {
            for (int h = 0; h < 9; h++) a.rs9[(k - ls) * 9 + h] = a.chunk9[ch * 9 + h] + pk_get(ex, h);
          }
          Pack2 o = pk_one(g);
          ex.lo += o.lo; ex.hi += o.hi;
        }
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl[CTL_LVL + d + 2] = ctl[CTL_NNODES];
    grid.sync();

    // ---- P4: scatter into the next level's order; reset counters
    const int le2 = ctl[CTL_LVL + d + 2];
    for (int p = blockIdx.x * BT + threadIdx.x; p < n_act; p += gridDim.x * BT) {
      int g = a.dig[p];
      if (g == NOD) {
        ordn[p] = ordc[p];
        nodn[p] = -1;
      } else {
        int k = nodc[p], kl = k - ls;
        int off = 0;
        for (int h = 0; h < g; h++) off += cntc[kl * 9 + h];
        int np = a.start[k] + off + a.rnk[p] - a.rs9[kl * 9 + g];
        ordn[np] = ordc[p];
        nodn[np] = g < 8 ? a.child_first[k] + __popc(a.cmask[k] & ((1u << g) - 1)) : -1;
      }
    }
    for (int q = blockIdx.x * BT + threadIdx.x; q < (le2 - le) * 9; q += gridDim.x * BT) cntn[q] = 0;
    d++;
    grid.sync();
  }
  if (local) {
    // hand over to k_build_local: the bounds of all ranges, fixed before any
    // range's levels overwrite the level-d node array of its positions
    const int nch = (n_act + LCH - 1) / LCH;
    const int *nod0 = (d & 1) ? a.nodeB : a.nodeA;
    for (int c = blockIdx.x * BT + threadIdx.x; c <= nch; c += gridDim.x * BT) {
      const int p = c * LCH;
      int b = n_act;
      if (p < n_act) {
        const int k = nod0[p];
        b = (k >= 0 && a.count[k] >= 2) ? a.start[k] : p;
      }
      a.chunk9[c] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl[CTL_DEPTH] = d;
      ctl[CTL_NGLOB] = ctl[CTL_NNODES];
      ctl[CTL_LOCALD] = d;
    }
  } else {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl[CTL_DEPTH] = d;
      ctl[CTL_NGLOB] = ctl[CTL_NNODES];
      ctl[CTL_LOCALD] = -1;
    }
    const int *fin = a.ord + (size_t)d * a.cap_pts;
    for (int p = blockIdx.x * BT + threadIdx.x; p < n_act; p += gridDim.x * BT) a.perm[p] = fin[p];
  }
}

// The block-local levels after k_build (nothing to do when the grid-wide
// levels finished the tree or ran out of capacity).
__global__ void __launch_bounds__(BT) k_build_local(BuildArgs a) {
  extern __shared__ __align__(16) unsigned char lsm[];
  __shared__ Pack2 sh[BT / 32 + 1];
  const int d0 = a.ctl[CTL_LOCALD];
  if (d0 < 0 || a.ctl[CTL_OVERFLOW]) return;
  build_local(a, d0, *a.d_nact, sh, *reinterpret_cast<LocalSmem *>(lsm));
}

// --------------------------------------------------------------- moments
// A node's moments are 15 independent sequential FP64 chains over its points
// in ascending slot order: cent (3), circ (3) and Cij (9).  The chains cannot
// be reassociated, so their latency is the floor; the kernels below keep the
// chain lanes fed from shared memory while other warps gather and precompute.
#define MW 8      // warps per block (small nodes: one warp per node)
#define BIGN LCH  // nodes with more points: a block each, early (all made grid-wide)
#define MIDN 128  // nodes with more points (up to BIGN): a block each, after the tree
#define TN 8      // nodes with at most this many points: a thread each
#define MC 256    // points per shared-memory chunk in the block kernel
#define MBT 512   // threads of the block kernel: warp 0 runs the chains, the rest gather

// The 15 moment chains over m staged points (row stride `stride` doubles:
// x(3), ghosti(3), x_m (ghosti_k - x_k) (9)), lane l < 15 owning chain l:
// lanes 0-2 sum x, lanes 6-14 sum the products, and lanes 3-5 take
// circ = (circ + ghosti) - x (src/tree.f90:160).  Every lane runs the same
// add-then-subtract, the subtrahend being +0 outside lanes 3-5 (s - 0 = s
// exactly), so the warp never splits into two serialised paths; each group
// of four points is loaded while the previous group's eight dependent
// roundings run, so the chain waits on the FP64 adds alone.
__device__ __forceinline__ double chain15(double acc, const double *rows, int stride, int m,
                                          int lane) {
  const bool cl = lane >= 3 && lane < 6;
  const double *pa = rows + lane, *pz = rows + (cl ? lane - 3 : lane);
  int q = 0;
  if (m >= 4) {
    // the next group's loads go out before this group's dependent roundings
    double a[4], z[4];
#pragma unroll
    for (int u = 0; u < 4; u++) { a[u] = pa[stride * u]; z[u] = cl ? pz[stride * u] : 0.; }
    for (q = 4; q + 4 <= m; q += 4) {
      double na[4], nz[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        na[u] = pa[stride * (q + u)];
        nz[u] = cl ? pz[stride * (q + u)] : 0.;
      }
#pragma unroll
      for (int u = 0; u < 4; u++) acc = __dsub_rn(__dadd_rn(acc, a[u]), z[u]);
#pragma unroll
      for (int u = 0; u < 4; u++) { a[u] = na[u]; z[u] = nz[u]; }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) acc = __dsub_rn(__dadd_rn(acc, a[u]), z[u]);
  }
  for (; q < m; q++) acc = __dsub_rn(__dadd_rn(acc, pa[stride * q]), cl ? pz[stride * q] : 0.);
  return acc;
}

// One thread per node of at most TN points, then one warp per node of at most MIDN points.
__global__ void __launch_bounds__(MW * 32) k_moments(const int *__restrict__ ctl, int cap_nodes, int k0,
                                                     const int *__restrict__ level,
                                                     const int *__restrict__ start,
                                                     const int *__restrict__ count,
                                                     const int *__restrict__ ord, int cap_pts,
                                                     const double *__restrict__ x,
                                                     const double *__restrict__ gi, double *cent,
                                                     double *circ, double *C, int *first) {
  __shared__ double buf[MW][32][15];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (ctl[CTL_OVERFLOW]) return;
  const int n_nodes = min(ctl[CTL_NNODES], cap_nodes);
  // nodes of at most TN points (most of a tree): one thread each, the 15
  // chains over the node's points in the warp path's order and roundings
  // (the next point's loads issued before the current point's operations)
  for (int kl = k0 + blockIdx.x * blockDim.x + threadIdx.x; kl < n_nodes;
       kl += gridDim.x * blockDim.x) {
    const int n = count[kl];
    if (n < 1 || n > TN) continue;
    const int *o = ord + (size_t)level[kl] * cap_pts + start[kl];
    double ac[3] = {0., 0., 0.}, ai[3] = {0., 0., 0.}, aC[9];
#pragma unroll
    for (int q = 0; q < 9; q++) aC[q] = 0.;
    int idx = o[0];
    const int idx0 = idx;
    double X[3], G[3];
#pragma unroll
    for (int c = 0; c < 3; c++) { X[c] = x[3 * idx + c]; G[c] = gi[3 * idx + c]; }
    for (int q = 0; q < n; q++) {
      double nX[3], nG[3];
      if (q + 1 < n) {
        const int ni = o[q + 1];
#pragma unroll
        for (int c = 0; c < 3; c++) { nX[c] = x[3 * ni + c]; nG[c] = gi[3 * ni + c]; }
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        ac[c] = __dadd_rn(ac[c], X[c]);
        ai[c] = __dsub_rn(__dadd_rn(ai[c], G[c]), X[c]);
      }
#pragma unroll
      for (int mm = 0; mm < 3; mm++)
#pragma unroll
        for (int kk = 0; kk < 3; kk++)
          aC[3 * mm + kk] = __dadd_rn(aC[3 * mm + kk], __dmul_rn(X[mm], __dsub_rn(G[kk], X[kk])));
      if (q + 1 < n) {
#pragma unroll
        for (int c = 0; c < 3; c++) { X[c] = nX[c]; G[c] = nG[c]; }
      }
    }
    double cm[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      cm[c] = __ddiv_rn(ac[c], (double)n);
      cent[3 * kl + c] = cm[c];
      circ[3 * kl + c] = ai[c];
    }
#pragma unroll
    for (int mm = 0; mm < 3; mm++)
#pragma unroll
      for (int kk = 0; kk < 3; kk++)
        C[9 * kl + 3 * mm + kk] = __dsub_rn(aC[3 * mm + kk], __dmul_rn(cm[mm], ai[kk]));
    first[kl] = idx0;
  }
  // nodes of TN+1..MIDN points: one warp per node, the next 32 points' gather
  // in flight while the chains run over the current 32
  for (int k = k0 + blockIdx.x * MW + wid; k < n_nodes; k += gridDim.x * MW) {
    int s = start[k], n = count[k];
    if (n <= TN || n > MIDN) continue;
    const int *o = ord + (size_t)level[k] * cap_pts + s;
    double acc = 0.;
    double X[3] = {0., 0., 0.}, G[3] = {0., 0., 0.};
    if (lane < n) {
      const int idx = o[lane];
#pragma unroll
      for (int c = 0; c < 3; c++) { X[c] = x[3 * idx + c]; G[c] = gi[3 * idx + c]; }
    }
    for (int base = 0; base < n; base += 32) {
      const int m = min(32, n - base);
      if (lane < m) {
        double *b = buf[wid][lane];
#pragma unroll
        for (int c = 0; c < 3; c++) { b[c] = X[c]; b[3 + c] = G[c]; }
#pragma unroll
        for (int mm = 0; mm < 3; mm++)
#pragma unroll
          for (int kk = 0; kk < 3; kk++) b[6 + 3 * mm + kk] = __dmul_rn(X[mm], __dsub_rn(G[kk], X[kk]));
      }
      __syncwarp();
      if (base + 32 + lane < n) {
        const int idx = o[base + 32 + lane];
#pragma unroll
        for (int c = 0; c < 3; c++) { X[c] = x[3 * idx + c]; G[c] = gi[3 * idx + c]; }
      }
      if (lane < 15) acc = chain15(acc, &buf[wid][0][0], 15, m, lane);
      __syncwarp();
    }
    double cm = lane < 3 ? __ddiv_rn(acc, (double)n) : 0.;
    // C(i,k) -= cent_i circ_k  (lane 6+3i+k)
    int ci = (lane - 6) / 3, ck = (lane - 6) % 3;
    double cen = __shfl_sync(0xffffffffu, cm, lane >= 6 && lane < 15 ? ci : 0);
    double cir = __shfl_sync(0xffffffffu, acc, lane >= 6 && lane < 15 ? 3 + ck : 0);
    if (lane < 3) cent[3 * k + lane] = cm;
    else if (lane < 6) circ[3 * k + lane - 3] = acc;
    else if (lane < 15) C[9 * k + 3 * ci + ck] = __dsub_rn(acc, __dmul_rn(cen, cir));
    if (lane == 0) first[k] = o[0];
  }
}

// List the non-root nodes (k >= k0) with lo < points <= hi (order irrelevant),
// among the nodes of the grid-wide levels (glob) or of the whole tree.  Nodes
// of more than BIGN points all come from the grid-wide levels, which are
// complete once k_build ends (the block-local levels may still be adding).
// late: 0 = every node, 1 = all but the late root children (qv_l1_late),
// 2 = those only.
__global__ void k_list_big(const int *__restrict__ ctl, int cap_nodes, int k0,
                           const int *__restrict__ count, int *list, int *nlist, int lo, int hi,
                           int glob, int late) {
  if (ctl[CTL_OVERFLOW]) return;
  const int n_nodes = min(ctl[glob ? CTL_NGLOB : CTL_NNODES], cap_nodes);
  const int l1_end = ctl[CTL_LVL + 2];  // the first node of level 2
  for (int k = k0 + blockIdx.x * blockDim.x + threadIdx.x; k < n_nodes; k += gridDim.x * blockDim.x) {
    if (!(count[k] > lo && count[k] <= hi)) continue;
    if (late) {
      const int j = qv_l1_pair(k);
      const bool lk = qv_l1_late(k, l1_end, count[k], j < n_nodes ? count[j] : 0);
      if (lk != (late == 2)) continue;
    }
    list[atomicAdd(nlist, 1)] = k;
  }
}

// One block per node with more than BIGN points: warps 1.. gather x, ghosti and
// the Cij products of the next chunk into shared memory while warp 0's lanes
// 0..14 run the chains over the current chunk (double buffered).
__global__ void __launch_bounds__(MBT) k_moments_big(const int *__restrict__ list,
                                                     const int *__restrict__ nlist,
                                                     const int *__restrict__ level,
                                                     const int *__restrict__ start,
                                                     const int *__restrict__ count,
                                                     const int *__restrict__ ord, int cap_pts,
                                                     const double *__restrict__ x,
                                                     const double *__restrict__ gi, double *cent,
                                                     double *circ, double *C, int *first,
                                                     int l1_late, PackArgs pk, int do_pack) {
  // l1_late: the late level-1 chains, whose centroid (and first point)
  // k_moments_cent stores; only circ and Cij are stored here.
  extern __shared__ double mb[];  // [2][MC][15]
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nl = *nlist;
  for (int li = blockIdx.x; li < nl; li += gridDim.x) {
    const int k = list[li];
    const int s = start[k], n = count[k];
    const int *o = ord + (size_t)level[k] * cap_pts + s;
    const int nch = (n + MC - 1) / MC;
    auto produce = [&](int ch, double *dst) {
      int base = ch * MC, m = min(MC, n - base);
      for (int q = threadIdx.x - 32; q < m; q += blockDim.x - 32) {
        int idx = o[base + q];
        double X[3], G[3];
#pragma unroll
        for (int c = 0; c < 3; c++) { X[c] = x[3 * idx + c]; G[c] = gi[3 * idx + c]; }
        double *b = dst + 15 * q;
#pragma unroll
        for (int c = 0; c < 3; c++) { b[c] = X[c]; b[3 + c] = G[c]; }
#pragma unroll
        for (int mm = 0; mm < 3; mm++)
#pragma unroll
          for (int kk = 0; kk < 3; kk++) b[6 + 3 * mm + kk] = __dmul_rn(X[mm], __dsub_rn(G[kk], X[kk]));
      }
    };
    __syncthreads();
    if (wid > 0) produce(0, mb);
    __syncthreads();
    double acc = 0.;
    for (int ch = 0; ch < nch; ch++) {
      double *cur = mb + (ch & 1) * MC * 15;
      if (wid > 0) {
        if (ch + 1 < nch) produce(ch + 1, mb + ((ch + 1) & 1) * MC * 15);
      } else if (lane < 15) {
        acc = chain15(acc, cur, 15, min(MC, n - ch * MC), lane);
      }
      __syncthreads();
    }
    if (wid == 0) {
      double cm = lane < 3 ? __ddiv_rn(acc, (double)n) : 0.;
      int ci = (lane - 6) / 3, ck = (lane - 6) % 3;
      double cen = __shfl_sync(0xffffffffu, cm, lane >= 6 && lane < 15 ? ci : 0);
      double cir = __shfl_sync(0xffffffffu, acc, lane >= 6 && lane < 15 ? 3 + ck : 0);
      if (lane < 3) {
        if (!l1_late) cent[3 * k + lane] = cm;
      } else if (lane < 6) {
        circ[3 * k + lane - 3] = acc;
      } else if (lane < 15) {
        C[9 * k + 3 * ci + ck] = __dsub_rn(acc, __dmul_rn(cen, cir));
      }
      if (lane == 0 && !l1_late) first[k] = o[0];
      __syncwarp();
      // the node's walk packs (a late root child: its payload)
      if (do_pack && lane == 0) pack_one(pk, k, l1_late ? 2 : 3);
    }
  }
}

// The centroid chains alone (one rounding per point: half the circ chain's
// latency) of the nodes of list = [count, nodes...], and their walk headers:
// warps 1.. stage x in chunks of MCC points, lanes 0..2 of warp 0 sum it, in
// the same order and roundings as chain15's lanes 0..2, so the value is the one
// k_moments_big computes.  One add per point leaves the chain only ~8 cycles a
// point, so the chunks are larger than k_moments_big's and each group of eight
// points is loaded while the previous group's adds run.
#define MCC 1024
__global__ void __launch_bounds__(MBT) k_moments_cent(const int *__restrict__ ctl,
                                                      const int *__restrict__ list,
                                                      const int *__restrict__ level,
                                                      const int *__restrict__ start,
                                                      const int *__restrict__ count,
                                                      const int *__restrict__ ord, int cap_pts,
                                                      const double *__restrict__ x, double *cent,
                                                      int *first, PackArgs pk) {
  extern __shared__ double mb[];  // [2][MCC][3]
  if (ctl[CTL_OVERFLOW]) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nl = list[0];
  for (int li = blockIdx.x; li < nl; li += gridDim.x) {
    const int k = list[1 + li];
    const int n = count[k];
    const int *o = ord + (size_t)level[k] * cap_pts + start[k];
    const int nch = (n + MCC - 1) / MCC;
    auto produce = [&](int ch, double *dst) {
      const int base = ch * MCC, m = min(MCC, n - base);
      for (int q = threadIdx.x - 32; q < m; q += blockDim.x - 32) {
        const int idx = o[base + q];
#pragma unroll
        for (int c = 0; c < 3; c++) dst[3 * q + c] = x[3 * idx + c];
      }
    };
    __syncthreads();
    if (wid > 0) produce(0, mb);
    __syncthreads();
    double acc = 0.;
    for (int ch = 0; ch < nch; ch++) {
      double *cur = mb + (ch & 1) * MCC * 3;
      if (wid > 0) {
        if (ch + 1 < nch) produce(ch + 1, mb + ((ch + 1) & 1) * MCC * 3);
      } else if (lane < 3) {
        const int m = min(MCC, n - ch * MCC);
        const double *b = cur + lane;
        int q = 0;
        if (m >= 8) {
          double a[8];
#pragma unroll
          for (int u = 0; u < 8; u++) a[u] = b[3 * u];
          for (q = 8; q + 8 <= m; q += 8) {
            double na[8];
#pragma unroll
            for (int u = 0; u < 8; u++) na[u] = b[3 * (q + u)];
#pragma unroll
            for (int u = 0; u < 8; u++) acc = __dadd_rn(acc, a[u]);
#pragma unroll
            for (int u = 0; u < 8; u++) a[u] = na[u];
          }
#pragma unroll
          for (int u = 0; u < 8; u++) acc = __dadd_rn(acc, a[u]);
        }
        for (; q < m; q++) acc = __dadd_rn(acc, b[3 * q]);
      }
      __syncthreads();
    }
    if (wid == 0 && lane < 3) cent[3 * k + lane] = __ddiv_rn(acc, (double)n);
    if (threadIdx.x == 0) first[k] = o[0];
    __syncwarp();
    if (threadIdx.x == 0) pack_one(pk, k, 1);  // the headers; the payload comes late
  }
}

// Root centroid: masked mean over all slots in ascending order
// (src/tree.f90:53-55) = sequential sums over the compacted active list.
// Warps 1.. stage chunks of positions in shared memory (double buffered);
// lanes 0..2 of warp 0 run the three chains.
#define RC 2048
__device__ __forceinline__ void root_cent_chain(const int n_act, const int *__restrict__ act,
                                                const double *__restrict__ x, double *cent) {
  extern __shared__ double rb[];  // [2][RC][3]
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nch = (n_act + RC - 1) / RC;
  auto produce = [&](int ch, double *dst) {
    int base = ch * RC, m = min(RC, n_act - base);
    for (int q = threadIdx.x - 32; q < m; q += blockDim.x - 32) {
      int i = act ? act[base + q] : base + q;
      dst[3 * q] = x[3 * i];
      dst[3 * q + 1] = x[3 * i + 1];
      dst[3 * q + 2] = x[3 * i + 2];
    }
  };
  if (wid > 0 && nch > 0) produce(0, rb);
  __syncthreads();
  double acc = 0.;
  for (int ch = 0; ch < nch; ch++) {
    double *cur = rb + (ch & 1) * RC * 3;
    if (wid > 0) {
      if (ch + 1 < nch) produce(ch + 1, rb + ((ch + 1) & 1) * RC * 3);
    } else if (lane < 3) {
      const int m = min(RC, n_act - ch * RC);
      const double *b = cur + lane;
      int q = 0;
      for (; q + 8 <= m; q += 8) {
        double a[8];
#pragma unroll
        for (int u = 0; u < 8; u++) a[u] = b[3 * (q + u)];
#pragma unroll
        for (int u = 0; u < 8; u++) acc = __dadd_rn(acc, a[u]);
      }
      for (; q < m; q++) acc = __dadd_rn(acc, b[3 * q]);
    }
    __syncthreads();
  }
  if (wid == 0 && lane < 3) cent[lane] = __ddiv_rn(acc, (double)n_act);
}

__global__ void __launch_bounds__(512) k_root_cent(const int *__restrict__ d_nact,
                                                   const int *__restrict__ act,
                                                   const double *__restrict__ x, double *cent) {
  root_cent_chain(*d_nact, act, x, cent);
}

// The estimate of the same centroid the walk starts from while the chain runs:
// a parallel sum S of the active positions and, per component, the bound
//   |exact - estimate| <= 2 gamma_n sum|x| / n + 4 u |estimate|,
// gamma_n = n u / (1 - n u), u = 2^-53.  Any order of summing n terms is within
// gamma_(n-1) sum|x| of the true sum (the reference's sequential sum
// included), and each of the two divisions by n rounds once.  est[3] is the
// Euclidean norm of the three component bounds, widened by a relative 1e-6
// (which also covers the rounding of sum|x| itself).  The same pass copies the
// active positions, in active order, to xc for the exact chain, so that the
// chain reads nothing another kernel may write before it is joined.  The last
// block to finish (ticket ctl[3]) reduces the block sums in block order and
// clears the counters of the walk's fix-up.
__global__ void __launch_bounds__(256) k_root_est(const int *__restrict__ d_nact,
                                                  const int *__restrict__ act,
                                                  const double *__restrict__ x, double *xc,
                                                  double *part, int *ctl, double *est,
                                                  double bound_scale) {
  const int n = *d_nact;
  double v[6] = {0., 0., 0., 0., 0., 0.};
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int i = act[q];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double y = x[3 * i + c];
      xc[3 * (size_t)q + c] = y;
      v[c] += y;
      v[3 + c] += fabs(y);
    }
  }
  __shared__ double red[6][8];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0) red[k][w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[threadIdx.x][k];
    part[6 * blockIdx.x + threadIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&ctl[3], 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double S[6] = {0., 0., 0., 0., 0., 0.};
    for (int b = 0; b < (int)gridDim.x; b++)
      for (int k = 0; k < 6; k++) S[k] += part[6 * b + k];
    const double u = 1.1102230246251565e-16, nu = n * u;
    const double gam = nu / (1. - nu);
    double e2 = 0.;
    for (int c = 0; c < 3; c++) {
      est[c] = S[c] / n;
      const double e = 2. * gam * S[3 + c] / n + 4. * u * fabs(est[c]);
      e2 += e * e;
    }
    est[3] = sqrt(e2) * (1. + 1e-6) * bound_scale + 1e-300;
    ctl[0] = 0;
    ctl[2] = 0;
    ctl[3] = 0;
  }
}

// When the root's headers start from the estimate: by size (-1; trees of at
// least QV_ROOT_SPEC_MIN slots), never (0) or always (1); and a factor on the
// estimate's bound.  Set only by the test hook qv_test_root_speculation.
static int g_root_spec_mode = -1;
static double g_root_bound_scale = 1.;

extern "C" int qv_test_root_speculation(int mode, double bound_scale) {
  if (mode < -1 || mode > 1 || !(bound_scale >= 1.)) return QV_ERR_ARG;
  g_root_spec_mode = mode;
  g_root_bound_scale = bound_scale;
  return QV_OK;
}

// When a mixed Tree build packs the big root children late: by size (-1;
// builds of at least QV_L1_LATE_MIN slots), never (0) or always (1).  Set only
// by the test hook qv_test_late_level1.
static int g_l1_late_mode = -1;

extern "C" int qv_test_late_level1(int mode) {
  if (mode < -1 || mode > 1) return QV_ERR_ARG;
  g_l1_late_mode = mode;
  return QV_OK;
}

// Put the exact root centroid in (cent[0..2] and the root's headers) once its
// chain has been joined.
__global__ void k_root_pack(PackArgs pk, const double *__restrict__ exact, double *cent) {
  if (threadIdx.x == 0) {
    for (int c = 0; c < 3; c++) cent[c] = exact[c];
    pack_one(pk, 0, 3);
  }
}

// The same centroid for every root of a forest: block r takes root r, whose
// active slots are fact[roots[r].z .. roots[r].z + roots[r].w).
__global__ void __launch_bounds__(512) k_forest_root_cent(int nroots, const int4 *__restrict__ roots,
                                                          const int *__restrict__ fact,
                                                          const double *__restrict__ x,
                                                          const int *__restrict__ ctl,
                                                          double *cent) {
  if (ctl[CTL_OVERFLOW]) return;
  for (int r = blockIdx.x; r < nroots; r += gridDim.x) {
    const int4 R = roots[r];
    if (R.w > 0) root_cent_chain(R.w, fact + R.z, x, cent + 3 * r);
    __syncthreads();
  }
}

// ------------------------------------------------------------ walk packs
__device__ __forceinline__ void split2(double v, float &h, float &l) {
  h = __double2float_rn(v);
  l = __double2float_rn(v - (double)h);
}

__device__ void pack_node(int k, int nroots, const double *__restrict__ pos,
                          const double *__restrict__ width, const double *__restrict__ cent,
                          const double *__restrict__ circ, const double *__restrict__ C,
                          const int *__restrict__ count, const int *__restrict__ child_first,
                          const int *__restrict__ nchild, const unsigned char *__restrict__ cmask,
                          const int *__restrict__ first,
                          const double *__restrict__ x, const double *__restrict__ gi,
                          const int *__restrict__ inf, const int *__restrict__ beh,
                          double theta, int extra, WNode64 *w64, WPay64 *p64, WNode32 *w32, SNode32 *c32,
                          WPay32 *p32, int *leaf_of, int n_leaf, int full, int what);

__device__ void pack_node(int k, int nroots, const double *__restrict__ pos,
                          const double *__restrict__ width, const double *__restrict__ cent,
                          const double *__restrict__ circ, const double *__restrict__ C,
                          const int *__restrict__ count, const int *__restrict__ child_first,
                          const int *__restrict__ nchild, const unsigned char *__restrict__ cmask,
                          const int *__restrict__ first,
                          const double *__restrict__ x, const double *__restrict__ gi,
                          const int *__restrict__ inf, const int *__restrict__ beh,
                          double theta, int extra, WNode64 *w64, WPay64 *p64, WNode32 *w32, SNode32 *c32,
                          WPay32 *p32, int *leaf_of, int n_leaf, int full, int what) {
  // what: 1 = the headers (w64, w32, c32), 2 = the payloads (p64, p32), 3 = both.
  // A payload alone (a late level-1 node: more than one point) reads only the
  // node's count and moments.
  const bool root = k < nroots;
  const int cnt = count[k];
  if (what & 1) {
    WNode64 h;
    h.cx = cent[3 * k]; h.cy = cent[3 * k + 1]; h.cz = cent[3 * k + 2];
    h.width = width[k];
    // geo_dist = |cent - (pos + width/2.)|, src/tree.f90:355-357
    double hw = width[k] / 2.;
    double g0 = __dsub_rn(h.cx, __dadd_rn(pos[3 * k], hw));
    double g1 = __dsub_rn(h.cy, __dadd_rn(pos[3 * k + 1], hw));
    double g2 = __dsub_rn(h.cz, __dadd_rn(pos[3 * k + 2], hw));
    h.geo = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(g0, g0), __dmul_rn(g1, g1)), __dmul_rn(g2, g2)));
    // a root's count is its system's slot count, empty slots included
    h.count = cnt;
    h.child_first = child_first[k];
    h.nchild = nchild[k];
    int f = first[k];
    h.finf = (f >= 0) ? inf[f] : 0;
    h.jb = (f >= 0 && h.finf > 0) ? beh[h.finf - 1] : 0;
    h.first = f;
    w64[k] = h;
    if (leaf_of && cnt == 1 && f >= 0 && f < n_leaf) leaf_of[f] = k;
    WNode32 h32;
    split2(h.cx, h32.ch[0], h32.cl[0]);
    split2(h.cy, h32.ch[1], h32.cl[1]);
    split2(h.cz, h32.ch[2], h32.cl[2]);
    // Opening test of src/tree.f90:354-365,394: theta = w/(d - geo) < tree_theta
    // (extra correction) or w/d < tree_theta.  For d > geo it is d > geo + w/theta.
    // The centroid lies in its cell, so geo <= (sqrt 3 / 2) w, and d <= geo then
    // gives w/d >= 2/sqrt 3: the cell opens whenever theta < 2/sqrt 3.  Under that
    // condition the test is d^2 > rc2 exactly; the walk compares in FP32 with a
    // margin and falls back to the FP64 expression near the threshold.  The root
    // (centroid anywhere, zero moments) always takes the FP64 path.
    bool fast = theta > 0. && (!extra || theta < 1.15);
    h32.count = cnt;
    h32.child_first = h.child_first;
    h32.nchild = h.nchild;
    h32.jb = h.jb;
    if (root || !fast) {
      h32.rhi = h32.rlo = -1.f;
    } else {
      double rc = (extra ? h.geo : 0.) + h.width / theta;
      double rc2 = rc * rc;
      h32.rhi = __double2float_rn(rc2 * (1. + 4e-6));
      h32.rlo = __double2float_rn(rc2 * (1. - 4e-6));
    }
    w32[k] = h32;
    if (full) {  // the candidate search's header
      SNode32 s32;
      for (int c = 0; c < 3; c++) {
        s32.ch[c] = h32.ch[c];
        s32.cl[c] = h32.cl[c];
        s32.lo[c] = __double2float_rd(pos[3 * k + c]);
      }
      double w4 = 4. * h.width * h.width;  // (2 width)^2
      s32.rhi = __double2float_rn(w4 * (1. + 4e-6));
      s32.rlo = __double2float_rn(w4 * (1. - 4e-6));
      s32.w = __double2float_ru(h.width);
      s32.count = cnt;
      s32.child_first = h.child_first;
      s32.nchild = h.nchild;
      s32.cmask = cmask[k];
      c32[k] = s32;
    }
  }
  if (!(what & 2)) return;
  WPay64 q;
  WPay32 r;
  const int f = cnt == 1 ? first[k] : -1;
  if (cnt == 1 && f >= 0) {
    for (int c = 0; c < 3; c++) {
      q.a[c] = x[3 * f + c];
      q.b[c] = gi[3 * f + c];
      split2(q.b[c], r.a[c], r.b[c]);
    }
    for (int c = 0; c < 9; c++) { q.C[c] = 0.; r.C[c] = 0.f; }
    for (int c = 0; c < 3; c++) r.C[c] = __double2float_rn(q.b[c] - q.a[c]);
  } else {
    const double *M = C + 9 * k;
    for (int c = 0; c < 3; c++) q.a[c] = root ? 0. : circ[3 * k + c];
    if (root) {
      for (int c = 0; c < 9; c++) q.C[c] = 0.;
    } else {
      for (int c = 0; c < 9; c++) q.C[c] = M[c];
    }
    // w_m = sum_kl eps(m,k,l) C(k,l)
    q.b[0] = q.C[5] - q.C[7];
    q.b[1] = q.C[6] - q.C[2];
    q.b[2] = q.C[1] - q.C[3];
    for (int c = 0; c < 3; c++) { r.a[c] = (float)q.a[c]; r.b[c] = (float)q.b[c]; }
    for (int c = 0; c < 9; c++) r.C[c] = (float)q.C[c];
  }
  q.pad = 0.;
  r.pad = 0.f;
  if (full) p64[k] = q;  // the FP64 walk's payload
  p32[k] = r;
}

// Everything a build starts from, in one launch: the root record
// (src/tree.f90:49-58: corner -L/2, width L, pcount = all slots, parray(1) =
// slot 1), the control block, the level-0 order (the active slots in
// ascending order), node ids of level 0 and zeroed digit counters.
__global__ void k_build_init(double *pos, double *width, int *count, int *start, int *parent,
                             int *child_first, int *nchild, int *level, unsigned char *digit,
                             unsigned char *cmask, int *first, double L, int n_slots, int *ctl,
                             int *ord, const int *__restrict__ act, int *nodeA, int *cnt9,
                             size_t ncnt9) {
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  if (tid == 0) {
    pos[0] = -L / 2.; pos[1] = -L / 2.; pos[2] = -L / 2.;
    width[0] = L;
    count[0] = n_slots;
    start[0] = 0;
    parent[0] = -1;
    child_first[0] = -1;
    nchild[0] = 0;
    level[0] = 0;
    digit[0] = 0xFF;
    cmask[0] = 0;
    first[0] = n_slots > 0 ? 0 : -1;
  }
  for (size_t q = tid; q < CTL_SIZE; q += stride) {
    int v = 0;
    if (q == CTL_NNODES) v = 1;
    else if (q == CTL_NS) v = n_slots > 1 ? 1 : 0;
    else if (q == CTL_LVL + 1) v = 1;
    else if (q == CTL_LOCALD) v = -1;
    ctl[q] = v;
  }
  for (size_t q = tid; q < (size_t)n_slots; q += stride) {
    ord[q] = act[q];
    nodeA[q] = 0;
  }
  for (size_t q = tid; q < ncnt9; q += stride) cnt9[q] = 0;
}

// The same start for a forest of independent systems: root r is system r's
// construct_tree root (corner -L/2, width L, pcount = the system's slots,
// parray(1) = its first slot); the level-0 order is the forest's active slots
// (each system's contiguous and ascending) and froot gives each position's root.
__global__ void k_forest_init(int nroots, const int4 *__restrict__ roots, double *pos,
                              double *width, int *count, int *start, int *parent,
                              int *child_first, int *nchild, int *level, unsigned char *digit,
                              unsigned char *cmask, int *first, double L, int n_fact, int *ctl,
                              int *ord, const int *__restrict__ fact,
                              const int *__restrict__ froot, int *nodeA, int *cnt9, size_t ncnt9) {
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t r = tid; r < (size_t)nroots; r += stride) {
    const int4 R = roots[r];
    pos[3 * r] = -L / 2.; pos[3 * r + 1] = -L / 2.; pos[3 * r + 2] = -L / 2.;
    width[r] = L;
    count[r] = R.y;
    start[r] = R.z;
    parent[r] = -1;
    child_first[r] = -1;
    nchild[r] = 0;
    level[r] = 0;
    digit[r] = 0xFF;
    cmask[r] = 0;
    first[r] = R.y > 0 ? R.x : -1;
  }
  if (tid == 0) {
    int nsplit = 0;
    for (int r = 0; r < nroots; r++) nsplit += roots[r].y > 1 ? 1 : 0;
    ctl[CTL_NS] = nsplit;
  }
  for (size_t q = tid; q < CTL_SIZE; q += stride) {
    if (q == CTL_NS) continue;
    int v = 0;
    if (q == CTL_NNODES) v = nroots;
    else if (q == CTL_LVL + 1) v = nroots;
    else if (q == CTL_LOCALD) v = -1;
    ctl[q] = v;
  }
  for (size_t q = tid; q < (size_t)n_fact; q += stride) {
    ord[q] = fact[q];
    nodeA[q] = froot[q];
  }
  for (size_t q = tid; q < ncnt9; q += stride) cnt9[q] = 0;
}

__device__ void pack_one(const PackArgs &P, int k, int what) {
  pack_node(k, P.nroots, P.pos, P.width, P.cent, P.circ, P.C, P.count, P.child_first, P.nchild,
            P.cmask, P.first, P.x, P.gi, P.inf, P.beh, P.theta, P.extra, P.w64, P.p64, P.w32,
            P.c32, P.p32, P.leaf_of, P.n_leaf, P.full, what);
}



// Walk packs of the nodes of at most max_count points once their moments are
// in (a forest: every node, max_count = INT_MAX; a single tree: the nodes
// k_moments sums, the other kernels pack theirs).  root_cent: the single tree's
// root centroid, read here in place of cent[0..2] (the chain that makes it runs
// on its own stream), or null when the roots' centroids are in place.
__global__ void k_pack_nodes(const int *__restrict__ ctl, int cap_nodes, PackArgs pk,
                             const double *root_cent, double *cent, int max_count) {
  if (ctl[CTL_OVERFLOW]) return;
  const int n_nodes = min(ctl[CTL_NNODES], cap_nodes);
  if (root_cent && blockIdx.x == 0 && threadIdx.x < 3) cent[threadIdx.x] = root_cent[threadIdx.x];
  __syncthreads();
  // node 0 falls to block 0, which made the copy before the barrier
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_nodes; k += gridDim.x * blockDim.x)
    if (pk.count[k] <= max_count) pack_one(pk, k, 3);
}

// The late payloads are in (k_moments_big packs them): set the ready flag of
// list = [count, nodes..., flag at 15] (release), which the mixed walk's first
// launch reads before it takes a task that needs them.
__global__ void k_l1_ready(int *list) {
  __threadfence();
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(list + 15), "r"(1) : "memory");
}

// --------------------------------------------------------------- host side
static int tree_reserve(qv_ctx *c, int n_act, int cap_nodes, int cap_levels) {
  TreeBuf &t = c->tree;
  int rc;
  if (n_act > t.cap_pts || cap_levels > t.cap_levels) {
    int np = std::max(n_act, t.cap_pts);
    int nl = std::max(cap_levels, t.cap_levels);
    if ((rc = qv_grow(c, (void **)&t.ord, sizeof(int) * (size_t)np * nl))) return rc;
    t.cap_levels = nl;
    if (np > t.cap_pts) {
      if ((rc = qv_grow(c, (void **)&t.nodeA, sizeof(int) * np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.nodeB, sizeof(int) * np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.dig, np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.rnk, sizeof(int) * np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.leaf_of, sizeof(int) * np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.permb, sizeof(int) * np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.root_xc, sizeof(double) * 3 * (size_t)np))) return rc;
      if ((rc = qv_grow(c, (void **)&t.cnt9, sizeof(int) * 9 * (size_t)(2 * np + 2)))) return rc;
      if ((rc = qv_grow(c, (void **)&t.rs9, sizeof(int) * 9 * (size_t)(np + 1)))) return rc;
      if ((rc = qv_grow(c, (void **)&t.chunk9, sizeof(int) * 9 * (size_t)(np / CH + 2)))) return rc;
      t.cap_pts = np;
    }
  }
  if (!t.ctl)
    if ((rc = qv_grow(c, (void **)&t.ctl, sizeof(int) * CTL_SIZE))) return rc;
  if (!t.l1list)
    if ((rc = qv_grow(c, (void **)&t.l1list, sizeof(int) * 16))) return rc;
  if (cap_nodes > t.cap_nodes) {
    size_t m = cap_nodes;
    if ((rc = qv_grow(c, (void **)&t.pos, sizeof(double) * 3 * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.width, sizeof(double) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.cent, sizeof(double) * 3 * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.circ, sizeof(double) * 3 * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.C, sizeof(double) * 9 * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.count, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.start, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.parent, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.child_first, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.nchild, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.first, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.level, sizeof(int) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.digit, m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.cmask, m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.w64, sizeof(WNode64) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.p64, sizeof(WPay64) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.w32, sizeof(WNode32) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.c32, sizeof(SNode32) * m))) return rc;
    if ((rc = qv_grow(c, (void **)&t.p32_raw, sizeof(WPay32) * (m + 1)))) return rc;
    t.p32 = t.p32_raw + 1;
    t.cap_nodes = cap_nodes;
  }
  return QV_OK;
}

int qv_aux_streams(qv_ctx *c) {
  if (c->aux[0]) return QV_OK;
  QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_fork2, cudaEventDisableTiming));
  QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
  // the long moment chains (aux[0], aux[3], aux[4]) get the highest priority:
  // their blocks go first when the build's other kernels free SMs
  int lo_pri = 0, hi_pri = 0;
  QV_CUDA(c, cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
  for (int k = 0; k < 5; k++) {
    const int pri = (k == 0 || k >= 3) ? hi_pri : lo_pri;
    QV_CUDA(c, cudaStreamCreateWithPriority(&c->aux[k], cudaStreamNonBlocking, pri));
    QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_join[k], cudaEventDisableTiming));
  }
  QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_l1, cudaEventDisableTiming));
  QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_l1list, cudaEventDisableTiming));
  QV_CUDA(c, cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  QV_CUDA(c, cudaFuncSetAttribute(k_moments_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * MC * 15 * (int)sizeof(double)));
  QV_CUDA(c, cudaFuncSetAttribute(k_root_cent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * RC * 3 * (int)sizeof(double)));
  return QV_OK;
}

// Co-resident blocks of the cooperative build on this context's device.
static int build_grid(qv_ctx *c) {
  if (c->build_grid) return c->build_grid;
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_build, BT, 0);
  if (per < 1) per = 1;
  if (per > 2) per = 2;
  c->build_grid = per * c->sm_count;
  return c->build_grid;
}

static PackArgs pack_args(qv_ctx *c, int nroots, int *leaf_of, int n_leaf) {
  const TreeBuf &t = c->tree;
  PackArgs pk;
  pk.nroots = nroots;
  pk.pos = t.pos; pk.width = t.width; pk.cent = t.cent; pk.circ = t.circ; pk.C = t.C;
  pk.count = t.count; pk.child_first = t.child_first; pk.nchild = t.nchild; pk.cmask = t.cmask;
  pk.first = t.first; pk.x = c->x; pk.gi = c->gi; pk.inf = c->infront; pk.beh = c->behind;
  pk.theta = c->p.tree_theta; pk.extra = c->p.tree_extra_correction;
  pk.w64 = t.w64; pk.p64 = t.p64; pk.w32 = t.w32; pk.c32 = t.c32; pk.p32 = t.p32;
  pk.leaf_of = leaf_of; pk.n_leaf = n_leaf;
  pk.full = 1;
  return pk;
}

int qv_launch_tree_build(qv_ctx *c) {
  TreeBuf &t = c->tree;
  t.valid = false;
  int rc;
  if (!c->ghosts_valid)
    if ((rc = qv_launch_ghosts(c))) return rc;
  // The active count stays on the device (c->d_nact); every launch below is
  // sized by the slot count n, so the host does not wait for the compaction.
  if ((rc = qv_compact_active_async(c))) return rc;
  const int n = c->n;
  if ((rc = qv_aux_streams(c))) return rc;
  // a chain of an earlier build that no reader joined still reads root_xc
  if (t.root_pending) {
    QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[1], 0));
    t.root_pending = false;
  }
  // ... or the node tables (late level-1 chains and payloads)
  if (t.l1_pending) {
    QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_l1, 0));
    t.l1_pending = false;
  }
  t.l1_late = false;
  // The mixed walk of a large tree takes the root children's far-field terms
  // after its own launch (their circ and Cij chains, two dependent roundings per
  // point over up to an eighth of the points, would otherwise hold the walk back).
  const bool late = c->p.precision == QV_PREC_MIXED && c->p.velocity == QV_VEL_TREE &&
                    (g_l1_late_mode > 0 || (g_l1_late_mode < 0 && n >= QV_L1_LATE_MIN));
  if (!t.root_est) {
    QV_CUDA(c, cudaMalloc((void **)&t.root_est, 8 * sizeof(double)));
    QV_CUDA(c, cudaMalloc((void **)&t.root_ctl, 4 * sizeof(int)));
    QV_CUDA(c, cudaMalloc((void **)&t.root_unc, QV_ROOT_UNC_CAP * sizeof(int4)));
    QV_CUDA(c, cudaMalloc((void **)&t.root_part, 6 * QV_ROOT_EST_BLOCKS * sizeof(double)));
    QV_CUDA(c, cudaMemsetAsync(t.root_ctl, 0, 4 * sizeof(int), c->stream));
  }
  if ((rc = tree_reserve(c, n, std::max(t.cap_nodes, 4 * n + 64),
                         std::max(t.cap_levels, std::min(QV_MAX_DEPTH + 1, 40)))))
    return rc;
  // The root centroid (the reference's sequential sum, src/tree.f90:53-55)
  // is a chain of n dependent FP64 adds.  On large trees it runs on a side
  // stream over a private copy of the active positions and is joined only by
  // the first reader of the tree after the walk's launch; the build and the
  // walk use the bounded estimate k_root_est makes here (see root_open).  On
  // small trees the chain is short: it starts here, beside the build (whose
  // cooperative grid then leaves SMs free), and the packs wait for it.
  const bool spec = g_root_spec_mode > 0 || (g_root_spec_mode < 0 && n >= QV_ROOT_SPEC_MIN);
  if (spec) {
    k_root_est<<<QV_ROOT_EST_BLOCKS, 256, 0, c->stream>>>(c->d_nact, c->act, c->x, t.root_xc,
                                                          t.root_part, t.root_ctl, t.root_est,
                                                          g_root_bound_scale);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
  } else {
    QV_CUDA(c, cudaEventRecord(c->ev_fork, c->stream));
    QV_CUDA(c, cudaStreamWaitEvent(c->aux[1], c->ev_fork, 0));
    k_root_cent<<<1, 512, 2 * RC * 3 * sizeof(double), c->aux[1]>>>(c->d_nact, c->act, c->x,
                                                                     t.root_est + 4);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    QV_CUDA(c, cudaEventRecord(c->ev_join[1], c->aux[1]));
  }
  bool chain_started = !spec;
  if (!t.h_ctl) {
    QV_CUDA(c, cudaMallocHost((void **)&t.h_ctl, sizeof(int) * CTL_SIZE));
    QV_CUDA(c, cudaEventCreateWithFlags(&t.ev_ctl, cudaEventDisableTiming));
  }
  int cap_nodes = std::max(t.cap_nodes, 4 * n + 64);
  int cap_levels = std::max(t.cap_levels, std::min(QV_MAX_DEPTH + 1, 40));
  for (int attempt = 0; attempt < 8; attempt++) {
    if ((rc = tree_reserve(c, n, cap_nodes, cap_levels))) return rc;
    qv_phase_begin(c, PH_BUILD_LEVELS);
    k_build_init<<<2 * c->sm_count, 256, 0, c->stream>>>(
        t.pos, t.width, t.count, t.start, t.parent, t.child_first, t.nchild, t.level, t.digit,
        t.cmask, t.first, c->p.box_size, n, t.ctl, t.ord, c->act, t.nodeA, t.cnt9,
        9 * (size_t)(2 * t.cap_pts + 2));
    QV_LAUNCH_CHECK(c);
    BuildArgs a;
    a.d_nact = c->d_nact; a.n_slots = n; a.cap_pts = t.cap_pts; a.cap_nodes = t.cap_nodes;
    a.cap_levels = t.cap_levels; a.nchunks = std::max(1, nblk(n, CH));
    a.x = c->x; a.gi = c->gi; a.pos = t.pos; a.width = t.width; a.count = t.count;
    a.start = t.start; a.parent = t.parent; a.child_first = t.child_first; a.nchild = t.nchild;
    a.level = t.level; a.digit = t.digit; a.cmask = t.cmask; a.ord = t.ord; a.nodeA = t.nodeA;
    a.nodeB = t.nodeB; a.rnk = t.rnk; a.cnt9A = t.cnt9; a.cnt9B = t.cnt9 + 9 * (size_t)(t.cap_pts + 1);
    a.rs9 = t.rs9; a.chunk9 = t.chunk9; a.ctl = t.ctl; a.dig = t.dig; a.perm = t.permb;
    int grid = std::min(build_grid(c), std::max(1, a.nchunks) * 4);
    grid = std::max(grid, 1);
    void *args[] = {&a};
    QV_CUDA(c, cudaLaunchCooperativeKernel((void *)k_build, grid, BT, args, 0, c->stream));
    QV_COUNT(c, 2);
    // the chains of the big nodes (all made by the grid-wide levels) start on a
    // side stream while the block-local levels finish the tree
    QV_CUDA(c, cudaEventRecord(c->ev_fork, c->stream));
    QV_CUDA(c, cudaStreamWaitEvent(c->aux[0], c->ev_fork, 0));
    if (!chain_started) {
      // the root centroid's chain starts behind the cooperative kernel, whose
      // blocks must all be resident at once: a one-block kernel holding an
      // SM's shared memory would delay it until the chain ended
      QV_CUDA(c, cudaStreamWaitEvent(c->aux[1], c->ev_fork, 0));
      k_root_cent<<<1, 512, 2 * RC * 3 * sizeof(double), c->aux[1]>>>(c->d_nact, nullptr,
                                                                       t.root_xc, t.root_est + 4);
      QV_LAUNCH_CHECK(c);
      QV_COUNT(c, 1);
      QV_CUDA(c, cudaEventRecord(c->ev_join[1], c->aux[1]));
      t.root_pending = true;
      chain_started = true;
    }
    QV_CUDA(c, cudaMemsetAsync(t.ctl + CTL_NBIG, 0, sizeof(int), c->aux[0]));
    k_list_big<<<4 * c->sm_count, 256, 0, c->aux[0]>>>(t.ctl, t.cap_nodes, 1, t.count, t.rnk,
                                                        t.ctl + CTL_NBIG, BIGN, INT_MAX, 1,
                                                        late ? 1 : 0);
    const PackArgs pk = pack_args(c, 1, t.leaf_of, n);
    k_moments_big<<<2 * c->sm_count, MBT, 2 * MC * 15 * sizeof(double), c->aux[0]>>>(
        t.rnk, t.ctl + CTL_NBIG, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, c->gi,
        t.cent, t.circ, t.C, t.first, 0, pk, 1);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 2);
    if (late) {
      // the big root children: their centroid chains (aux[4]; the packs wait
      // for them), their circ and Cij chains and then their payloads (aux[3];
      // event ev_l1, joined after the walk's launch)
      cudaStream_t s3 = c->aux[3], s4 = c->aux[4];
      QV_CUDA(c, cudaStreamWaitEvent(s3, c->ev_fork, 0));
      QV_CUDA(c, cudaMemsetAsync(t.l1list, 0, 16 * sizeof(int), s3));  // count, ready flag
      k_list_big<<<1, 256, 0, s3>>>(t.ctl, t.cap_nodes, 1, t.count, t.l1list + 1, t.l1list, BIGN,
                                    INT_MAX, 1, 2);
      QV_LAUNCH_CHECK(c);
      QV_CUDA(c, cudaEventRecord(c->ev_l1list, s3));
      QV_CUDA(c, cudaStreamWaitEvent(s4, c->ev_l1list, 0));
      k_moments_cent<<<8, MBT, 2 * MCC * 3 * sizeof(double), s4>>>(
          t.ctl, t.l1list, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, t.cent, t.first, pk);
      QV_LAUNCH_CHECK(c);
      QV_CUDA(c, cudaEventRecord(c->ev_join[4], s4));
      k_moments_big<<<8, MBT, 2 * MC * 15 * sizeof(double), s3>>>(
          t.l1list + 1, t.l1list, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, c->gi,
          t.cent, t.circ, t.C, t.first, 1, pk, 1);
      QV_LAUNCH_CHECK(c);
      k_l1_ready<<<1, 1, 0, s3>>>(t.l1list);
      QV_LAUNCH_CHECK(c);
      QV_CUDA(c, cudaEventRecord(c->ev_l1, s3));
      QV_COUNT(c, 4);
    }
    k_build_local<<<std::max(1, std::min(nblk(n, LCH), 2 * c->sm_count)), BT, LOCAL_SMEM,
                    c->stream>>>(a);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    qv_phase_end_async(c, PH_BUILD_LEVELS);
    qv_phase_begin(c, PH_BUILD_MOMENTS);
    // After the local levels, on a third stream: the control block to the host
    // and the moments of the nodes of MIDN..BIGN points (a block each); here,
    // the warp-per-node moments.  Every moment kernel packs the nodes it
    // finishes; the root is packed once its centroid (second stream) is in.
    QV_CUDA(c, cudaEventRecord(c->ev_fork2, c->stream));
    QV_CUDA(c, cudaStreamWaitEvent(c->aux[2], c->ev_fork2, 0));
    QV_CUDA(c, cudaMemcpyAsync(t.h_ctl, t.ctl, sizeof(int) * CTL_SIZE, cudaMemcpyDeviceToHost,
                               c->aux[2]));
    QV_CUDA(c, cudaEventRecord(t.ev_ctl, c->aux[2]));
    QV_CUDA(c, cudaMemsetAsync(t.ctl + CTL_NMID, 0, sizeof(int), c->aux[2]));
    k_list_big<<<4 * c->sm_count, 256, 0, c->aux[2]>>>(t.ctl, t.cap_nodes, 1, t.count, t.rs9,
                                                        t.ctl + CTL_NMID, MIDN, BIGN, 0, 0);
    k_moments_big<<<2 * c->sm_count, MBT, 2 * MC * 15 * sizeof(double), c->aux[2]>>>(
        t.rs9, t.ctl + CTL_NMID, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, c->gi,
        t.cent, t.circ, t.C, t.first, 0, pk, 1);
    QV_CUDA(c, cudaEventRecord(c->ev_join[2], c->aux[2]));
    QV_COUNT(c, 2);
    k_moments<<<16 * c->sm_count, MW * 32, 0, c->stream>>>(t.ctl, t.cap_nodes, 1, t.level, t.start,
                                                           t.count, t.ord, t.cap_pts, c->x, c->gi,
                                                           t.cent, t.circ, t.C, t.first);
    QV_LAUNCH_CHECK(c);
    // the packs of those nodes (of at most MIDN points) here, while the longer
    // chains run on; the chain kernels pack the nodes they finish.  Four times
    // the blocks of a full pack: each thread's few nodes are dependent loads
    // (first point, its links), and more of them in flight shortened this pass
    // by 0.13 ms at 0.8M points.
    k_pack_nodes<<<16 * c->sm_count, 128, 0, c->stream>>>(t.ctl, t.cap_nodes, pk, nullptr, t.cent,
                                                           MIDN);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 2);
    QV_CUDA(c, cudaEventRecord(c->ev_join[0], c->aux[0]));
    QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[0], 0));
    QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[2], 0));
    if (!spec) QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[1], 0));
    if (late) QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[4], 0));
    // every other node was packed by the kernel that summed its moments
    k_root_pack<<<1, 32, 0, c->stream>>>(pk, spec ? t.root_est : t.root_est + 4, t.cent);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    qv_phase_end_async(c, PH_BUILD_MOMENTS);
    QV_CUDA(c, cudaEventSynchronize(t.ev_ctl));
    const int *hc = t.h_ctl;
    if (hc[CTL_OVERFLOW]) {
      // the queued moment/pack kernels saw the flag and did nothing
      QV_CUDA(c, cudaStreamSynchronize(c->stream));
      if (late) QV_CUDA(c, cudaStreamSynchronize(c->aux[3]));
      if (hc[CTL_OVERFLOW] == 1) {
        cap_nodes *= 2;
        continue;
      }
      if (cap_levels >= QV_MAX_DEPTH + 1)
        return qv_fail(c, QV_ERR_TREE_DEPTH,
                       "octree deeper than %d levels (coincident or nearly coincident points)",
                       QV_MAX_DEPTH);
      cap_levels = QV_MAX_DEPTH + 1;
      continue;
    }
    t.n_nodes = hc[CTL_NNODES];
    t.depth = hc[CTL_DEPTH];
    t.n_act = hc[CTL_NACT];
    c->n_act = t.n_act;
    t.lvl_start.assign(hc + CTL_LVL, hc + CTL_LVL + t.depth + 2);
    t.perm = t.permb;
    t.n_leaf = n;
    t.valid = true;
    t.l1_late = t.l1_pending = late;
    return QV_OK;
  }
  return qv_fail(c, QV_ERR_NOMEM, "tree build did not fit after repeated growth");
}

extern "C" int qv_root_undecided(qv_ctx *c, int *count) {
  if (!c || !count) return QV_ERR_ARG;
  *count = 0;
  if (!c->tree.root_ctl) return QV_OK;
  if (cudaMemcpyAsync(count, c->tree.root_ctl, sizeof(int), cudaMemcpyDeviceToHost, c->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return qv_fail(c, QV_ERR_CUDA, "qv_root_undecided: copy failed");
  return QV_OK;
}

int qv_tree_finalize_root(qv_ctx *c) {
  TreeBuf &t = c->tree;
  if (t.l1_pending) {
    t.l1_pending = false;
    QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_l1, 0));
  }
  if (!t.root_pending) return QV_OK;
  t.root_pending = false;
  QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[1], 0));
  if (!t.valid) return QV_OK;
  k_root_pack<<<1, 32, 0, c->stream>>>(pack_args(c, 1, t.leaf_of, c->n), t.root_est + 4, t.cent);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

// ------------------------------------------------------------------ forest
// Independent systems' trees built together: one root per system at level 0,
// then the same level-synchronous kernel, moment chains and packs as a single
// tree.  Nothing here waits for the host, so a step that contains the build can
// be captured in a CUDA graph; capacities are reserved up front and an
// overflow leaves CTL_OVERFLOW set for the caller to read.
int qv_forest_reserve(qv_ctx *c, int n_fact, int cap_nodes) {
  int rc;
  if ((rc = qv_aux_streams(c))) return rc;
  QV_CUDA(c, cudaFuncSetAttribute(k_forest_root_cent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * RC * 3 * (int)sizeof(double)));
  return tree_reserve(c, std::max(n_fact, 1), cap_nodes, QV_MAX_DEPTH + 1);
}

int qv_forest_build(qv_ctx *c, const ForestArgs &f) {
  TreeBuf &t = c->tree;
  if (f.n_fact > t.cap_pts || t.cap_levels < QV_MAX_DEPTH + 1)
    return qv_fail(c, QV_ERR_STATE, "forest build without reserved capacity");
  k_forest_init<<<2 * c->sm_count, 256, 0, c->stream>>>(
      f.nroots, f.roots, t.pos, t.width, t.count, t.start, t.parent, t.child_first, t.nchild,
      t.level, t.digit, t.cmask, t.first, c->p.box_size, f.n_fact, t.ctl, t.ord, f.fact, f.froot,
      t.nodeA, t.cnt9, 9 * (size_t)(2 * t.cap_pts + 2));
  QV_LAUNCH_CHECK(c);
  BuildArgs a;
  a.d_nact = f.d_nfact; a.n_slots = f.n_fact; a.cap_pts = t.cap_pts; a.cap_nodes = t.cap_nodes;
  a.cap_levels = t.cap_levels; a.nchunks = std::max(1, nblk(f.n_fact, CH));
  a.x = c->x; a.gi = c->gi; a.pos = t.pos; a.width = t.width; a.count = t.count;
  a.start = t.start; a.parent = t.parent; a.child_first = t.child_first; a.nchild = t.nchild;
  a.level = t.level; a.digit = t.digit; a.cmask = t.cmask; a.ord = t.ord; a.nodeA = t.nodeA;
  a.nodeB = t.nodeB; a.rnk = t.rnk; a.cnt9A = t.cnt9; a.cnt9B = t.cnt9 + 9 * (size_t)(t.cap_pts + 1);
  a.rs9 = t.rs9; a.chunk9 = t.chunk9; a.ctl = t.ctl; a.dig = t.dig; a.perm = t.permb;
  int grid = std::max(1, std::min(build_grid(c), std::max(1, a.nchunks) * 4));
  // a cooperative launch written as a launch attribute, which stream capture
  // records as a cooperative kernel node
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(BT);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // the roots' centroid chains need only the active slots: a side stream,
  // from the start (the events fork and join inside a captured graph too)
  QV_CUDA(c, cudaEventRecord(c->ev_fork, c->stream));
  QV_CUDA(c, cudaStreamWaitEvent(c->aux[1], c->ev_fork, 0));
  k_forest_root_cent<<<std::min(f.nroots, 2 * c->sm_count), 512, 2 * RC * 3 * sizeof(double),
                       c->aux[1]>>>(f.nroots, f.roots, f.fact, c->x, t.ctl, t.cent);
  QV_CUDA(c, cudaEventRecord(c->ev_join[1], c->aux[1]));
  QV_CUDA(c, cudaLaunchKernelEx(&cfg, k_build, a));
  // the chains of the nodes of more than BIGN points (all made by the
  // grid-wide levels) on another side stream while the local levels run
  QV_CUDA(c, cudaEventRecord(c->ev_fork2, c->stream));
  QV_CUDA(c, cudaStreamWaitEvent(c->aux[0], c->ev_fork2, 0));
  QV_CUDA(c, cudaMemsetAsync(t.ctl + CTL_NBIG, 0, sizeof(int), c->aux[0]));
  k_list_big<<<4 * c->sm_count, 256, 0, c->aux[0]>>>(t.ctl, t.cap_nodes, f.nroots, t.count, t.rnk,
                                                      t.ctl + CTL_NBIG, BIGN, INT_MAX, 1, 0);
  PackArgs pk = pack_args(c, f.nroots, nullptr, 0);
  pk.full = 0;  // the batch runs the mixed walk only and no candidate search
  k_moments_big<<<2 * c->sm_count, MBT, 2 * MC * 15 * sizeof(double), c->aux[0]>>>(
      t.rnk, t.ctl + CTL_NBIG, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, c->gi, t.cent,
      t.circ, t.C, t.first, 0, pk, 0);
  QV_CUDA(c, cudaEventRecord(c->ev_join[0], c->aux[0]));
  k_build_local<<<std::max(1, std::min(nblk(f.n_fact, LCH), 2 * c->sm_count)), BT, LOCAL_SMEM,
                  c->stream>>>(a);
  QV_CUDA(c, cudaMemsetAsync(t.ctl + CTL_NMID, 0, sizeof(int), c->stream));
  k_list_big<<<4 * c->sm_count, 256, 0, c->stream>>>(t.ctl, t.cap_nodes, f.nroots, t.count, t.rs9,
                                                      t.ctl + CTL_NMID, MIDN, BIGN, 0, 0);
  k_moments_big<<<2 * c->sm_count, MBT, 2 * MC * 15 * sizeof(double), c->stream>>>(
      t.rs9, t.ctl + CTL_NMID, t.level, t.start, t.count, t.ord, t.cap_pts, c->x, c->gi, t.cent,
      t.circ, t.C, t.first, 0, pk, 0);
  k_moments<<<16 * c->sm_count, MW * 32, 0, c->stream>>>(t.ctl, t.cap_nodes, f.nroots, t.level,
                                                         t.start, t.count, t.ord, t.cap_pts, c->x,
                                                         c->gi, t.cent, t.circ, t.C, t.first);
  QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[0], 0));
  QV_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join[1], 0));
  k_pack_nodes<<<4 * c->sm_count, 128, 0, c->stream>>>(t.ctl, t.cap_nodes, pk, nullptr, t.cent,
                                                        INT_MAX);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 10);
  return QV_OK;
}
