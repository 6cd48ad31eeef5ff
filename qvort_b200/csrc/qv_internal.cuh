// qv_internal.cuh -- shared definitions of the B200 filament path.
//
// Device data layout (HBM): one context holds one filament system.  Point
// arrays keep the reference's slot order and interleaved xyz (x[3*i+c]) so a
// host gather of f(:) copies straight in; links stay 1-based with 0 = empty.
// The octree lives in flat node tables (breadth-first levels, children of a
// node contiguous in the fbl..btr order), with walk-ready FP64 and FP32 packs.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/qv.h"

#define QV_PI 3.14159265358979324  // src/cdata.f90:176
#define QV_DEPS 2.220446049250313e-16  // epsilon(0.) under -fdefault-real-8

// Bits of the device status word (qv_ctx::dstatus)
#define QV_STAT_SINGULAR 1  // a tree leaf closer than epsilon (src/tree.f90:372-376)
#define QV_STAT_STACK 2     // walk or search stack overflow
#define QV_STAT_HEAP 4      // a line scan's re-test heap overflowed
#define QV_STAT_STAGE 8     // a direct-sum source-tile copy did not land in time
#define QV_STAT_NAN 16      // a NaN in the positions at the end of a step

// Walk-ready node header, FP64 (64 B).  cent, width and the geometric offset
// geo = |cent - cell centre| (src/tree.f90:355-357) in FP64 so that every
// opening decision is taken exactly as the reference takes it.
struct __align__(16) WNode64 {
  double cx, cy, cz;
  double width, geo;
  int count;        // pcount (the root counts every slot, src/tree.f90:51)
  int child_first;  // first non-empty child; children are contiguous
  int nchild;       // number of non-empty children
  int jb;           // leaf: f(parray(1)%infront)%behind at build time (1-based)
  int finf;         // parray(1)%infront at build time (1-based)
  int first;        // slot of parray(1) (0-based), -1 if none
};

// FP64 payload (128 B): leaf -> segment x, ghosti; internal -> circ, the
// antisymmetric contraction w_m = sum_kl eps(m,k,l) C(k,l), and C (row-major).
struct __align__(16) WPay64 {
  double a[3];   // leaf x | circ
  double b[3];   // leaf gi | w
  double C[9];
  double pad;
};

// FP32 header (48 B): cent as a two-float (hi, lo) split of the FP64 value so
// that target-source differences keep FP64-level information, and the node's
// opening radius squared widened by a relative 4e-6 either way: a squared
// distance above rhi passes the test, one below rlo fails it, one in between
// is decided by the reference's FP64 expression.  w32 holds these headers for
// the velocity walk (radius geo + width/theta; rhi = rlo = -1 when only the
// FP64 test is valid).  See k_pack_nodes.
struct __align__(16) WNode32 {
  float ch[3], cl[3];
  float rhi, rlo;
  int count, child_first, nchild, jb;
};

// Candidate-search header (64 B): the same centroid split and widened radius
// for theta = width/dist < 0.5 (radius 2 width), plus the cell's box as an
// FP32 corner rounded down and a width rounded up, so that a lower bound on
// the distance from a target to anything inside the cell costs a few FP32
// operations, and the digits of the children present (bit g = child g).
struct __align__(16) SNode32 {
  float ch[3], cl[3];
  float rhi, rlo;
  float lo[3], w;
  int count, child_first, nchild, cmask;
};

// FP32 payload (64 B): internal -> circ, w, C; leaf -> ghosti as (hi, lo)
// and the segment vector s = ghosti - x in C[0..2].
struct __align__(16) WPay32 {
  float a[3];  // circ | gi hi
  float b[3];  // w | gi lo
  float C[9];  // C | s
  float pad;
};

struct TreeBuf {
  int cap_nodes = 0;  // allocated node slots
  int cap_pts = 0;    // allocated point slots (active points)
  int cap_levels = 0; // levels of per-level order storage
  int n_nodes = 0, depth = 0, n_act = 0;
  bool valid = false;
  // node records (build)
  double *pos = nullptr, *width = nullptr, *cent = nullptr, *circ = nullptr, *C = nullptr;
  int *count = nullptr, *start = nullptr, *parent = nullptr, *child_first = nullptr,
      *nchild = nullptr, *first = nullptr, *level = nullptr;
  unsigned char *digit = nullptr, *cmask = nullptr;
  // walk packs
  WNode64 *w64 = nullptr;
  WPay64 *p64 = nullptr;
  WNode32 *w32 = nullptr;
  SNode32 *c32 = nullptr;
  WPay32 *p32 = nullptr;  // = p32_raw + 1: node 1's payload starts a 128-byte line
  WPay32 *p32_raw = nullptr;
  // build scratch
  int *ord = nullptr;       // cap_levels * cap_pts: per-level orders
  int *nodeA = nullptr, *nodeB = nullptr;  // node of each position
  unsigned char *dig = nullptr;
  int *rnk = nullptr;
  int *cnt9 = nullptr, *rs9 = nullptr;     // per node of a level
  int *chunk9 = nullptr;                   // per chunk of positions
  int *ctl = nullptr;                      // device control block
  int *perm = nullptr;                     // final (DFS) order of active points
  int *permb = nullptr;                    // its storage, written by the build
  int *leaf_of = nullptr;                  // slot -> its one-point leaf (unverified)
  int n_leaf = 0;                          // slots covered by leaf_of
  int *h_ctl = nullptr;                    // pinned copy of the control block
  cudaEvent_t ev_ctl = nullptr;
  std::vector<int> lvl_start;
  // Root centroid.  The exact value (the reference's sequential sum, a chain
  // of n dependent FP64 adds) runs on a side stream; until it is joined the
  // root's headers hold an estimate whose distance from it is bounded:
  // root_est = [estimate (3), bound, exact (3), spare].  root_ctl = [count of
  // root decisions left undecided by the bound, spare, redo flag, ticket].
  double *root_est = nullptr;
  int *root_ctl = nullptr;
  int4 *root_unc = nullptr;  // the undecided (target, task slot, evals, far evals)
  double *root_part = nullptr;  // per-block partial sums of the estimate
  double *root_xc = nullptr;    // the active positions in active order (the chain's input)
  bool root_pending = false;    // headers hold the estimate
  // Late level-1 moments.  The circ and Cij chains of the root's children of
  // more than QV_L1_BIG points are the longest sequential sums of a large tree
  // (two dependent roundings per point).  In a mixed-precision Tree build of at
  // least QV_L1_LATE_MIN slots they run on a side stream while the walk runs:
  // those nodes' headers (centroid from its own, shorter chain) are packed with
  // the rest, their payloads once the chains end (event ev_l1 of the context).
  // l1list = [count, nodes...].
  int *l1list = nullptr;
  bool l1_late = false;     // this tree's big level-1 payloads come late
  bool l1_pending = false;  // ... and no reader has joined them yet
};
#define QV_L1_LATE_MIN 65536  // slots from which a mixed Tree build packs level 1 late
#define QV_L1_BIG 512         // level-1 nodes of more points take the late path

// Whether root child k (1 <= k < l1_end, the level-1 nodes) takes the late
// path: it and the node that shares its 128-byte line of FP32 payloads (the
// walk reads those through L1, and node 1 starts a line) hold more than
// QV_L1_BIG points each.  A line that an early reader brought into L1 then
// never also holds a late payload.
__host__ __device__ inline bool qv_l1_late(int k, int l1_end, int count_k, int count_pair) {
  const int j = ((k - 1) ^ 1) + 1;  // its line partner
  return k >= 1 && k < l1_end && j < l1_end && count_k > QV_L1_BIG && count_pair > QV_L1_BIG;
}
__host__ __device__ inline int qv_l1_pair(int k) { return ((k - 1) ^ 1) + 1; }
#define QV_ROOT_UNC_CAP 8192
#define QV_ROOT_SPEC_MIN 32768  // slots from which the root starts from its estimate
#define QV_ROOT_EST_BLOCKS 296

// Phases timed with CUDA events when profiling is on (qv_profile).
enum {
  PH_GHOSTS = 0, PH_BUILD, PH_LIA, PH_NONLOCAL, PH_UPDATE, PH_CLOSEST, PH_WRAP,
  PH_BUILD_LEVELS,   // inside PH_BUILD: init + the level-synchronous kernel
  PH_BUILD_MOMENTS,  // inside PH_BUILD: moment chains, root centroid join, packs
  PH_LINE,           // pinsert / premove
  PH_WALK,           // inside PH_NONLOCAL: the mixed walk's kernel alone (its first launch)
  PH_N
};

struct qv_ctx {
  qv_params p;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int n = 0, cap = 0;
  double *x = nullptr, *u = nullptr, *u1 = nullptr, *u2 = nullptr, *u3 = nullptr;
  double *gi = nullptr, *gb = nullptr, *gii = nullptr, *gbb = nullptr;
  double *u_li = nullptr, *u_bs = nullptr, *closestd = nullptr;
  int *infront = nullptr, *behind = nullptr, *closest = nullptr;
  int *act = nullptr;  // compacted active slots (direct sums)
  int n_act = 0;
  int *d_nact = nullptr;  // device copy of n_act (tree path)
  int *blkcnt = nullptr;  // per-256-slot block counts of the compaction (n/256+2)
  double *dpart = nullptr;  // direct-sum partial sums, grown on demand
  size_t dpart_bytes = 0;
  // adjoint scratch: per-point adjoints of x and the four ghosts, per-node
  // adjoints of (cent, circ, Cij)
  double *adj_xb = nullptr, *adj_gib = nullptr, *adj_gbb = nullptr, *adj_giib = nullptr,
         *adj_gbbb = nullptr, *adj_nb = nullptr;
  int adj_n = 0;
  size_t adj_nb_bytes = 0;
  double *src64 = nullptr;  // direct-sum source pack (FP64)
  float *src32 = nullptr;   // direct-sum source pack (FP32 hi/lo)
  unsigned long long *evals = nullptr;  // device eval counter
  int *dstatus = nullptr;               // device status word
  double *dscalar = nullptr;            // device scalar scratch
  double *walk_part = nullptr;          // per-image partial sums of the walk
  int *walk_next = nullptr;             // the mixed walk's task counters
  int *lk = nullptr;                    // staged host links: infront, behind, closest, verdict
  size_t lk_ints = 0;
  int *h_lk = nullptr;                  // pinned: the link check's verdict
  size_t walk_part_bytes = 0;
  bool ghosts_valid = false;
  bool ghosts_stored = false;  // ghost arrays hold values (possibly from before a move)
  // line operations (pinsert / premove): flag and list scratch, sequential state
  void *line_flags = nullptr, *line_st = nullptr, *line_rec = nullptr;
  void *line_host = nullptr;       // pinned copy of the ordered passes' state
  int *line_clr = nullptr;         // slots the line operations cleared (QV_LINE_CLR_CAP)
  int *h_clr = nullptr;            // pinned: their count and the first QV_LINE_CLR_HOST
  cudaEvent_t ev_pins = nullptr;   // recorded behind each pinsert scan
  cudaEvent_t ev_line = nullptr;   // recorded when that copy is queued
  unsigned long long *h_stat = nullptr;  // pinned: evaluation counters and status word
  cudaEvent_t ev_in = nullptr;  // qv_step_exchange: the side-stream inputs are in
  bool in_pending = false;      // ... and the next update must wait for them
  size_t line_cap = 0;
  TreeBuf tree;
  int sm_count = 148;
  int build_grid = 0;  // co-resident blocks of the cooperative tree build
  size_t smem_walk = 0, smem_search = 0;  // dynamic shared memory opted in on this device
  // instrumentation
  bool profile = false;
  cudaEvent_t ev_beg[PH_N] = {}, ev_end[PH_N] = {};
  bool ev_pending[PH_N] = {};
  double phase_ms[PH_N] = {};
  long long launches = 0;
  unsigned long long *evals_far = nullptr;
  cudaStream_t aux[5] = {};  // side streams for independent chains
  cudaEvent_t ev_fork = nullptr, ev_fork2 = nullptr, ev_join[5] = {};
  cudaEvent_t ev_l1 = nullptr, ev_l1list = nullptr;  // late level-1 moments (TreeBuf)
  unsigned char *walk_defer = nullptr;  // per (task slot, target): deferred level-1 far cells
  size_t walk_defer_bytes = 0;
  long long last_leaf = 0, last_far = 0;
  char err[512] = {0};
};

// ---------------------------------------------------------------- errors
int qv_fail(qv_ctx *c, int code, const char *fmt, ...);
#define QV_CUDA(ctx, call)                                                     \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return qv_fail((ctx), QV_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__,   \
                     #call, cudaGetErrorString(e_));                           \
  } while (0)
#define QV_LAUNCH_CHECK(ctx) QV_CUDA(ctx, cudaGetLastError())

int qv_grow(qv_ctx *c, void **ptr, size_t bytes);
void qv_phase_begin(qv_ctx *c, int ph);
void qv_phase_end(qv_ctx *c, int ph);
void qv_phase_end_async(qv_ctx *c, int ph);
void qv_phase_collect(qv_ctx *c);
#define QV_COUNT(c, k) ((c)->launches += (k))

// ---------------------------------------------------------------- kernels
int qv_launch_ghosts(qv_ctx *c);
int qv_launch_lia(qv_ctx *c);
int qv_launch_direct(qv_ctx *c);
int qv_launch_tree_build(qv_ctx *c);
// Join the exact root centroid and re-pack the root with it, and join the late
// level-1 moments and payloads (no-op when both are in already).  Every reader
// of the tree calls it; the mixed walk after its launch.
int qv_tree_finalize_root(qv_ctx *c);
int qv_launch_walk(qv_ctx *c);
int qv_launch_ab(qv_ctx *c);
int qv_launch_rk3_stage(qv_ctx *c, int stage);
int qv_launch_wrap(qv_ctx *c);
int qv_launch_closest(qv_ctx *c);
int qv_launch_closest_ex(qv_ctx *c, const int *d_n, const int *d_skip, int n_grid);
// pinsert in two halves: everything queued (flags, lists, the ordered pass),
// then the wait for the new slot count (growing and resuming when the slots
// ran out; *resumed tells whether that happened)
int qv_line_insert_queue(qv_ctx *c);
int qv_line_insert_finish(qv_ctx *c, int *inserted, bool *resumed);
const int *qv_line_count_dev(qv_ctx *c);   // device slot count after pinsert
const int *qv_line_status_dev(qv_ctx *c);  // device status of the ordered passes
int qv_launch_energy(qv_ctx *c, double *out_host);
int qv_compact_active(qv_ctx *c);
int qv_grow_points(qv_ctx *c, int new_cap);
int qv_line_insert(qv_ctx *c, int *inserted);
int qv_line_remove(qv_ctx *c, int *removed);
int qv_line_reconnect(qv_ctx *c, int *count);
// The log of slots cleared by premove and reconnection (clear_particle):
// reset it, and queue the copy of its count and first entries to c->h_clr.
#define QV_LINE_CLR_CAP 65536
#define QV_LINE_CLR_HOST 4096
int qv_line_clear_log_reset(qv_ctx *c);
int qv_line_clear_log_queue(qv_ctx *c);
// ordered compaction kernels (qv_direct.cu): counts of nonzero flags per
// 256-slot block, their exclusive scan (total to *total), the scatter
__global__ void k_count_active(int n, const int *__restrict__ inf, int *blk_cnt);
__global__ void k_scan_small(int m, int *v, int *total);
__global__ void k_scatter_active(int n, const int *__restrict__ inf, const int *blk_off, int *act);
#define QV_COMPACT1_MAX 65536
__global__ void k_compact1(int n, const int *__restrict__ flag, int *out, int *total);
int qv_compact_active_async(qv_ctx *c);
int qv_aux_streams(qv_ctx *c);

// A forest of independent trees (one root per system) in c->tree.
// roots[r] = (first slot, slot count, first position in fact, active count);
// fact = the forest's active slots, each system's contiguous and ascending;
// froot[q] = root of position q; d_nfact = device copy of n_fact.
struct ForestArgs {
  int nroots = 0, n_fact = 0;
  const int4 *roots = nullptr;
  const int *fact = nullptr, *froot = nullptr, *d_nfact = nullptr;
};
int qv_forest_reserve(qv_ctx *c, int n_fact, int cap_nodes);
int qv_forest_build(qv_ctx *c, const ForestArgs &f);
// control-block words read by forest users on the device
#define QV_CTL_OVERFLOW 3
#define QV_CTL_DEPTH 4
#define QV_CTL_NNODES 0

// ---------------------------------------------------------------- helpers
// Straight-segment Biot-Savart term in FP32, without the G/(4 pi) factor:
//   (|R1|+|R2|) / (|R1||R2| (|R1||R2| + R1.R2)) * (R1 x R2)
// (src/tree.f90:380-390), written with q = 1/(|R1||R2|) as
//   (1/|R1| + 1/|R2|) q / (1 + cos) * (R1 x s),  cos = R1.R2 q,
// where s = ghosti - x is the segment vector (R2 = R1 + s).  R1 x R2 equals
// R1 x s, and the latter does not cancel when the segment is far away
// (R1 ~ R2); s is an FP64 difference rounded once to FP32.
// When cos < 0 the sum 1 + cos cancels; it is then taken from the identity
// (1 + cos)(1 - cos) = sin^2 = |R1 x s|^2 q^2, which has no cancellation.
__device__ __forceinline__ void qv_seg32(float r1x, float r1y, float r1z, float r2x, float r2y,
                                         float r2z, float sx, float sy, float sz, float r1s,
                                         float &ox, float &oy, float &oz) {
  float r2s = fmaf(r2x, r2x, fmaf(r2y, r2y, r2z * r2z));
  float dd = fmaf(r1x, r2x, fmaf(r1y, r2y, r1z * r2z));
  float ra = rsqrtf(r1s), rb = rsqrtf(r2s);
  float q = ra * rb;
  float cx = fmaf(r1y, sz, -r1z * sy);
  float cy = fmaf(r1z, sx, -r1x * sz);
  float cz = fmaf(r1x, sy, -r1y * sx);
  float cs = dd * q;
  float f = (ra + rb) * q;
  if (cs >= 0.f) {
    f = __fdividef(f, 1.f + cs);  // 1 + cos >= 1
  } else {
    const float den = fmaf(cx, cx, fmaf(cy, cy, cz * cz)) * (q * q) / (1.f - cs);
    f = den > 0.f ? __fdividef(f, den) : 0.f;
  }
  ox = f * cx;
  oy = f * cy;
  oz = f * cz;
}

__host__ __device__ inline int qv_img_count(int bc) {
  return bc == QV_BC_PERIODIC ? 26 : bc == QV_BC_OPENX ? 8 : bc == QV_BC_OPENXY ? 2 : 0;
}
// Shift multipliers of image m in the reference's loop order
// (src/timestep.f90:235-257): peri, perj, perk from -1..1, skipping 0,0,0.
__host__ __device__ inline void qv_img_shift(int bc, int m, int *a, int *b, int *cc) {
  if (bc == QV_BC_PERIODIC) {
    int q = m < 13 ? m : m + 1;
    *a = q / 9 - 1; *b = (q / 3) % 3 - 1; *cc = q % 3 - 1;
  } else if (bc == QV_BC_OPENX) {
    int q = m < 4 ? m : m + 1;
    *a = 0; *b = q / 3 - 1; *cc = q % 3 - 1;
  } else {
    *a = 0; *b = 0; *cc = m == 0 ? -1 : 1;
  }
}
