// qv_direct.cu -- direct desingularised Biot-Savart sum with periodic images
// (biot_savart / biot_savart_shift, src/timestep.f90:462-507), one thread per
// target, source segments staged tile by tile in shared memory.
//
// FP64 kernel: the reference's formula
//   u += G/(2 pi) (d x s)/(4ac - b^2) [(2c+b)/sqrt(a+b+c) - b/sqrt(a)]
// with d = x_j + shift - x_i, s = ghosti_j - x_j, a=|d|^2, b=2 d.s, c=|s|^2.
//
// Mixed kernel: FP32 pair terms in the stable straight-segment form the
// reference uses for tree leaves (src/tree.f90:380-390),
//   u += G/(4 pi) (|R1|+|R2|)/(|R1||R2|(|R1||R2| + R1.R2)) R1 x R2,
// with R1 = x_j + shift - x_i and R2 = ghosti_j + shift - x_i recentred on the
// target from FP64 data (every FP64 coordinate carried as a hi/lo float pair,
// so the difference keeps FP64-level information before it is rounded), and
// Kahan-compensated FP32 accumulation.  The two forms agree analytically; the
// stable one avoids the (2c+b)/sqrt - b/sqrt cancellation that FP32 cannot
// afford for far segments.
//
// Skip rules differ between the unshifted and shifted sums exactly as in the
// reference (src/timestep.f90:471 vs :496).
//
// Work split: blockIdx.x = tile of 128 targets, blockIdx.y = chunk of sources;
// per-chunk partial sums go to a buffer and are added in fixed chunk order,
// so results are deterministic.

#include "qv_internal.cuh"
#include "qv_tma.cuh"

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

#define DTILE 128

// ------------------------------------------------------------- compaction
__global__ void k_count_active(int n, const int *__restrict__ inf, int *blk_cnt) {
  __shared__ int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int a = (i < n && inf[i] != 0) ? 1 : 0;
  int w = __syncthreads_count(a);
  if (threadIdx.x == 0) blk_cnt[blockIdx.x] = w;
  (void)s;
}
__global__ void k_scan_small(int m, int *v, int *total) {
  // single block exclusive scan of m ints (m up to a few 100k)
  __shared__ int part[1024];
  int per = (m + blockDim.x - 1) / blockDim.x;
  int lo = threadIdx.x * per, hi = min(m, lo + per);
  int s = 0;
  for (int k = lo; k < hi; k++) s += v[k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < blockDim.x; off <<= 1) {
    int t = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += t;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int k = lo; k < hi; k++) {
    int t = v[k];
    v[k] = run;
    run += t;
  }
  if (threadIdx.x == blockDim.x - 1) *total = part[threadIdx.x];
}
__global__ void k_scatter_active(int n, const int *__restrict__ inf, const int *blk_off, int *act) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int a = (i < n && inf[i] != 0) ? 1 : 0;
  unsigned m = __ballot_sync(0xffffffffu, a);
  __shared__ int wsum[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wsum[wid] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int r = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) { int t = wsum[k]; wsum[k] = r; r += t; }
  }
  __syncthreads();
  if (a) act[blk_off[blockIdx.x] + wsum[wid] + __popc(m & ((1u << lane) - 1))] = i;
}

// Ordered compaction of the k in [0, n) with flag[k] != 0 into out, count to
// *total, for n <= QV_COMPACT1_MAX in one block: warp w takes a contiguous
// segment of the flags 32 at a time (coalesced loads, one ballot each, lane i
// keeps the ballots of iterations i and i + 32); a scan of the 32 warp counts
// gives each segment's base, and a second pass over the kept ballots writes
// the indices in order.
__global__ void __launch_bounds__(1024) k_compact1(int n, const int *__restrict__ flag, int *out,
                                                   int *total) {
  __shared__ int wbase[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int seg = ((n + 1023) / 1024) * 32;  // per warp, a multiple of 32
  const int iters = seg / 32;                // <= 64 for n <= QV_COMPACT1_MAX
  const int lo = w * seg;
  unsigned m0 = 0, m1 = 0;
  int cnt = 0;
#pragma unroll 8
  for (int it = 0; it < iters; it++) {
    const int k = lo + it * 32 + lane;
    const unsigned b = __ballot_sync(0xffffffffu, k < n && flag[k] != 0);
    if (lane == (it & 31)) {
      if (it < 32) m0 = b; else m1 = b;
    }
    cnt += __popc(b);
  }
  if (lane == 0) wbase[w] = cnt;
  __syncthreads();
  if (w == 0) {
    const int v = wbase[lane];
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    wbase[lane] = inc - v;
    if (lane == 31) *total = inc;
  }
  __syncthreads();
  int base = wbase[w];
  for (int it = 0; it < iters; it++) {
    const unsigned b = __shfl_sync(0xffffffffu, it < 32 ? m0 : m1, it & 31);
    if ((b >> lane) & 1u) out[base + __popc(b & ((1u << lane) - 1))] = lo + it * 32 + lane;
    base += __popc(b);
  }
}

// Stable compaction of the active slots (ascending index) into c->act.
int qv_compact_active(qv_ctx *c) {
  if (c->n <= QV_COMPACT1_MAX) {
    k_compact1<<<1, 1024, 0, c->stream>>>(c->n, c->infront, c->act, c->d_nact);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    QV_CUDA(c, cudaMemcpyAsync(&c->n_act, c->d_nact, sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream));
    QV_CUDA(c, cudaStreamSynchronize(c->stream));
    return QV_OK;
  }
  int nb = nblk(c->n, 256);
  int *tmp = c->blkcnt;
  k_count_active<<<nb, 256, 0, c->stream>>>(c->n, c->infront, tmp);
  k_scan_small<<<1, 1024, 0, c->stream>>>(nb, tmp, tmp + nb);
  k_scatter_active<<<nb, 256, 0, c->stream>>>(c->n, c->infront, tmp, c->act);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 3);
  QV_CUDA(c, cudaMemcpyAsync(&c->n_act, tmp + nb, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  QV_CUDA(c, cudaStreamSynchronize(c->stream));
  return QV_OK;
}

// The same compaction without waiting for it: the count goes to c->d_nact.
int qv_compact_active_async(qv_ctx *c) {
  if (c->n <= QV_COMPACT1_MAX) {
    k_compact1<<<1, 1024, 0, c->stream>>>(c->n, c->infront, c->act, c->d_nact);
    QV_LAUNCH_CHECK(c);
    QV_COUNT(c, 1);
    return QV_OK;
  }
  int nb = nblk(c->n, 256);
  int *tmp = c->blkcnt;
  k_count_active<<<nb, 256, 0, c->stream>>>(c->n, c->infront, tmp);
  k_scan_small<<<1, 1024, 0, c->stream>>>(nb, tmp, c->d_nact);
  k_scatter_active<<<nb, 256, 0, c->stream>>>(c->n, c->infront, tmp, c->act);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 3);
  return QV_OK;
}

// ------------------------------------------------------------ source packs
// FP64: x(3), s=gi-x(3), c=|gi-x|^2, slot (1-based) as double.
// FP32: x hi(3), x lo(3), gi hi(3), gi lo(3), slot bits, s = gi - x (3).
__global__ void k_pack_sources(int na, const int *__restrict__ act, const double *__restrict__ x,
                               const double *__restrict__ gi, double *s64, float *s32) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= na) return;
  int j = act[q];
  double X[3], G[3];
#pragma unroll
  for (int k = 0; k < 3; k++) { X[k] = x[3 * j + k]; G[k] = gi[3 * j + k]; }
  double *o = s64 + 8 * q;
  double e0 = G[0] - X[0], e1 = G[1] - X[1], e2 = G[2] - X[2];
  o[0] = X[0]; o[1] = X[1]; o[2] = X[2];
  o[3] = e0; o[4] = e1; o[5] = e2;
  o[6] = __dadd_rn(__dadd_rn(__dmul_rn(e0, e0), __dmul_rn(e1, e1)), __dmul_rn(e2, e2));
  o[7] = (double)(j + 1);
  float *f = s32 + 16 * q;
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

// ------------------------------------------------------------ pair terms
__device__ __forceinline__ void pair64(double dx, double dy, double dz, double sx, double sy,
                                       double sz, double c, double &ax, double &ay, double &az) {
  double a = dx * dx + dy * dy + dz * dz;
  double b = 2. * (dx * sx + dy * sy + dz * sz);
  double disc = 4. * a * c - b * b;
  if (disc == 0.) return;  // src/timestep.f90:476
  double fac = (2. * c + b) * rsqrt(a + b + c) - b * rsqrt(a);
  double sc = fac / disc;
  ax += (dy * sz - dz * sy) * sc;
  ay += (dz * sx - dx * sz) * sc;
  az += (dx * sy - dy * sx) * sc;
}

struct Kahan3 {
  float s[3], c[3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < 3; k++) s[k] = c[k] = 0.f;
  }
  __device__ __forceinline__ void add(float a0, float a1, float a2) {
    float a[3] = {a0, a1, a2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float y = __fsub_rn(a[k], c[k]);
      float t = __fadd_rn(s[k], y);
      c[k] = __fsub_rn(__fsub_rn(t, s[k]), y);
      s[k] = t;
    }
  }
  __device__ __forceinline__ double get(int k) const { return (double)s[k] - (double)c[k]; }
};


template <int BC>
__device__ __forceinline__ void img_mul(int m, int &a, int &b, int &c) {
  qv_img_shift(BC, m, &a, &b, &c);
}

__device__ __forceinline__ double shifted(double v, int a, double L) {
  return a == 0 ? v : (a > 0 ? v + L : v - L);
}

// ------------------------------------------------------------ TMA staging
// A source tile is a contiguous run of the pack (64 bytes per source in both
// packs), so one 1-D bulk copy of the TMA engine (cp.async.bulk into this
// block's own shared memory) moves it there and signals an mbarrier with its
// byte count.  Two buffers alternate: the copy of tile t+1 runs while tile t
// is summed.  The pack base is a device allocation (256-byte aligned) and
// every tile starts at a multiple of 64 bytes with a size that is a multiple
// of 64 bytes, which the copy's 16-byte rules ask for.  Each wait is bounded
// (QV_STAGE_WAIT_NS of wall time, and an iteration cap); a wait that runs out
// sets QV_STAT_STAGE in the status word and the block stops summing, so a
// copy that never lands ends the launch with an error, not a hang.

// Test hook (qv_test_stage_timeout): nonzero makes every tile acquire report
// a wait that ran out, without waiting, so that the error path -- drain the
// copies in flight, set QV_STAT_STAGE, return QV_ERR_CUDA -- runs while every
// copy still lands.  Process-wide; read when a direct-sum kernel is launched.
static int g_stage_fail = 0;

extern "C" int qv_test_stage_timeout(int enable) {
  g_stage_fail = enable ? 1 : 0;
  return QV_OK;
}

// Double-buffered tile pipeline over sources [j0, j1) of a pack with 64-byte
// rows.  begin() starts tile 0; acquire(t) starts tile t+1 and waits for tile
// t (every thread of the block calls it; the result is block-uniform);
// release() ends the use of the current tile; abort(t) drains the copies a
// failed acquire(t) may have left in flight and reports the failure.
struct TilePipe {
  const unsigned char *src;  // pack base
  int j0, j1, ntile;
  int fail;  // test hook: acquire() reports a wait that ran out without waiting
  // shared-memory addresses: stage k's buffer at buf + k * DTILE * 64, its
  // barrier at bar + 8 k
  unsigned buf, bar;

  __device__ __forceinline__ unsigned bar_of(int t) const { return bar + 8u * (t & 1); }
  __device__ __forceinline__ unsigned parity_of(int t) const { return (unsigned)(t >> 1) & 1u; }
  __device__ __forceinline__ void start(int t) const {
    const int t0 = j0 + t * DTILE, m = min(DTILE, j1 - t0);
    stage_copy(buf + (unsigned)(DTILE * 64) * (t & 1), src + (size_t)t0 * 64, (unsigned)m * 64u,
               bar_of(t));
  }
  __device__ __forceinline__ void begin() const {
    if (threadIdx.x == 0) {
      mbar_init(bar);
      mbar_init(bar + 8u);
      mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0 && ntile > 0) start(0);
  }
  __device__ __forceinline__ bool acquire(int t) const {
    // buffer (t+1)&1 was last read in iteration t-1, which release() closed
    if (threadIdx.x == 0 && t + 1 < ntile) start(t + 1);
    const bool got = fail ? false : mbar_wait(bar_of(t), parity_of(t));
    return __syncthreads_and(got) != 0;
  }
  __device__ __forceinline__ void release() const { __syncthreads(); }
  // kept out of line: inlined, its waits made the FP64 kernels spill
  __device__ __noinline__ void abort(int t, int *status) const {
    if (threadIdx.x == 0) {
      mbar_wait(bar_of(t), parity_of(t));
      if (t + 1 < ntile) mbar_wait(bar_of(t + 1), parity_of(t + 1));
      if (status) atomicOr(status, QV_STAT_STAGE);
    }
  }
};

// stages: 2 * DTILE * 64 contiguous bytes of shared memory; bars: 2 barriers
__device__ __forceinline__ TilePipe make_pipe(const void *src, int j0, int j1, const void *stages,
                                              const unsigned long long *bars, int fail) {
  TilePipe p;
  p.fail = fail;
  p.src = static_cast<const unsigned char *>(src);
  p.j0 = j0;
  p.j1 = j1;
  p.ntile = j1 > j0 ? (j1 - j0 + DTILE - 1) / DTILE : 0;
  p.buf = smem_u32(stages);
  p.bar = smem_u32(bars);
  return p;
}

// ------------------------------------------------------------ FP64 kernel
template <int BC>
__global__ void __launch_bounds__(DTILE) k_direct64(int na, const int *__restrict__ act,
                                                    const double *__restrict__ x,
                                                    const int *__restrict__ beh,
                                                    const double *__restrict__ src, int chunk_len,
                                                    double L, double *part, int *status,
                                                    int stage_fail) {
  constexpr int NIMG = BC == QV_BC_PERIODIC ? 26 : BC == QV_BC_OPENX ? 8 : BC == QV_BC_OPENXY ? 2 : 0;
  __shared__ __align__(128) double tiles[2][DTILE * 8];
  __shared__ __align__(8) unsigned long long bars[2];
  int q = blockIdx.x * DTILE + threadIdx.x;
  bool live = q < na;
  int i = live ? act[q] : 0;
  double xi0 = live ? x[3 * i] : 0., xi1 = live ? x[3 * i + 1] : 0., xi2 = live ? x[3 * i + 2] : 0.;
  int bi = live ? beh[i] : -1, ii = i + 1;
  double a0x = 0., a0y = 0., a0z = 0., a1x = 0., a1y = 0., a1z = 0.;
  int j0 = blockIdx.y * chunk_len, j1 = min(na, j0 + chunk_len);
  const TilePipe pipe = make_pipe(src, j0, j1, tiles, bars, stage_fail);
  pipe.begin();
  for (int t = 0; t < pipe.ntile; t++) {
    if (!pipe.acquire(t)) {
      pipe.abort(t, status);
      return;
    }
    const int m = min(DTILE, j1 - (j0 + t * DTILE));
    const double *tile = tiles[t & 1];
    for (int k = 0; k < m; k++) {
      const double *s = tile + 8 * k;
      int jj = (int)s[7];
      double dx = s[0] - xi0, dy = s[1] - xi1, dz = s[2] - xi2;
      if (jj != ii && jj != bi) pair64(dx, dy, dz, s[3], s[4], s[5], s[6], a0x, a0y, a0z);
      if (NIMG > 0 && jj != bi) {
#pragma unroll
        for (int im = 0; im < NIMG; im++) {
          int ma, mb, mc;
          img_mul<BC>(im, ma, mb, mc);
          pair64(shifted(dx, ma, L), shifted(dy, mb, L), shifted(dz, mc, L), s[3], s[4], s[5],
                 s[6], a1x, a1y, a1z);
        }
      }
    }
    pipe.release();
  }
  if (live) {
    double *o = part + ((size_t)blockIdx.y * na + q) * 6;
    o[0] = a0x; o[1] = a0y; o[2] = a0z; o[3] = a1x; o[4] = a1y; o[5] = a1z;
  }
}

// ------------------------------------------------------------ mixed kernel
// Every staged source is read from shared memory once and summed against the
// thread's NT targets in all images.  An image (a, b, c) shifts the source by
// (a L, b L, c L), so its R1 = x_j + shift - x_i and R2 = gi_j + shift - x_i
// take, per axis, one of at most three values: the target recentred per axis
// and shift (t = x_i - m L as a hi/lo float pair, made once per thread) gives
// those values with two FP32 adds each, and their squares, the products
// R1.R2 and the partial products of R1 x s are formed per axis too.  Each of
// the 27 pair terms then costs a few adds besides its two rsqrt and one
// reciprocal.  Per source, the 26 image terms are summed in plain FP32 and
// that sum, like the main-image term, goes into a Kahan-compensated sum.
//
// Pair term: the straight-segment form of qv_seg32 (src/tree.f90:380-390),
// (1/|R1| + 1/|R2|) q / (1 + cos) (R1 x s), q = 1/(|R1||R2|), cos = R1.R2 q,
// with 1 + cos taken from sin^2 / (1 - cos) when cos < 0.  Both cases are
// computed with selects and one division, without a branch: a branch per pair
// keeps the compiler from interleaving the 27 independent image pairs of a
// source, which costs more than the few extra multiplies.
__device__ __forceinline__ void seg_terms(float r1s, float r2s, float dd, float cx, float cy,
                                          float cz, float &ox, float &oy, float &oz) {
  const float ra = rsqrtf(r1s), rb = rsqrtf(r2s);
  const float q = ra * rb;
  const float cs = dd * q;
  const float f = (ra + rb) * q;
  // one division for both signs of cos: f / (1 + cos), or, when cos < 0,
  // f (1 - cos) / (|R1 x s|^2 q^2) (the same quotient, without cancellation)
  const bool pos = cs >= 0.f;
  const float s2 = fmaf(cx, cx, fmaf(cy, cy, cz * cz)) * (q * q);
  const float num = pos ? f : f * (1.f - cs);
  const float den = pos ? 1.f + cs : s2;
  const float g = den > 0.f ? __fdividef(num, den) : 0.f;
  ox = g * cx;
  oy = g * cy;
  oz = g * cz;
}

// seg_terms where cos is known to be positive: f / (1 + cos).
__device__ __forceinline__ void seg_terms_pos(float r1s, float r2s, float dd, float cx, float cy,
                                              float cz, float &ox, float &oy, float &oz) {
  const float ra = rsqrtf(r1s), rb = rsqrtf(r2s);
  const float q = ra * rb;
  const float cs = dd * q;
  const float f = (ra + rb) * q;
  const float g = __fdividef(f, 1.f + cs);
  ox = g * cx;
  oy = g * cy;
  oz = g * cz;
}

template <int BC, int NT>
__global__ void __launch_bounds__(DTILE) k_direct32(int na, const int *__restrict__ act,
                                                    const double *__restrict__ x,
                                                    const int *__restrict__ beh,
                                                    const float *__restrict__ src, int chunk_len,
                                                    double L, double *part, int *status,
                                                    int stage_fail) {
  // shifts per axis (the reference's image loops, src/timestep.f90:235-257)
  constexpr int PX = BC == QV_BC_PERIODIC ? 3 : 1;
  constexpr int PY = (BC == QV_BC_PERIODIC || BC == QV_BC_OPENX) ? 3 : 1;
  constexpr int PZ = BC == QV_BC_OPEN ? 1 : 3;
  __shared__ __align__(128) float4 tiles[2][DTILE * 4];
  __shared__ __align__(8) unsigned long long bars[2];
  // per target: slot, skip slots, the recentred target per axis and shift
  int qk[NT], bi[NT], ii[NT];
  float th[NT][3][3], tl[NT][3][3];
  Kahan3 k0[NT], k1[NT];
#pragma unroll
  for (int k = 0; k < NT; k++) {
    const int q = (blockIdx.x * NT + k) * DTILE + threadIdx.x;
    const bool live = q < na;
    const int i = live ? act[q] : 0;
    qk[k] = q;
    bi[k] = live ? beh[i] : -1;
    ii[k] = live ? i + 1 : -7;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double xc = live ? x[3 * i + c] : 0.;
      const int P = c == 0 ? PX : c == 1 ? PY : PZ;
#pragma unroll
      for (int m = 0; m < 3; m++) {
        const double t = P == 3 ? shifted(xc, 1 - m, L) : xc;  // x_i - (m-1) L
        th[k][c][m] = __double2float_rn(t);
        tl[k][c][m] = __double2float_rn(t - (double)th[k][c][m]);
      }
    }
    k0[k].zero();
    k1[k].zero();
  }
  const int j0 = blockIdx.y * chunk_len, j1 = min(na, j0 + chunk_len);
  const TilePipe pipe = make_pipe(src, j0, j1, tiles, bars, stage_fail);
  pipe.begin();
  for (int t = 0; t < pipe.ntile; t++) {
    if (!pipe.acquire(t)) {
      pipe.abort(t, status);
      return;
    }
    const int m = min(DTILE, j1 - (j0 + t * DTILE));
    const float4 *tile = tiles[t & 1];
#pragma unroll 1
    for (int e = 0; e < m; e++) {
      // A = (xh0 xh1 xh2 xl0) B = (xl1 xl2 gh0 gh1) C = (gh2 gl0 gl1 gl2) D = (slot s0 s1 s2)
      const float4 A = tile[4 * e], B = tile[4 * e + 1], Cc = tile[4 * e + 2], D = tile[4 * e + 3];
      const int jj = __float_as_int(D.x);
      const float sx = D.y, sy = D.z, sz = D.w;
#pragma unroll
      for (int k = 0; k < NT; k++) {
        const bool skip_src = jj == bi[k];  // src/timestep.f90:471, 496
        if (PX * PY * PZ == 1) {
          if (skip_src) continue;
          // open boundaries, the main image alone: the operations of the
          // batched direct items (qv_batch.cu), so that a batched system is
          // bitwise the same system run alone
          if (jj == ii[k]) continue;
          const float r1x = (A.x - th[k][0][1]) + (A.w - tl[k][0][1]);
          const float r1y = (A.y - th[k][1][1]) + (B.x - tl[k][1][1]);
          const float r1z = (A.z - th[k][2][1]) + (B.y - tl[k][2][1]);
          const float r2x = (B.z - th[k][0][1]) + (Cc.y - tl[k][0][1]);
          const float r2y = (B.w - th[k][1][1]) + (Cc.z - tl[k][1][1]);
          const float r2z = (Cc.x - th[k][2][1]) + (Cc.w - tl[k][2][1]);
          const float r1s = fmaf(r1x, r1x, fmaf(r1y, r1y, r1z * r1z));
          float ox, oy, oz;
          qv_seg32(r1x, r1y, r1z, r2x, r2y, r2z, sx, sy, sz, r1s, ox, oy, oz);
          k0[k].add(ox, oy, oz);
          continue;
        }
        float r1x[3], r2x[3], r1y[3], r2y[3], r1z[3], r2z[3];
#pragma unroll
        for (int s = 0; s < 3; s++) {
          r1x[s] = (A.x - th[k][0][s]) + (A.w - tl[k][0][s]);
          r2x[s] = (B.z - th[k][0][s]) + (Cc.y - tl[k][0][s]);
          r1y[s] = (A.y - th[k][1][s]) + (B.x - tl[k][1][s]);
          r2y[s] = (B.w - th[k][1][s]) + (Cc.z - tl[k][1][s]);
          r1z[s] = (A.z - th[k][2][s]) + (B.y - tl[k][2][s]);
          r2z[s] = (Cc.x - th[k][2][s]) + (Cc.w - tl[k][2][s]);
        }
        // per axis: |R1|^2, |R2|^2 and R1.R2 parts, and the parts of R1 x s
        float a1x[3], a2x[3], pdx[3], xsz[3], xsy[3];
        float a1y[3], a2y[3], pdy[3], ysz[3], ysx[3];
        float a1z[3], a2z[3], pdz[3], zsy[3], zsx[3];
#pragma unroll
        for (int s = 0; s < 3; s++) {
          a1x[s] = r1x[s] * r1x[s]; a2x[s] = r2x[s] * r2x[s]; pdx[s] = r1x[s] * r2x[s];
          xsz[s] = r1x[s] * sz; xsy[s] = r1x[s] * sy;
          a1y[s] = r1y[s] * r1y[s]; a2y[s] = r2y[s] * r2y[s]; pdy[s] = r1y[s] * r2y[s];
          ysz[s] = r1y[s] * sz; ysx[s] = r1y[s] * sx;
          a1z[s] = r1z[s] * r1z[s]; a2z[s] = r2z[s] * r2z[s]; pdz[s] = r1z[s] * r2z[s];
          zsy[s] = r1z[s] * sy; zsx[s] = r1z[s] * sx;
        }
        // When |R1| > |s| in every image, every image's cos is positive
        // (R1.R2 >= |R1| (|R1| - |s|)): the warp then takes the select-free
        // form of the term for this source, the pos case of seg_terms.  The
        // least |R1|^2 over the images is the sum over axes of each axis' least
        // square; the factor 1.0001 covers the rounding of both sides.
        float m1 = PX == 3 ? fminf(fminf(a1x[0], a1x[1]), a1x[2]) : a1x[1];
        m1 += PY == 3 ? fminf(fminf(a1y[0], a1y[1]), a1y[2]) : a1y[1];
        m1 += PZ == 3 ? fminf(fminf(a1z[0], a1z[1]), a1z[2]) : a1z[1];
        const float ss = fmaf(sx, sx, fmaf(sy, sy, sz * sz));
        const bool fast = __all_sync(0xffffffffu, skip_src || m1 > 1.0001f * ss);
        if (skip_src) continue;
        float ix = 0.f, iy = 0.f, iz = 0.f;
        auto images = [&](auto term) {
#pragma unroll
          for (int a = 0; a < PX; a++) {
            const int sa = PX == 3 ? a : 1;  // index of the x shift (1 = none)
#pragma unroll
            for (int b = 0; b < PY; b++) {
              const int sb = PY == 3 ? b : 1;
#pragma unroll
              for (int cc = 0; cc < PZ; cc++) {
                const int sc = PZ == 3 ? cc : 1;
                const bool main_img = sa == 1 && sb == 1 && sc == 1;
                if (main_img && jj == ii[k]) continue;
                float ox, oy, oz;
                term(a1x[sa] + a1y[sb] + a1z[sc], a2x[sa] + a2y[sb] + a2z[sc],
                     pdx[sa] + pdy[sb] + pdz[sc], ysz[sb] - zsy[sc], zsx[sc] - xsz[sa],
                     xsy[sa] - ysx[sb], ox, oy, oz);
                if (main_img) {
                  k0[k].add(ox, oy, oz);
                } else {
                  ix += ox;
                  iy += oy;
                  iz += oz;
                }
              }
            }
          }
        };
        if (fast) images(seg_terms_pos);
        else images(seg_terms);
        if (PX * PY * PZ > 1) k1[k].add(ix, iy, iz);
      }
    }
    pipe.release();
  }
#pragma unroll
  for (int k = 0; k < NT; k++) {
    if (qk[k] < na) {
      double *o = part + ((size_t)blockIdx.y * na + qk[k]) * 6;
      for (int c = 0; c < 3; c++) { o[c] = k0[k].get(c); o[3 + c] = k1[k].get(c); }
    }
  }
}

template <int BC>
static void launch_direct32(dim3 grid, cudaStream_t s, int na, const int *act, const double *x,
                            const int *beh, const float *src, int chunk_len, double L,
                            double *part, int *status, int stage_fail) {
  // one target per thread: two (NT = 2) took 17 % longer on the tangle
  k_direct32<BC, 1><<<grid, DTILE, 0, s>>>(na, act, x, beh, src, chunk_len, L, part, status,
                                           stage_fail);
}

// u_bs = s0 + s1, u = (u_li + s0) + s1, in fixed chunk order.
__global__ void k_direct_reduce(int na, int nchunk, const int *__restrict__ act,
                                const double *__restrict__ part, double scale,
                                const double *__restrict__ u_li, double *u, double *u_bs) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= na) return;
  int i = act[q];
  double s0[3] = {0., 0., 0.}, s1[3] = {0., 0., 0.};
  for (int k = 0; k < nchunk; k++) {
    const double *o = part + ((size_t)k * na + q) * 6;
    for (int c = 0; c < 3; c++) { s0[c] += o[c]; s1[c] += o[3 + c]; }
  }
  for (int c = 0; c < 3; c++) {
    double b0 = s0[c] * scale, b1 = s1[c] * scale;
    u_bs[3 * i + c] = b0 + b1;
    u[3 * i + c] = (u_li[3 * i + c] + b0) + b1;
  }
}

// Source packs of the compacted active list (c->act, c->n_act).
int qv_pack_sources64(qv_ctx *c) {
  if (c->n_act == 0) return QV_OK;
  k_pack_sources<<<nblk(c->n_act, 256), 256, 0, c->stream>>>(c->n_act, c->act, c->x, c->gi,
                                                             c->src64, c->src32);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  return QV_OK;
}

int qv_launch_direct(qv_ctx *c) {
  int na = c->n_act;
  if (na == 0) return QV_OK;
  int tb = nblk(c->n_act, 256);
  k_pack_sources<<<tb, 256, 0, c->stream>>>(na, c->act, c->x, c->gi, c->src64, c->src32);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 1);
  bool mixed = c->p.precision == QV_PREC_MIXED;
  int bx = nblk(na, DTILE);
  // enough chunks to fill ~4 blocks per SM, each chunk at least 4 tiles
  int want = (4 * c->sm_count + bx - 1) / bx;
  int maxch = max(1, na / (4 * DTILE));
  int nchunk = max(1, min(want, maxch));
  int chunk_len = ((nblk(na, nchunk) + DTILE - 1) / DTILE) * DTILE;
  nchunk = nblk(na, chunk_len);
  size_t need = sizeof(double) * 6 * (size_t)na * nchunk;
  if (need > c->dpart_bytes) {
    int rc = qv_grow(c, (void **)&c->dpart, need);
    if (rc) return rc;
    c->dpart_bytes = need;
  }
  double *part = c->dpart;
  dim3 grid(bx, nchunk);
  double L = c->p.box_size;
  switch (c->p.boundary) {
#define QV_DIRECT_CASE(BCV)                                                                   \
  case BCV:                                                                                   \
    if (mixed)                                                                                \
      launch_direct32<BCV>(grid, c->stream, na, c->act, c->x, c->behind, c->src32,           \
                                                     chunk_len, L, part, c->dstatus,          \
                                                     g_stage_fail);                           \
    else                                                                                      \
      k_direct64<BCV><<<grid, DTILE, 0, c->stream>>>(na, c->act, c->x, c->behind, c->src64,  \
                                                     chunk_len, L, part, c->dstatus,          \
                                                     g_stage_fail);                           \
    break;
    QV_DIRECT_CASE(QV_BC_OPEN)
    QV_DIRECT_CASE(QV_BC_PERIODIC)
    QV_DIRECT_CASE(QV_BC_OPENX)
    QV_DIRECT_CASE(QV_BC_OPENXY)
#undef QV_DIRECT_CASE
    default:
      return qv_fail(c, QV_ERR_UNSUPPORTED, "boundary %d not supported", c->p.boundary);
  }
  QV_LAUNCH_CHECK(c);
  double scale = mixed ? c->p.quant_circ / (4. * QV_PI) : c->p.quant_circ / (2. * QV_PI);
  k_direct_reduce<<<tb, 256, 0, c->stream>>>(na, nchunk, c->act, part, scale, c->u_li, c->u,
                                             c->u_bs);
  QV_LAUNCH_CHECK(c);
  QV_COUNT(c, 2);
  return QV_OK;
}

// ------------------------------------------------------ caller-owned scratch
// The same direct sum with every temporary placed in memory the caller
// provides (no allocation): act (n ints), blk (n/256+3 ints: block counts,
// the active count, a status word), src64 (8n doubles), src32 (16n floats),
// part (max_chunks * 6n doubles).  Writes only u_bs (the non-local velocity,
// f(:)%u_s_BS of src/timestep.f90:229-240) and returns after the sum is done.
__global__ void k_direct_reduce_bs(int na, int nchunk, const int *__restrict__ act,
                                   const double *__restrict__ part, double scale, double *u_bs) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= na) return;
  int i = act[q];
  double s0[3] = {0., 0., 0.}, s1[3] = {0., 0., 0.};
  for (int k = 0; k < nchunk; k++) {
    const double *o = part + ((size_t)k * na + q) * 6;
    for (int c = 0; c < 3; c++) { s0[c] += o[c]; s1[c] += o[3 + c]; }
  }
  for (int c = 0; c < 3; c++) u_bs[3 * i + c] = s0[c] * scale + s1[c] * scale;
}

int qv_direct_scratch(cudaStream_t s, const qv_params *p, int sm_count, int n, const double *x,
                      const int *inf, const int *beh, const double *gi, int *act, int *blk,
                      double *src64, float *src32, double *part, int max_chunks, double *u_bs) {
  int nb = nblk(n, 256);
  k_count_active<<<nb, 256, 0, s>>>(n, inf, blk);
  k_scan_small<<<1, 1024, 0, s>>>(nb, blk, blk + nb);
  k_scatter_active<<<nb, 256, 0, s>>>(n, inf, blk, act);
  int na = 0;
  if (cudaMemcpyAsync(&na, blk + nb, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return QV_ERR_CUDA;
  if (cudaMemsetAsync(u_bs, 0, sizeof(double) * 3 * (size_t)n, s) != cudaSuccess) return QV_ERR_CUDA;
  if (na == 0) return QV_OK;
  int tb = nblk(na, 256);
  bool mixed = p->precision == QV_PREC_MIXED;
  int *stat = blk + nb + 1;
  if (cudaMemsetAsync(stat, 0, sizeof(int), s) != cudaSuccess) return QV_ERR_CUDA;
  k_pack_sources<<<tb, 256, 0, s>>>(na, act, x, gi, src64, src32);
  int bx = nblk(na, DTILE);
  int want = (4 * sm_count + bx - 1) / bx;
  int maxch = max(1, na / (4 * DTILE));
  int nchunk = max(1, min(min(want, maxch), max_chunks));
  int chunk_len = ((nblk(na, nchunk) + DTILE - 1) / DTILE) * DTILE;
  nchunk = nblk(na, chunk_len);
  dim3 grid(bx, nchunk);
  double L = p->box_size;
  switch (p->boundary) {
#define QV_DIRECT_SCRATCH_CASE(BCV)                                                      \
  case BCV:                                                                              \
    if (mixed)                                                                           \
      launch_direct32<BCV>(grid, s, na, act, x, beh, src32, chunk_len, L, part,          \
                                             stat, g_stage_fail);                        \
    else                                                                                 \
      k_direct64<BCV><<<grid, DTILE, 0, s>>>(na, act, x, beh, src64, chunk_len, L, part,  \
                                             stat, g_stage_fail);                        \
    break;
    QV_DIRECT_SCRATCH_CASE(QV_BC_OPEN)
    QV_DIRECT_SCRATCH_CASE(QV_BC_PERIODIC)
    QV_DIRECT_SCRATCH_CASE(QV_BC_OPENX)
    QV_DIRECT_SCRATCH_CASE(QV_BC_OPENXY)
#undef QV_DIRECT_SCRATCH_CASE
    default:
      return QV_ERR_UNSUPPORTED;
  }
  double scale = mixed ? p->quant_circ / (4. * QV_PI) : p->quant_circ / (2. * QV_PI);
  k_direct_reduce_bs<<<tb, 256, 0, s>>>(na, nchunk, act, part, scale, u_bs);
  if (cudaGetLastError() != cudaSuccess) return QV_ERR_CUDA;
  int st = 0;
  if (cudaMemcpyAsync(&st, stat, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return QV_ERR_CUDA;
  return st ? QV_ERR_CUDA : QV_OK;
}
