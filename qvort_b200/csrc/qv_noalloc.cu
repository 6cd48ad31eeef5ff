// qv_noalloc.cu -- the direct Biot-Savart sum for callers that cannot
// allocate device memory.
//
// Some hosts of this library must not call cudaMalloc/cudaFree on their hot
// path: a Fortran or C driver that reserves its whole device memory budget up
// front and hands out fixed buffers (so that a long run never fails halfway
// on an allocation), a code embedded in another framework that owns the
// device allocator, or a time-critical loop that cannot afford the implicit
// device synchronisation of cudaMalloc/cudaFree.  qv_velocity_direct_noalloc
// serves them: the caller passes device inputs and the output, and every
// temporary lives in the file-scope array below, sized for
// QV_NOALLOC_MAX_POINTS slots.  Each GPU that loads the library holds that
// array (about 9 MB) until the process exits.
//
// Sharing: every call uses the same array and the array keeps the last call's
// contents.  Nothing in it has to start at zero (each call overwrites all it
// reads), but two calls that overlap on the GPU (different streams, or
// different host threads on the same device) race on it; serialise them.
#include <mutex>

#include "qv_internal.cuh"

namespace {

constexpr size_t kAlign = 256;
constexpr size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

constexpr int kMaxN = QV_NOALLOC_MAX_POINTS;
constexpr int kMaxChunks = 8;
// layout of the scratch array (byte offsets, each 256-aligned)
constexpr size_t kOffGi = 0;
constexpr size_t kOffAct = kOffGi + up(sizeof(double) * 3 * kMaxN);
constexpr size_t kOffBlk = kOffAct + up(sizeof(int) * kMaxN);
constexpr size_t kOffSrc64 = kOffBlk + up(sizeof(int) * (kMaxN / 256 + 3));
constexpr size_t kOffSrc32 = kOffSrc64 + up(sizeof(double) * 8 * kMaxN);
constexpr size_t kOffPart = kOffSrc32 + up(sizeof(float) * 16 * kMaxN);
constexpr size_t kBytes = kOffPart + up(sizeof(double) * 6 * (size_t)kMaxChunks * kMaxN);

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kBytes];

int qv_direct_scratch(cudaStream_t s, const qv_params *p, int sm_count, int n, const double *x,
                      const int *inf, const int *beh, const double *gi, int *act, int *blk,
                      double *src64, float *src32, double *part, int max_chunks, double *u_bs);

// ghosti only (the direct sum needs the +1 neighbour), get_ghost_p
// (src/periodic.f90:23-165) restricted to ginfront.
__global__ void k_noalloc_ghosti(int n, const double *__restrict__ x, const int *__restrict__ inf,
                                 double *gi, int lo_axis, double L) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int a = inf[i];
  if (a == 0) return;
  double h = L / 2.;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double xi = x[3 * i + c], g = x[3 * (a - 1) + c];
    if (c >= lo_axis) {
      if ((xi - g) > h)
        g = g + L;
      else if ((xi - g) < (-h))
        g = g - L;
    }
    gi[3 * i + c] = g;
  }
}

// Address of this device's scratch array.  cudaGetSymbolAddress runs once per
// device, with that device current, on the first call made there.
static int scratch_for_current_device(unsigned char **base) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return QV_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return QV_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return QV_ERR_CUDA;
    }
    g_scratch_addr[dev] = ptr;
  }
  *base = static_cast<unsigned char *>(g_scratch_addr[dev]);
  return QV_OK;
}

extern "C" int qv_velocity_direct_noalloc(const qv_params *p, int n, const double *x,
                                          const int *infront, const int *behind, double *u_bs,
                                          void *stream) {
  if (!p || n < 0 || (n > 0 && (!x || !infront || !behind || !u_bs))) return QV_ERR_ARG;
  if (n > QV_NOALLOC_MAX_POINTS) return QV_ERR_NOALLOC_LIMIT;
  if (p->boundary < QV_BC_OPEN || p->boundary > QV_BC_OPENXY) return QV_ERR_UNSUPPORTED;
  if (p->precision != QV_PREC_FP64 && p->precision != QV_PREC_MIXED) return QV_ERR_ARG;
  if (p->boundary != QV_BC_OPEN && !(p->box_size > 0)) return QV_ERR_ARG;
  if (n == 0) return QV_OK;
  unsigned char *base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double *gi = reinterpret_cast<double *>(base + kOffGi);
  int *act = reinterpret_cast<int *>(base + kOffAct);
  int *blk = reinterpret_cast<int *>(base + kOffBlk);
  double *src64 = reinterpret_cast<double *>(base + kOffSrc64);
  float *src32 = reinterpret_cast<float *>(base + kOffSrc32);
  double *part = reinterpret_cast<double *>(base + kOffPart);
  int lo = p->boundary == QV_BC_PERIODIC ? 0 : p->boundary == QV_BC_OPENX ? 1
         : p->boundary == QV_BC_OPENXY ? 2 : 3;
  k_noalloc_ghosti<<<(n + 255) / 256, 256, 0, s>>>(n, x, infront, gi, lo, p->box_size);
  if (cudaGetLastError() != cudaSuccess) return QV_ERR_CUDA;
  rc = qv_direct_scratch(s, p, sms, n, x, infront, behind, gi, act, blk, src64, src32, part,
                         kMaxChunks, u_bs);
  if (rc) return rc;
  return cudaStreamSynchronize(s) == cudaSuccess ? QV_OK : QV_ERR_CUDA;
}
