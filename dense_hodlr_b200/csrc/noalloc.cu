// Full-kernel product Y = K X that allocates no device memory.
//
// Some callers cannot call cudaMalloc when they need K x.  An application
// whose memory manager has reserved the device memory up front (a caching
// allocator that holds the GPU, a fixed budget set at start-up) would see a
// new allocation fail or push it over its budget.  A plugin hosted by such a
// framework is often not allowed to allocate behind the framework's back.
// And latency-bound code avoids cudaMalloc/cudaFree because they can
// synchronise the device.  A HODLR handle allocates on creation, so these
// callers cannot use hodlr_kernel_matvec_device.  This entry point takes the
// points, X and Y as caller-owned device buffers and keeps its only scratch
// -- the partial sums of the column splits of kmatvec.cu -- in the
// file-scope array below, which every GPU that loads the library holds until
// the process exits.
#include <mutex>

#include "../../include/hodlr_b200.h"
#include "common.cuh"
#include "kmatvec.h"

namespace {

// Shared by every call on a device; holds the last call's partial sums
// (HODLR_NOALLOC_SPLITS column splits at most, splits * n * nrhs doubles).
static __device__ __align__(256) double
    g_noalloc_scratch[HODLR_NOALLOC_SPLITS * HODLR_NOALLOC_MAX_ELEMS];

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device.  In host code
// `g_noalloc_scratch` names a host-side stand-in, so the address is fetched
// with cudaGetSymbolAddress, once per device, with that device current.
cudaError_t scratch_address(int dev, double** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int hodlr_kernel_matvec_noalloc(int n, int dim, const double* d_pts,
                                           const hodlr_kernel_desc* kernel, int nrhs,
                                           const double* d_x, int ldx, double* d_y, int ldy,
                                           void* stream) {
  if (n <= 0 || dim < 1 || dim > 3 || !d_pts || !kernel || nrhs < 1 || nrhs > 16 || !d_x ||
      !d_y || ldx < n || ldy < n)
    return HODLR_ERR_ARG;
  if (kernel->type < 0 || kernel->type > 4 || !(kernel->length_scale > 0)) return HODLR_ERR_ARG;
  if ((int64_t)n * nrhs > HODLR_NOALLOC_MAX_ELEMS) return HODLR_ERR_ARG;  // scratch limit
  // An error left pending by the caller's earlier CUDA work would be read
  // (and cleared) by the launch check below and reported as this call's:
  // leave it pending for its owner and launch nothing.
  if (cudaPeekAtLastError() != cudaSuccess) return HODLR_ERR_STATE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HODLR_ERR_CUDA;
  double* scratch = nullptr;
  if (scratch_address(dev, &scratch) != cudaSuccess) return HODLR_ERR_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return HODLR_ERR_CUDA;
  int nsplit = kmatvec_splits(n, sms);
  if (nsplit > HODLR_NOALLOC_SPLITS) nsplit = HODLR_NOALLOC_SPLITS;
  KmatvecLaunch L;
  L.src.pts = d_pts;
  L.src.A = nullptr;
  L.src.ld = n;
  L.src.kp = hx_make_kparams(kernel->type, dim, kernel->length_scale, kernel->diag_shift,
                             kernel->diag_replace, kernel->diag_value);
  L.src.dense = 0;
  L.src.kps = nullptr;
  L.src.psys = nullptr;
  L.X = d_x;
  L.ldx = ldx;
  L.Y = d_y;
  L.ldy = ldy;
  L.ws = scratch;  // every partial the reduction reads is written first: nothing to clear
  L.n = n;
  L.nrhs = nrhs;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (kmatvec_launch(L, nsplit, s) != 0) return HODLR_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? HODLR_OK : HODLR_ERR_CUDA;
}
