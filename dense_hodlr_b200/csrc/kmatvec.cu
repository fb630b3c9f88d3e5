// Full-kernel product Y = K X in FP64 with every entry generated on the fly.
// Replaces kernelMatrix::operator* (src/kernel.cpp:27-35), which the
// reference uses for the residual ||K x - b|| / ||b|| (src/HODLR_Matrix.cpp:
// 785-787), and supplies the residual of iterative refinement and GMRES.
//
// Compute-bound on the FP64 pipe: the distance, rsqrt / Tang exp from
// kfast.cuh (specialised per kernel family at compile time, so an entry costs
// ~25 FP64 instructions and no dispatch) and one FMA per right-hand side.  A
// CTA owns RPT * KT rows (RPT per thread, sharing every staged column value),
// NR accumulators per row in registers; column coordinates and X rows are
// staged through shared memory KT at a time.  Column ranges are split over
// gridDim.y when the row tiles alone cannot fill the GPU; the partial sums
// are added in a fixed order by kmatvec_reduce.
#include "common.cuh"
#include "kfast.cuh"
#include "kmatvec.h"

namespace {

constexpr int KT = 128;
constexpr int RPT = 2;  // rows per thread

__constant__ double c_tang[64] = HX_TANG_TABLE_INIT;

template <int NR, int KTYPE, int DIM>
__global__ void __launch_bounds__(KT) kmatvec_kernel(KmatvecLaunch L) {
  __shared__ double xs[DIM > 0 ? DIM : 1][KT];
  __shared__ double vs[NR][KT];
  __shared__ double tab[64];
  const int n = L.n;
  const int nsplit = gridDim.y;
  const int per = ((n + nsplit - 1) / nsplit + KT - 1) / KT * KT;
  const int jb = blockIdx.y * per, je = min(n, jb + per);
  if (threadIdx.x < 64) tab[threadIdx.x] = c_tang[threadIdx.x];
  int row[RPT];
  bool live[RPT];
  double xi[RPT][DIM > 0 ? DIM : 1];
  double acc[RPT][NR];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    row[q] = blockIdx.x * (KT * RPT) + q * KT + threadIdx.x;
    live[q] = row[q] < n;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[q][d] = live[q] ? L.src.pts[d * L.src.ld + row[q]] : 0.0;
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[q][c] = 0.0;
  }
  const double a = L.src.kp.a;
  for (int j0 = jb; j0 < je; j0 += KT) {
    const int jn = min(KT, je - j0);
    __syncthreads();
    if (threadIdx.x < jn) {
      const int j = j0 + threadIdx.x;
#pragma unroll
      for (int d = 0; d < DIM; ++d) xs[d][threadIdx.x] = L.src.pts[d * L.src.ld + j];
#pragma unroll
      for (int c = 0; c < NR; ++c)
        vs[c][threadIdx.x] = c < L.nrhs ? L.X[(int64_t)c * L.ldx + j] : 0.0;
    }
    __syncthreads();
#pragma unroll 2
    for (int t = 0; t < jn; ++t) {
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        double kij;
        if (DIM == 0) {  // dense input
          kij = live[q] ? L.src.A[(int64_t)(j0 + t) * L.src.ld + row[q]] : 0.0;
        } else {
          // off-diagonal formula everywhere; the diagonal is corrected below
          double r2 = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            double dd = xi[q][d] - xs[d][t];
            r2 = fma(dd, dd, r2);
          }
          kij = hx_kernel_r2_fast_t<KTYPE>(a, r2, tab);
        }
#pragma unroll
        for (int c = 0; c < NR; ++c) acc[q][c] = fma(kij, vs[c][t], acc[q][c]);
      }
    }
  }
  // K_ii = f(0) + shift (or the replaced value); f(0) = 1 for every family
  const hx_kparams kp = L.src.kp;
  const double dcorr = kp.diag_replace ? kp.diag_value - 1.0 : kp.shift;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    if (!live[q]) continue;
    if (DIM > 0 && row[q] >= jb && row[q] < je)
#pragma unroll
      for (int c = 0; c < NR; ++c)
        if (c < L.nrhs) acc[q][c] = fma(dcorr, L.X[(int64_t)c * L.ldx + row[q]], acc[q][c]);
#pragma unroll
    for (int c = 0; c < NR; ++c)
      if (c < L.nrhs) {
        if (nsplit == 1)
          L.Y[(int64_t)c * L.ldy + row[q]] = acc[q][c];
        else
          L.ws[((int64_t)blockIdx.y * L.nrhs + c) * n + row[q]] = acc[q][c];
      }
  }
}

__global__ void kmatvec_reduce(KmatvecLaunch L, int nsplit) {
  const int64_t total = (int64_t)L.n * L.nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nsplit; ++q) s += L.ws[q * total + e];
    int i = (int)(e % L.n), c = (int)(e / L.n);
    L.Y[(int64_t)c * L.ldy + i] = s;
  }
}

template <int NR, int KTYPE>
void launch_dim(const KmatvecLaunch& L, dim3 grid, cudaStream_t s) {
  if (L.src.dense)
    kmatvec_kernel<NR, KTYPE, 0><<<grid, KT, 0, s>>>(L);
  else if (L.src.kp.dim == 1)
    kmatvec_kernel<NR, KTYPE, 1><<<grid, KT, 0, s>>>(L);
  else if (L.src.kp.dim == 2)
    kmatvec_kernel<NR, KTYPE, 2><<<grid, KT, 0, s>>>(L);
  else
    kmatvec_kernel<NR, KTYPE, 3><<<grid, KT, 0, s>>>(L);
}

template <int NR>
void launch_type(const KmatvecLaunch& L, dim3 grid, cudaStream_t s) {
  if (L.src.dense) {
    kmatvec_kernel<NR, 0, 0><<<grid, KT, 0, s>>>(L);
    return;
  }
  switch (L.src.kp.type) {
    case HX_KERNEL_GAUSSIAN: launch_dim<NR, HX_KERNEL_GAUSSIAN>(L, grid, s); break;
    case HX_KERNEL_MATERN32: launch_dim<NR, HX_KERNEL_MATERN32>(L, grid, s); break;
    case HX_KERNEL_INV_MULTIQUADRIC: launch_dim<NR, HX_KERNEL_INV_MULTIQUADRIC>(L, grid, s); break;
    case HX_KERNEL_QUADRATIC: launch_dim<NR, HX_KERNEL_QUADRATIC>(L, grid, s); break;
    default: launch_dim<NR, HX_KERNEL_EXPONENTIAL>(L, grid, s); break;
  }
}

}  // namespace

int kmatvec_splits(int n, int num_sms) {
  int tiles = (n + KT * RPT - 1) / (KT * RPT);
  int want = 8 * num_sms;
  int sp = (want + tiles - 1) / tiles;
  int maxsp = (n + 2047) / 2048;
  if (sp > maxsp) sp = maxsp;
  return sp < 1 ? 1 : sp;
}

int kmatvec_launch(const KmatvecLaunch& L, int nsplit, cudaStream_t s) {
  dim3 grid((L.n + KT * RPT - 1) / (KT * RPT), nsplit);
  if (L.nrhs <= 1)
    launch_type<1>(L, grid, s);
  else if (L.nrhs <= 4)
    launch_type<4>(L, grid, s);
  else if (L.nrhs <= 8)
    launch_type<8>(L, grid, s);
  else if (L.nrhs <= 16)
    launch_type<16>(L, grid, s);
  else
    return (int)cudaErrorInvalidValue;
  if (nsplit > 1) kmatvec_reduce<<<1024, 256, 0, s>>>(L, nsplit);
  return (int)cudaGetLastError();
}
