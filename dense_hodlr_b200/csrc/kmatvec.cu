// Full-kernel product Y = K X in FP64 with every entry generated on the fly.
// Replaces kernelMatrix::operator* (src/kernel.cpp:27-35), which the
// reference uses for the residual ||K x - b|| / ||b|| (src/HODLR_Matrix.cpp:
// 785-787).  Entries come from kfun.h, so they are the exact values ACA saw.
//
// A CTA owns 128 rows (one per thread, NRHS accumulators in registers) and a
// range of columns; column coordinates and X rows are staged through shared
// memory 128 at a time.  Column ranges are split over gridDim.y when the row
// tiles alone cannot fill the GPU; the partial sums are added in a fixed
// order by kmatvec_reduce.
#include "common.cuh"
#include "kmatvec.h"

namespace {

constexpr int KT = 128;

template <int NR>
__global__ void __launch_bounds__(KT) kmatvec_kernel(KmatvecLaunch L) {
  __shared__ double xs[3][KT];
  __shared__ double vs[NR][KT];
  const int i = blockIdx.x * KT + threadIdx.x;
  const int n = L.n;
  const int nsplit = gridDim.y;
  const int per = ((n + nsplit - 1) / nsplit + KT - 1) / KT * KT;
  const int jb = blockIdx.y * per, je = min(n, jb + per);
  const bool live = i < n;
  const int dim = L.src.kp.dim;
  double xi[3] = {0.0, 0.0, 0.0};
  if (live && !L.src.dense)
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < dim) xi[d] = L.src.pts[d * L.src.ld + i];
  double acc[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) acc[c] = 0.0;
  for (int j0 = jb; j0 < je; j0 += KT) {
    const int jn = min(KT, je - j0);
    __syncthreads();
    if (threadIdx.x < jn) {
      const int j = j0 + threadIdx.x;
      if (!L.src.dense)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (d < dim) xs[d][threadIdx.x] = L.src.pts[d * L.src.ld + j];
#pragma unroll
      for (int c = 0; c < NR; ++c)
        vs[c][threadIdx.x] = c < L.nrhs ? L.X[(int64_t)c * L.ldx + j] : 0.0;
    }
    __syncthreads();
    if (live) {
      for (int t = 0; t < jn; ++t) {
        const int j = j0 + t;
        double kij;
        if (L.src.dense) {
          kij = L.src.A[(int64_t)j * L.src.ld + i];
        } else if (i == j && L.src.kp.diag_replace) {
          kij = L.src.kp.diag_value;
        } else {
          double r2 = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d)
            if (d < dim) {
              double q = __dsub_rn(xi[d], xs[d][t]);
              r2 = __dadd_rn(r2, __dmul_rn(q, q));
            }
          kij = hx_kernel_r2(L.src.kp, r2);
          if (i == j) kij = __dadd_rn(kij, L.src.kp.shift);
        }
#pragma unroll
        for (int c = 0; c < NR; ++c) acc[c] = fma(kij, vs[c][t], acc[c]);
      }
    }
  }
  if (live)
#pragma unroll
    for (int c = 0; c < NR; ++c)
      if (c < L.nrhs) {
        if (nsplit == 1)
          L.Y[(int64_t)c * L.ldy + i] = acc[c];
        else
          L.ws[((int64_t)blockIdx.y * L.nrhs + c) * n + i] = acc[c];
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

}  // namespace

int kmatvec_splits(int n, int num_sms) {
  int tiles = (n + KT - 1) / KT;
  int want = 4 * num_sms;
  int sp = (want + tiles - 1) / tiles;
  int maxsp = (n + 1023) / 1024;
  if (sp > maxsp) sp = maxsp;
  return sp < 1 ? 1 : sp;
}

int kmatvec_launch(const KmatvecLaunch& L, int nsplit, cudaStream_t s) {
  dim3 grid((L.n + KT - 1) / KT, nsplit);
  if (L.nrhs <= 1)
    kmatvec_kernel<1><<<grid, KT, 0, s>>>(L);
  else if (L.nrhs <= 4)
    kmatvec_kernel<4><<<grid, KT, 0, s>>>(L);
  else if (L.nrhs <= 8)
    kmatvec_kernel<8><<<grid, KT, 0, s>>>(L);
  else if (L.nrhs <= 16)
    kmatvec_kernel<16><<<grid, KT, 0, s>>>(L);
  else
    return (int)cudaErrorInvalidValue;
  if (nsplit > 1) kmatvec_reduce<<<1024, 256, 0, s>>>(L, nsplit);
  return (int)cudaGetLastError();
}
