// Grouped batched FP64 GEMMs for the Woodbury level updates.
//
// Replaces the per-node Eigen products of recLU_Factorize / recLU_Solve:
//   V^T * (K^-1 U) and V^T * X   (src/HODLR_Matrix.cpp:672-673, 679-680, 743-744)
//   X - (K^-1 U) * y             (src/HODLR_Matrix.cpp:686-687, 749-750)
// All nodes of one tree level are one launch.  A tile list maps every CTA to
// (problem, tile row, tile column, K split); TN products with a long
// reduction dimension (the top levels) are split along K into a workspace
// and summed in a fixed order by gemm_splitk_reduce, so results do not
// depend on scheduling.  The products run on the FP64 tensor-core
// instruction (mma.m8n8k4.f64).
#include "common.cuh"
#include "gemm.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// mode: 0 store C = A^T B (or split partial), 1 C -= A B, 2 store C = A B, 3 C += A B
//
// The products run on the FP64 tensor-core instruction mma.m8n8k4.f64: warp
// w (of 8) owns rows 32 (w % 2) .. +32 and columns 16 (w / 2) .. +16 of the
// 64 x 64 tile as 4 x 2 MMA tiles of 8 x 8; each k tile of 16 is four MMA
// steps of k = 4.  A and B tiles are staged in shared memory, the next one
// loaded into registers while the current one is consumed (two buffers, one
// barrier per k tile).  The accumulators then go through shared memory, so
// that C is read and written by thread (tx, ty) at rows tx + 16 i and columns
// ty + 16 j: a warp touches 16 consecutive rows of two columns (coalesced C
// traffic: the update of the ancestor columns is most of the bytes).
template <bool TRANS_A, int MODE>
__global__ void __launch_bounds__(NT) gemm_kernel(const GemmProblem* __restrict__ probs,
                                                  const int4* __restrict__ tiles,
                                                  double* __restrict__ ws) {
  constexpr int LDS = BM + 2;  // padded row of a staged k slice (BM == BN)
  constexpr int LDC = BM + 1;  // padded row of the staged result tile
  static_assert(BM == BN && 2 * 2 * BK * LDS >= BN * LDC, "result tile fits the operand buffers");
  __shared__ double smem[2 * 2 * BK * LDS];
  auto As = [&](int b, int k, int m) -> double& { return smem[(b * BK + k) * LDS + m]; };
  auto Bs = [&](int b, int k, int n) -> double& { return smem[((2 + b) * BK + k) * LDS + n]; };
  const int4 t = tiles[blockIdx.x];
  const GemmProblem P = probs[t.x];
  const int m0 = t.y * BM, n0 = t.z * BN;
  const int ks = t.w;
  const int kchunk = P.kchunk > 0 ? P.kchunk : P.K;
  const int kb = ks * kchunk, ke = min(P.K, kb + kchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  const int fr = lane >> 2, fk = lane & 3;  // fragment row / k of this lane
  constexpr int LA = (BK * BM) / NT, LB = (BK * BN) / NT;
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  double ra[LA], rb[LB];
  auto load = [&](int k0) {
#pragma unroll
    for (int r = 0; r < LA; ++r) {
      const int e = threadIdx.x + r * NT;
      int kk, mm;
      if (TRANS_A) {  // A is K x M (column-major): contiguous along k
        kk = e % BK;
        mm = e / BK;
      } else {  // A is M x K: contiguous along m
        mm = e % BM;
        kk = e / BM;
      }
      const int gk = k0 + kk, gm = m0 + mm;
      double v = 0.0;
      if (gk < ke && gm < P.M)
        v = TRANS_A ? __ldg(P.A + (int64_t)gm * P.lda + gk) : __ldg(P.A + (int64_t)gk * P.lda + gm);
      ra[r] = v;
    }
#pragma unroll
    for (int r = 0; r < LB; ++r) {  // B (K x N, column-major)
      const int e = threadIdx.x + r * NT;
      const int kk = e % BK, nn = e / BK;
      const int gk = k0 + kk, gn = n0 + nn;
      rb[r] = (gk < ke && gn < P.N) ? __ldg(P.B + (int64_t)gn * P.ldb + gk) : 0.0;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int r = 0; r < LA; ++r) {
      const int e = threadIdx.x + r * NT;
      if (TRANS_A)
        As(buf, e % BK, e / BK) = ra[r];
      else
        As(buf, e / BM, e % BM) = ra[r];
    }
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      const int e = threadIdx.x + r * NT;
      Bs(buf, e % BK, e / BK) = rb[r];
    }
  };

  // NN-subtract: the C tile is read before the k loop (it does not change
  // there), so its load overlaps the products instead of stalling the epilogue
  double cold[4][4];
  if (MODE == 1 || MODE == 3) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + ty + 16 * j;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int gm = m0 + tx + 16 * i;
        cold[i][j] = (gn < P.N && gm < P.M) ? P.C[(int64_t)gn * P.ldc + gm] : 0.0;
      }
    }
  }
  int buf = 0;
  if (kb < ke) {
    load(kb);
    store(0);
  }
  __syncthreads();
  for (int k0 = kb; k0 < ke; k0 += BK) {
    const bool more = k0 + BK < ke;
    if (more) load(k0 + BK);  // in flight while this tile is consumed
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double a[4], b[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As(buf, kk + fk, wm + 8 * i + fr);
#pragma unroll
      for (int j = 0; j < 2; ++j) b[j] = Bs(buf, kk + fk, wn + 8 * j + fr);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_884(acc[i][j], a[i], b[j]);
    }
    if (more) store(buf ^ 1);  // the other buffer: last read before the previous barrier
    __syncthreads();
    buf ^= 1;
  }
  // accumulators (lane: row fr, columns 2 fk, 2 fk + 1 of each 8 x 8 tile)
  // to the staged result tile, then out in the coalesced mapping
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        smem[(wn + 8 * j + 2 * fk + e) * LDC + wm + 8 * i + fr] = acc[i][j][e];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int gn = n0 + ty + 16 * j;
    if (gn >= P.N) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int gm = m0 + tx + 16 * i;
      if (gm >= P.M) continue;
      const double v = smem[(ty + 16 * j) * LDC + tx + 16 * i];
      if (MODE == 1) {
        P.C[(int64_t)gn * P.ldc + gm] = cold[i][j] - v;
      } else if (MODE == 3) {
        P.C[(int64_t)gn * P.ldc + gm] = cold[i][j] + v;
      } else if (MODE == 0 && P.splits > 1) {
        ws[P.ws_off + ((int64_t)ks * P.N + gn) * P.M + gm] = v;
      } else {
        P.C[(int64_t)gn * P.ldc + gm] = v;
      }
    }
  }
}

__global__ void splitk_reduce_kernel(const GemmProblem* __restrict__ probs, int nprob,
                                     const double* __restrict__ ws) {
  const GemmProblem P = probs[blockIdx.y];
  if (P.splits <= 1) return;
  const int64_t total = (int64_t)P.M * P.N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < P.splits; ++q) s += ws[P.ws_off + q * total + e];
    int gm = (int)(e % P.M), gn = (int)(e / P.M);
    P.C[(int64_t)gn * P.ldc + gm] = s;
  }
}

}  // namespace

int gemm_tn_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles, int nprob,
                   double* d_ws, bool any_split, cudaStream_t s) {
  if (ntiles == 0) return 0;
  gemm_kernel<true, 0><<<ntiles, NT, 0, s>>>(d_probs, d_tiles, d_ws);
  if (any_split) splitk_reduce_kernel<<<dim3(64, nprob), 256, 0, s>>>(d_probs, nprob, d_ws);
  return (int)cudaGetLastError();
}

int gemm_nn_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles, cudaStream_t s) {
  if (ntiles == 0) return 0;
  gemm_kernel<false, 2><<<ntiles, NT, 0, s>>>(d_probs, d_tiles, nullptr);
  return (int)cudaGetLastError();
}

int gemm_nn_sub_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles,
                       cudaStream_t s) {
  if (ntiles == 0) return 0;
  gemm_kernel<false, 1><<<ntiles, NT, 0, s>>>(d_probs, d_tiles, nullptr);
  return (int)cudaGetLastError();
}

int gemm_nn_add_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles,
                       cudaStream_t s) {
  if (ntiles == 0) return 0;
  gemm_kernel<false, 3><<<ntiles, NT, 0, s>>>(d_probs, d_tiles, nullptr);
  return (int)cudaGetLastError();
}

// Host-side planning: tile list and split-K workspace layout.
void gemm_plan(std::vector<GemmProblem>& probs, std::vector<int4>& tiles, int64_t& ws_elems,
               bool allow_split, int target_ctas) {
  tiles.clear();
  ws_elems = 0;
  int64_t mn_tiles = 0;
  for (auto& p : probs) mn_tiles += (int64_t)((p.M + BM - 1) / BM) * ((p.N + BN - 1) / BN);
  for (size_t q = 0; q < probs.size(); ++q) {
    GemmProblem& p = probs[q];
    if (p.M <= 0 || p.N <= 0 || p.K <= 0) {
      p.splits = 1;
      p.kchunk = 0;
      continue;
    }
    int tm = (p.M + BM - 1) / BM, tn = (p.N + BN - 1) / BN;
    int splits = 1;
    if (allow_split && mn_tiles < target_ctas) {
      int want = (int)((target_ctas + mn_tiles - 1) / mn_tiles);
      int maxs = std::max(1, p.K / 512);
      splits = std::max(1, std::min(want, maxs));
    }
    int kchunk = (p.K + splits - 1) / splits;
    kchunk = ((kchunk + BK - 1) / BK) * BK;
    splits = (p.K + kchunk - 1) / kchunk;
    p.splits = splits;
    p.kchunk = splits > 1 ? kchunk : 0;
    if (splits > 1) {
      p.ws_off = ws_elems;
      ws_elems += (int64_t)splits * p.M * p.N;
    }
    // grouped raster: column tiles in groups of GW, row tiles outer within a
    // group, so an A tile is reused from L2 by GW consecutive CTAs and a
    // group's B tiles by every row tile (each tile computes the same values
    // in any order)
    constexpr int GW = 8;
    for (int ks = 0; ks < splits; ++ks)
      for (int jg = 0; jg < tn; jg += GW)
        for (int i = 0; i < tm; ++i)
          for (int j = jg; j < std::min(tn, jg + GW); ++j) tiles.push_back(make_int4((int)q, i, j, ks));
  }
}
