// Grouped batched FP64 GEMM interface (gemm.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <vector>

// Arithmetic of the tensor-core path (umma_gemm.cu).
enum { HODLR_GEMM_FP64 = 0, HODLR_GEMM_TF32 = 1, HODLR_GEMM_BF16 = 2, HODLR_GEMM_TF32X3 = 3 };

// One product of a group.  TN: C (M x N) = A^T B with A K x M, B K x N.
// NN-sub: C (M x N) -= A B with A M x K, B K x N.  All column-major.
struct GemmProblem {
  const double* A;
  const double* B;
  double* C;
  int M, N, K;
  int lda, ldb, ldc;
  int splits;      // K splits (TN only), set by gemm_plan
  int kchunk;      // K per split
  int64_t ws_off;  // workspace offset of split partials
};

void gemm_plan(std::vector<GemmProblem>& probs, std::vector<int4>& tiles, int64_t& ws_elems,
               bool allow_split, int target_ctas);
int gemm_tn_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles, int nprob,
                   double* d_ws, bool any_split, cudaStream_t s);
int gemm_nn_sub_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles,
                       cudaStream_t s);
// C (M x N) = A B, A M x K, B K x N (no split along K)
int gemm_nn_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles, cudaStream_t s);
// C (M x N) += A B
int gemm_nn_add_launch(const GemmProblem* d_probs, const int4* d_tiles, int ntiles,
                       cudaStream_t s);

// tcgen05 forms of the same products (operands converted to prec in shared
// memory, FP32 accumulation in tensor memory, FP64 results).
void umma_plan(std::vector<GemmProblem>& probs, std::vector<int4>& tiles, int64_t& ws_elems,
               bool allow_split, int target_ctas);
int umma_tn_launch(int prec, const GemmProblem* d_probs, const int4* d_tiles, int ntiles, int nprob,
                   double* d_ws, bool any_split, unsigned* err, cudaStream_t s);
int umma_nn_sub_launch(int prec, const GemmProblem* d_probs, const int4* d_tiles, int ntiles,
                       unsigned* err, cudaStream_t s);
