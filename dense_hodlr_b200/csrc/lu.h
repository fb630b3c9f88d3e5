// Batched LU interfaces (lu.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hodlr_internal.h"

struct LeafLULaunch {
  const int* leaf_min;
  const int* leaf_size;
  const int64_t* lu_off;  // offset of each leaf's s x s LU in `lu`
  double* lu;
  int* perm;              // length N: row permutation of each leaf, local indices
  EntrySrc src;
  unsigned* err;
  // optional: the assembled leaf blocks before factoring, leaf (r0, s) at
  // a_copy[r0 + i + j * lda_copy] (i, j < s)
  double* a_copy;
  int64_t lda_copy;
};

struct LeafSolveLaunch {
  const int* leaf_min;
  const int* leaf_size;
  const int64_t* lu_off;
  const double* lu;
  const int* perm;
  double* X;     // N x ncols panel, column-major
  int64_t ldx;
  int ncols;
  unsigned* err;  // DEV_ERR_INDEX: a permutation entry outside its leaf
};

struct SchurNode {
  int kb, kt;       // ranks of the bottom / top off-diagonal blocks
  int coff;         // number of ancestor columns (Schur right-hand sides)
  // unknown order of the capacitance system: 0 [bottom rank; top rank], the
  // Schur matrix of recLU (src/HODLR_Matrix.cpp:663-670); 1 [top; bottom],
  // the perturbI matrix I + VT U of recSM (src/perturbI.cpp:28-38)
  int order;
  int64_t s_off;    // S (sd x sd) offset
  int64_t z_off;    // Z (sd x zcols) offset
  int64_t r_off;    // right-hand sides (sd x cols) offset for the solve
  int64_t p_off;    // pivots offset
};

struct SchurLaunch {
  const SchurNode* nodes;
  double* S;
  const double* Z;
  double* R;
  int* piv;
  unsigned* err;
};

int leaf_lu_launch(const LeafLULaunch& L, int nleaves, int smax, cudaStream_t s);
int leaf_solve_launch(const LeafSolveLaunch& L, int nleaves, int smax, cudaStream_t s);
// Capacitance matrices of at least this size are factored by the multi-CTA
// blocked LU (panel, swap + triangular solve, tiled trailing update per 32
// columns); smaller ones by one CTA each.
constexpr int SCHUR_BIG_SD = 384;
// The factorization's solves of the ancestor columns go blocked from this
// size (one 32-row diagonal block): the blocked solve reads each 32-row block
// of the LU once per 64 columns and keeps every SM busy, where one CTA per 16
// columns runs a latency-bound substitution per tile (measured on the 2D
// Matern workload at N = 262144: factorization 0.146 s with the blocked solve
// from 128 rows, 0.141 from 64, 0.128 from 32).
constexpr int SCHUR_BIG_SOLVE_SD = 32;
// sd: host array of the nodes' capacitance sizes (kb + kt), in node order.
int schur_factor_launch(const SchurLaunch& L, int nnodes, const int* sd, cudaStream_t s);
// Kernel launches schur_factor_launch makes for these sizes.
int schur_factor_launches(const int* sd, int nnodes);
int schur_solve_launch(const SchurLaunch& L, int nnodes, int ncols, int max_cols, int max_sd,
                       cudaStream_t s);
// The factorization's solves y = S^-1 Z of the `coff` ancestor columns of every
// node (R at r_off, ld sd); nodes with sd >= SCHUR_BIG_SOLVE_SD by the
// blocked solve.  sd: host array of the nodes' sizes.  *launches: kernels launched.
int schur_solve_factor_launch(const SchurLaunch& L, int nnodes, const int* sd, int coff,
                              cudaStream_t s, int* launches);
