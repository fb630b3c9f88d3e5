// Full-kernel FP64 product interface (kmatvec.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hodlr_internal.h"

struct KmatvecLaunch {
  EntrySrc src;
  const double* X;
  int64_t ldx;
  double* Y;
  int64_t ldy;
  double* ws;  // nsplit x nrhs x n partials (nsplit > 1)
  int n, nrhs;
  // forest form only: per-system flags; a flagged system's rows are skipped
  // (Y keeps what it held).  Null: every system.
  const unsigned char* skip = nullptr;
};

int kmatvec_splits(int n, int num_sms);
int kmatvec_launch(const KmatvecLaunch& L, int nsplit, cudaStream_t s);

// Symmetric form (closed-form kernels, nrhs <= 8): number of workspace
// slices (0 when it does not apply); L.ws must hold slices * nrhs * n.
int kmatvec_sym_slices(int n, int nrhs, bool dense);
int kmatvec_sym_launch(const KmatvecLaunch& L, int slices, cudaStream_t s);

// Forest of independent systems: block-diagonal product.  d_items holds
// (first row, system start, system end, system id) per 256-row tile, grouped
// by kernel family t in [type_off[t], type_off[t+1]), t < HX_FOREST_TYPES.
constexpr int HX_FOREST_TYPES = 5;
constexpr int HX_FOREST_TILE = 256;
int kmatvec_forest_launch(const KmatvecLaunch& L, const int4* d_items, const int* type_off,
                          cudaStream_t s);
