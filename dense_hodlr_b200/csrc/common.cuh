// Shared device helpers for the HODLR kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <limits.h>

#include "kfun.h"
#include "hodlr_internal.h"

#define HODLR_INLINE __device__ __forceinline__

// Dynamic shared memory of a launch: opted in at its exact size before every
// launch.  The 48 KB a kernel gets without the opt-in counts its static
// shared memory too, so a dynamic size just under 48 KB can still need it.
inline cudaError_t smem_opt_in(const void* fn, size_t dyn_bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_bytes);
}

// Status codes of the C ABI (mirrored in include/hodlr_b200.h).
enum {
  HS_OK = 0,
  HS_ERR_ARG = 1,
  HS_ERR_CUDA = 2,
  HS_ERR_ALLOC = 3,
  HS_ERR_UNSUPPORTED = 4,
  HS_ERR_SINGULAR = 5,
  HS_ERR_STATE = 6,
  HS_ERR_NONFINITE = 7,
  HS_ERR_TIMEOUT = 8,
};

// Device error word bits (written by kernels, read by the host after a sync).
enum {
  DEV_ERR_TIMEOUT = 1,      // a bounded spin wait gave up
  DEV_ERR_NONFINITE = 2,    // a NaN/Inf entry or residual was produced
  DEV_ERR_SINGULAR = 4,     // an exact-zero LU pivot
  DEV_ERR_INDEX = 8,        // a pivot / permutation index outside its range (access skipped)
  // where DEV_ERR_INDEX was raised
  DEV_ERR_AT_LEAF_PERM = 16,     // leaf solve: row permutation
  DEV_ERR_AT_SOLVE_PIV = 32,     // capacitance solve (one CTA per column tile): interchanges
  DEV_ERR_AT_BLOCKED_PIV = 64,   // blocked ancestor-column solve: interchanges
  DEV_ERR_AT_LU_SWAP = 128,      // multi-CTA LU: interchanges outside the panel
};

// The entry source for blocks of the system that holds point i: in a forest
// of independent systems each has its own kernel; otherwise s itself.
HODLR_INLINE EntrySrc src_for(const EntrySrc& s, int i) {
  EntrySrc t = s;
  if (s.kps) t.kp = s.kps[__ldg(s.psys + i)];
  return t;
}

HODLR_INLINE double src_entry(const EntrySrc& s, int i, int j) {
  if (s.dense) return __ldg(s.A + (int64_t)j * s.ld + i);
  return hx_entry(s.kp, s.pts, s.ld, i, j);
}

// Entry K(i, j) when the coordinates of i are already in registers.
HODLR_INLINE double src_entry_xi(const EntrySrc& s, const double* xi, int i, int j) {
  if (s.dense) return __ldg(s.A + (int64_t)j * s.ld + i);
  if (i == j && s.kp.diag_replace) return s.kp.diag_value;
  double r2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < s.kp.dim) {
      double t = __dsub_rn(xi[d], __ldg(s.pts + d * s.ld + j));
      r2 = __dadd_rn(r2, __dmul_rn(t, t));
    }
  }
  double v = hx_kernel_r2(s.kp, r2);
  if (i == j) v = __dadd_rn(v, s.kp.shift);
  return v;
}

// Same, with the coordinates of column point j in registers (column pass).
HODLR_INLINE double src_entry_xj(const EntrySrc& s, const double* xj, int i, int j) {
  if (s.dense) return __ldg(s.A + (int64_t)j * s.ld + i);
  if (i == j && s.kp.diag_replace) return s.kp.diag_value;
  double r2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < s.kp.dim) {
      double t = __dsub_rn(__ldg(s.pts + d * s.ld + i), xj[d]);
      r2 = __dadd_rn(r2, __dmul_rn(t, t));
    }
  }
  double v = hx_kernel_r2(s.kp, r2);
  if (i == j) v = __dadd_rn(v, s.kp.shift);
  return v;
}

// (value, index) argmax with the lowest index winning ties: the result is
// the first maximum whatever the reduction order.
HODLR_INLINE void argmax_merge(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

HODLR_INLINE void warp_argmax(double& v, int& i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double v2 = __shfl_down_sync(0xffffffffu, v, o);
    int i2 = __shfl_down_sync(0xffffffffu, i, o);
    argmax_merge(v, i, v2, i2);
  }
}

HODLR_INLINE int warp_min_int(int x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_down_sync(0xffffffffu, x, o));
  return x;
}

HODLR_INLINE double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

HODLR_INLINE unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Iteration cap of every spin wait: ~2^26 polls with a 128 ns back-off is
// several seconds, far above any legitimate wait of these kernels.
#define HODLR_SPIN_LIMIT (1u << 26)
