// Batched LU kernels of the recLU factorization and solve.
//
//  leaf_lu_kernel     assembles every leaf block from the kernel (or the dense
//                     input) and factors it with row partial pivoting, one CTA
//                     per leaf, all in shared memory.  Replaces the leaf path
//                     of storeLRinTree (src/HODLR_Matrix.cpp:303-312) and
//                     PartialPivLU(leafMatrix) (src/HODLR_Matrix.cpp:625).
//  leaf_solve_kernel  applies the leaf LU to a tile of a wide panel: the
//                     leafLU.solve of recLU_Factorize / recLU_Solve
//                     (src/HODLR_Matrix.cpp:626,703).
//  schur_form_kernel  builds S = [[I, V_b^T K_t^-1 U_t], [V_t^T K_b^-1 U_b, I]]
//                     (src/HODLR_Matrix.cpp:663-673) from the level product Z.
//  dense_lu_kernel    factors each node's S in place (src/HODLR_Matrix.cpp:675).
//  dense_lu_solve_kernel  y = S^-1 rhs (src/HODLR_Matrix.cpp:682,746).
// Pivoting takes the first maximum |a| of the column, as PartialPivLU does.
#include "common.cuh"
#include "lu.h"

namespace {

constexpr int LNT = 256;

// ------------------------------------------------------------- leaf LU
__global__ void __launch_bounds__(LNT) leaf_lu_kernel(LeafLULaunch L) {
  extern __shared__ double a[];  // s x s, leading dimension s | 1
  __shared__ double red_v[LNT / 32];
  __shared__ int red_i[LNT / 32];
  __shared__ int s_piv;
  const int leaf = blockIdx.x;
  const int r0 = L.leaf_min[leaf], s = L.leaf_size[leaf];
  const int lda = s | 1;
  const int tid = threadIdx.x;
  int* perm = L.perm + r0;  // final row permutation, local indices
  // assemble
  for (int e = tid; e < s * s; e += LNT) {
    int i = e % s, j = e / s;
    a[j * lda + i] = src_entry(L.src, r0 + i, r0 + j);
  }
  for (int i = tid; i < s; i += LNT) perm[i] = i;
  __syncthreads();
  bool singular = false, nonfinite = false;
  for (int p = 0; p < s; ++p) {
    // pivot search in column p, rows p..s-1, first maximum
    if (tid < 32) {
      double bv = -1.0;
      int bi = INT_MAX;
      for (int i = p + tid; i < s; i += 32) {
        double v = fabs(a[p * lda + i]);
        if (v > bv) {
          bv = v;
          bi = i;
        }
      }
      warp_argmax(bv, bi);
      if (tid == 0) s_piv = (bi == INT_MAX) ? p : bi;
    }
    __syncthreads();
    const int q = s_piv;
    if (q != p) {
      for (int j = tid; j < s; j += LNT) {
        double t = a[j * lda + p];
        a[j * lda + p] = a[j * lda + q];
        a[j * lda + q] = t;
      }
      if (tid == 0) {
        int t = perm[p];
        perm[p] = perm[q];
        perm[q] = t;
      }
    }
    __syncthreads();
    const double d = a[p * lda + p];
    if (d == 0.0) {
      singular = true;
      __syncthreads();
      continue;
    }
    if (!isfinite(d)) nonfinite = true;
    for (int i = p + 1 + tid; i < s; i += LNT) a[p * lda + i] = a[p * lda + i] / d;
    __syncthreads();
    // rank-1 update of the trailing block
    const int rem = s - p - 1;
    for (int e = tid; e < rem * rem; e += LNT) {
      int i = p + 1 + e % rem, j = p + 1 + e / rem;
      a[j * lda + i] = fma(-a[p * lda + i], a[j * lda + p], a[j * lda + i]);
    }
    __syncthreads();
  }
  double* out = L.lu + L.lu_off[leaf];
  for (int e = tid; e < s * s; e += LNT) {
    int i = e % s, j = e / s;
    out[(int64_t)j * s + i] = a[j * lda + i];
  }
  if (tid == 0) {
    if (singular) atomicOr(L.err, DEV_ERR_SINGULAR);
    if (nonfinite) atomicOr(L.err, DEV_ERR_NONFINITE);
  }
}

// ---------------------------------------------------------- leaf solve
// X[leaf rows, c0 : c0+TC] <- U^-1 L^-1 P X.  One CTA per (leaf, column tile).
template <int TC>
__global__ void __launch_bounds__(LNT) leaf_solve_kernel(LeafSolveLaunch L) {
  extern __shared__ double sm[];
  const int leaf = blockIdx.y;
  const int c0 = blockIdx.x * TC;
  const int ncol = min(TC, L.ncols - c0);
  if (ncol <= 0) return;
  const int r0 = L.leaf_min[leaf], s = L.leaf_size[leaf];
  const int lda = s | 1;
  double* lu = sm;                    // s x s
  double* x = sm + (size_t)s * lda;   // s x TC, x[c * (s|1) + i]
  const int ldx = s | 1;
  const int tid = threadIdx.x;
  const double* g = L.lu + L.lu_off[leaf];
  for (int e = tid; e < s * s; e += LNT) {
    int i = e % s, j = e / s;
    lu[j * lda + i] = g[(int64_t)j * s + i];
  }
  const int* perm = L.perm + r0;
  for (int e = tid; e < s * ncol; e += LNT) {
    int i = e % s, c = e / s;
    x[c * ldx + i] = L.X[(int64_t)(c0 + c) * L.ldx + r0 + perm[i]];
  }
  __syncthreads();
  // thread layout: column c = tid % TC, row group rg = tid / TC
  constexpr int RG = LNT / TC;
  const int c = tid % TC, rg = tid / TC;
  const bool active = c < ncol;
  // forward: unit lower
  for (int p = 0; p < s - 1; ++p) {
    if (active) {
      const double xp = x[c * ldx + p];
      for (int i = p + 1 + rg; i < s; i += RG) x[c * ldx + i] = fma(-lu[p * lda + i], xp, x[c * ldx + i]);
    }
    __syncthreads();
  }
  // backward: upper
  for (int p = s - 1; p >= 0; --p) {
    if (active && rg == 0) x[c * ldx + p] = x[c * ldx + p] / lu[p * lda + p];
    __syncthreads();
    if (active) {
      const double xp = x[c * ldx + p];
      for (int i = rg; i < p; i += RG) x[c * ldx + i] = fma(-lu[p * lda + i], xp, x[c * ldx + i]);
    }
    __syncthreads();
  }
  for (int e = tid; e < s * ncol; e += LNT) {
    int i = e % s, cc = e / s;
    L.X[(int64_t)(c0 + cc) * L.ldx + r0 + i] = x[cc * ldx + i];
  }
}

// ---------------------------------------------------------- Schur form
// S[node] (sd x sd, sd = kb + kt): identity blocks on the diagonal, the level
// products of Z on the off-diagonal blocks.
__global__ void schur_form_kernel(SchurLaunch L) {
  const int node = blockIdx.x;
  const SchurNode N = L.nodes[node];
  const int sd = N.kb + N.kt;
  double* S = L.S + N.s_off;
  const double* Z = L.Z + N.z_off;  // sd x zcols, ld sd
  for (int64_t e = threadIdx.x; e < (int64_t)sd * sd; e += blockDim.x) {
    int i = (int)(e % sd), j = (int)(e / sd);
    double v;
    if (i < N.kb && j < N.kb)
      v = (i == j) ? 1.0 : 0.0;
    else if (i >= N.kb && j >= N.kb)
      v = (i == j) ? 1.0 : 0.0;
    else if (i < N.kb)  // top-right: V_b^T K_t^-1 U_t = Z rows [0,kb), cols coff + (j - kb)
      v = Z[(int64_t)(N.coff + j - N.kb) * sd + i];
    else  // bottom-left: V_t^T K_b^-1 U_b = Z rows [kb, sd), cols coff + j
      v = Z[(int64_t)(N.coff + j) * sd + i];
    S[(int64_t)j * sd + i] = v;
  }
}

// ------------------------------------------------------ dense batched LU
// Right-looking LU of S in global memory (it stays in L2 for these sizes).
__global__ void __launch_bounds__(LNT) dense_lu_kernel(SchurLaunch L) {
  __shared__ int s_piv;
  const int node = blockIdx.x;
  const SchurNode N = L.nodes[node];
  const int n = N.kb + N.kt;
  double* a = L.S + N.s_off;
  int* piv = L.piv + N.p_off;
  const int tid = threadIdx.x;
  bool singular = false;
  for (int p = 0; p < n; ++p) {
    if (tid < 32) {
      double bv = -1.0;
      int bi = INT_MAX;
      for (int i = p + tid; i < n; i += 32) {
        double v = fabs(a[(int64_t)p * n + i]);
        if (v > bv) {
          bv = v;
          bi = i;
        }
      }
      warp_argmax(bv, bi);
      if (tid == 0) {
        s_piv = (bi == INT_MAX) ? p : bi;
        piv[p] = s_piv;
      }
    }
    __syncthreads();
    const int q = s_piv;
    if (q != p)
      for (int j = tid; j < n; j += LNT) {
        double t = a[(int64_t)j * n + p];
        a[(int64_t)j * n + p] = a[(int64_t)j * n + q];
        a[(int64_t)j * n + q] = t;
      }
    __syncthreads();
    const double d = a[(int64_t)p * n + p];
    if (d == 0.0) {
      singular = true;
      continue;
    }
    for (int i = p + 1 + tid; i < n; i += LNT) a[(int64_t)p * n + i] /= d;
    __syncthreads();
    const int rem = n - p - 1;
    // column-by-column trailing update: warp w updates columns w, w+8, ...
    const int w = tid >> 5, lane = tid & 31;
    for (int jj = w; jj < rem; jj += LNT / 32) {
      const int j = p + 1 + jj;
      const double u = a[(int64_t)j * n + p];
      if (u != 0.0)
        for (int i = p + 1 + lane; i < n; i += 32)
          a[(int64_t)j * n + i] = fma(-a[(int64_t)p * n + i], u, a[(int64_t)j * n + i]);
    }
    __syncthreads();
  }
  if (tid == 0 && singular) atomicOr(L.err, DEV_ERR_SINGULAR);
}

// y = S^-1 rhs for `ncols` right-hand sides stored in R (ld sd) at r_off;
// one CTA per (node, column chunk), a warp per column.
__global__ void __launch_bounds__(LNT) dense_lu_solve_kernel(SchurLaunch L, int ncols) {
  const int node = blockIdx.y;
  const SchurNode N = L.nodes[node];
  const int n = N.kb + N.kt;
  const double* a = L.S + N.s_off;
  const int* piv = L.piv + N.p_off;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cols = ncols < 0 ? N.coff : ncols;
  for (int col = blockIdx.x * (LNT / 32) + w; col < cols; col += gridDim.x * (LNT / 32)) {
    double* x = L.R + N.r_off + (int64_t)col * n;
    // row interchanges, in order
    if (lane == 0)
      for (int p = 0; p < n; ++p) {
        int q = piv[p];
        if (q != p) {
          double t = x[p];
          x[p] = x[q];
          x[q] = t;
        }
      }
    __syncwarp();
    for (int p = 0; p < n; ++p) {
      const double xp = x[p];
      __syncwarp();
      for (int i = p + 1 + lane; i < n; i += 32) x[i] = fma(-a[(int64_t)p * n + i], xp, x[i]);
      __syncwarp();
    }
    for (int p = n - 1; p >= 0; --p) {
      if (lane == 0) x[p] = x[p] / a[(int64_t)p * n + p];
      __syncwarp();
      const double xp = x[p];
      for (int i = lane; i < p; i += 32) x[i] = fma(-a[(int64_t)p * n + i], xp, x[i]);
      __syncwarp();
    }
  }
}

}  // namespace

int leaf_lu_launch(const LeafLULaunch& L, int nleaves, int smax, cudaStream_t s) {
  size_t smem = sizeof(double) * (size_t)smax * (smax | 1);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(leaf_lu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  leaf_lu_kernel<<<nleaves, LNT, smem, s>>>(L);
  return (int)cudaGetLastError();
}

int leaf_solve_launch(const LeafSolveLaunch& L, int nleaves, int smax, cudaStream_t s) {
  if (L.ncols <= 0) return 0;
  if (L.ncols <= 16) {
    constexpr int TC = 16;
    size_t smem = sizeof(double) * (size_t)(smax | 1) * (smax + TC);
    cudaFuncSetAttribute(leaf_solve_kernel<TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    leaf_solve_kernel<TC><<<dim3((L.ncols + TC - 1) / TC, nleaves), LNT, smem, s>>>(L);
  } else {
    constexpr int TC = 64;
    size_t smem = sizeof(double) * (size_t)(smax | 1) * (smax + TC);
    cudaFuncSetAttribute(leaf_solve_kernel<TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    leaf_solve_kernel<TC><<<dim3((L.ncols + TC - 1) / TC, nleaves), LNT, smem, s>>>(L);
  }
  return (int)cudaGetLastError();
}

int schur_factor_launch(const SchurLaunch& L, int nnodes, cudaStream_t s) {
  if (nnodes == 0) return 0;
  schur_form_kernel<<<nnodes, 256, 0, s>>>(L);
  dense_lu_kernel<<<nnodes, LNT, 0, s>>>(L);
  return (int)cudaGetLastError();
}

int schur_solve_launch(const SchurLaunch& L, int nnodes, int ncols, int max_cols,
                       cudaStream_t s) {
  if (nnodes == 0 || max_cols <= 0) return 0;
  int gx = (max_cols + (LNT / 32) - 1) / (LNT / 32);
  if (gx > 64) gx = 64;
  dense_lu_solve_kernel<<<dim3(gx, nnodes), LNT, 0, s>>>(L, ncols);
  return (int)cudaGetLastError();
}
