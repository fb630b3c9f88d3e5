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
//  schur_lu_kernel    blocked partial-pivot LU of each node's S in place
//                     (SchurLU = PartialPivLU(S), src/HODLR_Matrix.cpp:675).
//  schur_solve_kernel y = S^-1 rhs by the stored LU (src/HODLR_Matrix.cpp:682,746).
// Pivoting takes the first maximum |a| of the column, as PartialPivLU does.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "lu.h"

namespace {

constexpr int LNT = 256;

// ------------------------------------------------------------- leaf LU
__global__ void __launch_bounds__(LNT) leaf_lu_kernel(LeafLULaunch L) {
  extern __shared__ double a[];  // s x s, leading dimension s | 1
  __shared__ int s_piv;
  const int leaf = blockIdx.x;
  const int r0 = L.leaf_min[leaf], s = L.leaf_size[leaf];
  const int lda = s | 1;
  const int tid = threadIdx.x;
  int* perm = L.perm + r0;  // final row permutation, local indices
  const EntrySrc S = src_for(L.src, r0);  // the kernel of this leaf's system
  // assemble
  for (int e = tid; e < s * s; e += LNT) {
    int i = e % s, j = e / s;
    a[j * lda + i] = src_entry(S, r0 + i, r0 + j);
  }
  for (int i = tid; i < s; i += LNT) perm[i] = i;
  __syncthreads();
  if (L.a_copy)
    for (int e = tid; e < s * s; e += LNT) {
      int i = e % s, j = e / s;
      L.a_copy[r0 + i + (int64_t)j * L.lda_copy] = a[j * lda + i];
    }
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

// ------------------------------------------------ blocked tile solves
// x <- U^-1 L^-1 x for `ncol` columns of a tile in shared memory (x[c*ldx+i]),
// where the unit-lower L and the upper U are read through `A(i, j)` (the
// packed LU of an n x n matrix).  Diagonal blocks of BS rows are solved by one
// thread per column; the rows below / above are updated by all threads.
constexpr int BS = 16;

struct SmemLU {
  const double* a;
  int lda;
  __device__ double operator()(int i, int j) const { return a[j * lda + i]; }
};
struct GlobalLU {
  const double* a;
  int n;
  __device__ double operator()(int i, int j) const { return __ldg(a + (int64_t)j * n + i); }
};

template <class LU>
__device__ void lu_solve_tile(const LU& A, int n, double* x, int ldx, int ncol) {
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int b0 = 0; b0 < n; b0 += BS) {  // forward, unit lower
    const int be = min(n, b0 + BS);
    for (int c = tid; c < ncol; c += NT) {
      double* xc = x + c * ldx;
      for (int i = b0 + 1; i < be; ++i) {
        double t = xc[i];
        for (int p = b0; p < i; ++p) t = fma(-A(i, p), xc[p], t);
        xc[i] = t;
      }
    }
    __syncthreads();
    const int rem = n - be;
    for (int e = tid; e < rem * ncol; e += NT) {
      const int r = be + e % rem, c = e / rem;
      double* xc = x + c * ldx;
      double t = xc[r];
      for (int p = b0; p < be; ++p) t = fma(-A(r, p), xc[p], t);
      xc[r] = t;
    }
    __syncthreads();
  }
  for (int be = n; be > 0; be -= BS) {  // backward, upper
    const int b0 = max(0, be - BS);
    for (int c = tid; c < ncol; c += NT) {
      double* xc = x + c * ldx;
      for (int i = be - 1; i >= b0; --i) {
        double t = xc[i];
        for (int p = i + 1; p < be; ++p) t = fma(-A(i, p), xc[p], t);
        xc[i] = t / A(i, i);
      }
    }
    __syncthreads();
    for (int e = tid; e < b0 * ncol; e += NT) {
      const int r = e % b0, c = e / b0;
      double* xc = x + c * ldx;
      double t = xc[r];
      for (int p = b0; p < be; ++p) t = fma(-A(r, p), xc[p], t);
      xc[r] = t;
    }
    __syncthreads();
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
    const int pi = perm[i];
    if (pi < 0 || pi >= s) {  // never written by a valid leaf LU: skip and report
      if (L.err) atomicOr(L.err, DEV_ERR_INDEX | DEV_ERR_AT_LEAF_PERM);
      x[c * ldx + i] = 0.0;
      continue;
    }
    x[c * ldx + i] = L.X[(int64_t)(c0 + c) * L.ldx + r0 + pi];
  }
  __syncthreads();
  lu_solve_tile(SmemLU{lu, lda}, s, x, ldx, ncol);
  for (int e = tid; e < s * ncol; e += LNT) {
    int i = e % s, cc = e / s;
    L.X[(int64_t)(c0 + cc) * L.ldx + r0 + i] = x[cc * ldx + i];
  }
}

// ---------------------------------------------------------- Schur form
// S[node] (sd x sd, sd = kb + kt): identity blocks on the diagonal, the level
// products of Z on the off-diagonal blocks.  With n1 the size of the first
// unknown block (kb in recLU order, kt in recSM order), Z's rows follow the
// same order and its own-level columns start at coff: the upper-right block
// is Z[:n1, coff + (j - n1)], the lower-left Z[n1:, coff + j].
// CTA (node, y) fills every gridDim.y-th slice of the node's entries, so a
// large S is written by many CTAs.
__global__ void schur_form_kernel(SchurLaunch L) {
  const int node = blockIdx.x;
  const SchurNode N = L.nodes[node];
  const int sd = N.kb + N.kt;
  double* S = L.S + N.s_off;
  const double* Z = L.Z + N.z_off;  // sd x zcols, ld sd
  const int n1 = N.order ? N.kt : N.kb;
  for (int64_t e = threadIdx.x + (int64_t)blockIdx.y * blockDim.x; e < (int64_t)sd * sd;
       e += (int64_t)blockDim.x * gridDim.y) {
    int i = (int)(e % sd), j = (int)(e / sd);
    double v;
    if ((i < n1) == (j < n1))
      v = (i == j) ? 1.0 : 0.0;
    else if (i < n1)  // recLU: V_b^T K_t^-1 U_t; recSM: V_t^T K_b^-1 U_b
      v = Z[(int64_t)(N.coff + j - n1) * sd + i];
    else  // recLU: V_t^T K_b^-1 U_b; recSM: V_b^T K_t^-1 U_t
      v = Z[(int64_t)(N.coff + j) * sd + i];
    S[(int64_t)j * sd + i] = v;
  }
}

// ------------------------------------------------------ dense batched LU
// Blocked right-looking LU with row partial pivoting, S in global memory (L2
// resident).  Panels of PNB columns are factored in shared memory; the
// trailing matrix is updated with 4x4 register tiles.  The row interchanges
// of a panel are applied to the whole row, so the packed result and `piv`
// are those of an unblocked partial-pivot LU with the same pivot choices
// (LAPACK getrf convention).
constexpr int SNT = 512;

// One CTA factors columns [jlo, jhi) of the n x n matrix a (columns < jlo
// final, their interchanges already applied to columns >= jlo): the pivots of
// those columns go to piv, their interchanges are applied to the columns of
// [jlo, jhi) only, and the columns >= jhi are not touched.  jlo = 0,
// jhi = n is the whole LU.
__device__ bool lu_columns(double* a, int n, int* piv, int jlo, int jhi, int pnb, double* pan,
                           double* red_v, int* red_i, int* lpiv) {
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  bool singular = false;
  for (int j0 = jlo; j0 < jhi; j0 += pnb) {
    const int nb = min(pnb, jhi - j0), rows = n - j0;
    for (int e = tid; e < rows * nb; e += SNT) {
      int r = e % rows, c = e / rows;
      pan[c * rows + r] = a[(int64_t)(j0 + c) * n + j0 + r];
    }
    __syncthreads();
    for (int c = 0; c < nb; ++c) {
      // pivot: first maximum |.| of panel column c, rows c..rows-1
      double bv = -1.0;
      int bi = INT_MAX;
      for (int r = c + tid; r < rows; r += SNT) {
        double v = fabs(pan[c * rows + r]);
        if (v > bv) {
          bv = v;
          bi = r;
        }
      }
      warp_argmax(bv, bi);
      if (lane == 0) {
        red_v[w] = bv;
        red_i[w] = bi;
      }
      __syncthreads();
      if (w == 0) {
        bv = lane < SNT / 32 ? red_v[lane] : -1.0;
        bi = lane < SNT / 32 ? red_i[lane] : INT_MAX;
        warp_argmax(bv, bi);
        if (lane == 0) lpiv[c] = (bi == INT_MAX) ? c : bi;
      }
      __syncthreads();
      const int q = lpiv[c];
      if (q != c)
        for (int cc = tid; cc < nb; cc += SNT) {
          double t = pan[cc * rows + c];
          pan[cc * rows + c] = pan[cc * rows + q];
          pan[cc * rows + q] = t;
        }
      __syncthreads();
      const double d = pan[c * rows + c];
      if (d == 0.0) {
        singular = true;
        continue;
      }
      for (int r = c + 1 + tid; r < rows; r += SNT) pan[c * rows + r] /= d;
      __syncthreads();
      const int rr = rows - c - 1, cols = nb - c - 1;
      for (int e = tid; e < rr * cols; e += SNT) {
        int r = c + 1 + e % rr, cc = c + 1 + e / rr;
        pan[cc * rows + r] = fma(-pan[c * rows + r], pan[cc * rows + c], pan[cc * rows + r]);
      }
      __syncthreads();
    }
    // panel back to global, pivots, interchanges in the other columns of the range
    for (int e = tid; e < rows * nb; e += SNT) {
      int r = e % rows, c = e / rows;
      a[(int64_t)(j0 + c) * n + j0 + r] = pan[c * rows + r];
    }
    if (tid < nb) piv[j0 + tid] = j0 + lpiv[tid];
    for (int col = jlo + tid; col < jhi; col += SNT) {
      if (col >= j0 && col < j0 + nb) continue;
      double* ac = a + (int64_t)col * n;
      for (int c = 0; c < nb; ++c) {
        const int q = lpiv[c];
        if (q != c) {
          double t = ac[j0 + c];
          ac[j0 + c] = ac[j0 + q];
          ac[j0 + q] = t;
        }
      }
    }
    __syncthreads();
    const int rest = n - j0 - nb;      // trailing rows
    const int crest = jhi - j0 - nb;   // trailing columns inside the range
    if (rest > 0 && crest > 0) {
      // U12 = L11^-1 A12, one thread per column
      for (int col = j0 + nb + tid; col < jhi; col += SNT) {
        double* ac = a + (int64_t)col * n + j0;
        for (int i = 1; i < nb; ++i) {
          double t = ac[i];
          for (int p = 0; p < i; ++p) t = fma(-pan[p * rows + i], ac[p], t);
          ac[i] = t;
        }
      }
      __syncthreads();
      // A22 -= L21 U12 with 4x4 register tiles
      const int tr = (rest + 3) / 4, tc = (crest + 3) / 4;
      for (int tt = tid; tt < tr * tc; tt += SNT) {
        const int ti = (tt % tr) * 4, tj = (tt / tr) * 4;
        double acc[4][4];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
        for (int p = 0; p < nb; ++p) {
          double l[4], u[4];
#pragma unroll
          for (int x = 0; x < 4; ++x) l[x] = (ti + x < rest) ? pan[p * rows + nb + ti + x] : 0.0;
#pragma unroll
          for (int y = 0; y < 4; ++y)
            u[y] = (tj + y < crest) ? a[(int64_t)(j0 + nb + tj + y) * n + j0 + p] : 0.0;
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) acc[x][y] = fma(l[x], u[y], acc[x][y]);
        }
#pragma unroll
        for (int y = 0; y < 4; ++y) {
          if (tj + y >= crest) continue;
          double* ac = a + (int64_t)(j0 + nb + tj + y) * n + j0 + nb + ti;
#pragma unroll
          for (int x = 0; x < 4; ++x)
            if (ti + x < rest) ac[x] -= acc[x][y];
        }
      }
      __syncthreads();
    }
  }
  return singular;
}

// Whole LU of every node with sd < big_sd, one CTA per node (larger nodes are
// left to the multi-CTA path below).
__global__ void __launch_bounds__(SNT) schur_lu_kernel(SchurLaunch L, int pnb, int big_sd) {
  extern __shared__ double pan[];  // rows x pnb panel, leading dimension rows
  __shared__ double red_v[SNT / 32];
  __shared__ int red_i[SNT / 32];
  __shared__ int lpiv[64];
  const SchurNode N = L.nodes[blockIdx.x];
  const int n = N.kb + N.kt;
  if (n >= big_sd) return;
  const bool singular =
      lu_columns(L.S + N.s_off, n, L.piv + N.p_off, 0, n, pnb, pan, red_v, red_i, lpiv);
  if (threadIdx.x == 0 && singular) atomicOr(L.err, DEV_ERR_SINGULAR);
}

// ------------------------------------------- multi-CTA LU of large nodes
// Right-looking, outer panels of BNB columns.  Per panel j0, for every large
// node (its index in BigNodes): (1) one CTA factors the panel columns
// [j0, j0+BNB) with lu_columns; (2) many CTAs apply the panel's interchanges
// to every other column and form U12 = L11^-1 A12 right of the panel; (3)
// A22 -= L21 U12 in 64 x 64 tiles over all SMs.  The pivot choices are the
// column-wise first maxima, as in the one-CTA kernel.
constexpr int BNB = 32;
constexpr int BIG_MAX = 1024;  // nodes per launch (kernel parameter: 4 KB)
struct BigNodes {
  int idx[BIG_MAX];
  int count;
};

__global__ void __launch_bounds__(SNT) big_panel_kernel(SchurLaunch L, BigNodes B, int j0, int pnb) {
  extern __shared__ double pan[];
  __shared__ double red_v[SNT / 32];
  __shared__ int red_i[SNT / 32];
  __shared__ int lpiv[64];
  const SchurNode N = L.nodes[B.idx[blockIdx.x]];
  const int n = N.kb + N.kt;
  if (j0 >= n) return;
  const bool singular = lu_columns(L.S + N.s_off, n, L.piv + N.p_off, j0, min(n, j0 + BNB), pnb,
                                   pan, red_v, red_i, lpiv);
  if (threadIdx.x == 0 && singular) atomicOr(L.err, DEV_ERR_SINGULAR);
}

// One thread per column outside the panel: the panel's interchanges, then
// (right of the panel) the unit-lower solve with L11.
__global__ void __launch_bounds__(256) big_swap_trsm_kernel(SchurLaunch L, BigNodes B, int j0) {
  __shared__ double l11[BNB][BNB + 1];
  __shared__ int sp[BNB];
  const SchurNode N = L.nodes[B.idx[blockIdx.y]];
  const int n = N.kb + N.kt;
  if (j0 >= n) return;
  const int nb = min(BNB, n - j0);
  double* a = L.S + N.s_off;
  const int* piv = L.piv + N.p_off;
  for (int e = threadIdx.x; e < BNB * BNB; e += blockDim.x) {
    const int i = e % BNB, p = e / BNB;
    l11[i][p] = (i < nb && p < nb) ? a[(int64_t)(j0 + p) * n + j0 + i] : 0.0;
  }
  if (threadIdx.x < BNB) sp[threadIdx.x] = threadIdx.x < nb ? piv[j0 + threadIdx.x] : 0;
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n || (col >= j0 && col < j0 + nb)) return;
  double* ac = a + (int64_t)col * n;
  for (int c = 0; c < nb; ++c) {
    const int q = sp[c];
    if (q < j0 + c || q >= n) {  // not an LU interchange: skip and report
      atomicOr(L.err, DEV_ERR_INDEX | DEV_ERR_AT_LU_SWAP);
      continue;
    }
    if (q != j0 + c) {
      const double t = ac[j0 + c];
      ac[j0 + c] = ac[q];
      ac[q] = t;
    }
  }
  if (col < j0) return;
  double u[BNB];
#pragma unroll
  for (int i = 0; i < BNB; ++i) u[i] = i < nb ? ac[j0 + i] : 0.0;
#pragma unroll
  for (int i = 1; i < BNB; ++i)
#pragma unroll
    for (int p = 0; p < i; ++p) u[i] = fma(-l11[i][p], u[p], u[i]);
#pragma unroll
  for (int i = 0; i < BNB; ++i)
    if (i < nb) ac[j0 + i] = u[i];
}

// A22 -= L21 U12: CTA (ti, tj, node) owns a 64 x 64 tile, 256 threads with
// 4 x 4 outputs each; L21 and U12 tiles staged in shared memory.
constexpr int BT = 64;
__global__ void __launch_bounds__(256) big_update_kernel(SchurLaunch L, BigNodes B, int j0) {
  __shared__ double ls[BNB][BT + 1];  // L21 tile, [p][row]
  __shared__ double us[BNB][BT + 1];  // U12 tile, [p][col]
  const SchurNode N = L.nodes[B.idx[blockIdx.z]];
  const int n = N.kb + N.kt;
  const int r0 = j0 + BNB + blockIdx.x * BT, c0 = j0 + BNB + blockIdx.y * BT;
  if (r0 >= n || c0 >= n) return;
  double* a = L.S + N.s_off;
  for (int e = threadIdx.x; e < BNB * BT; e += blockDim.x) {
    const int i = e % BT, p = e / BT;
    ls[p][i] = r0 + i < n ? a[(int64_t)(j0 + p) * n + r0 + i] : 0.0;
    us[p][i] = c0 + i < n ? a[(int64_t)(c0 + i) * n + j0 + p] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // rows tx + 16x, cols ty + 16y
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
#pragma unroll 8
  for (int p = 0; p < BNB; ++p) {
    double l[4], u[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) l[x] = ls[p][tx + 16 * x];
#pragma unroll
    for (int y = 0; y < 4; ++y) u[y] = us[p][ty + 16 * y];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = fma(l[x], u[y], acc[x][y]);
  }
#pragma unroll
  for (int y = 0; y < 4; ++y) {
    const int c = c0 + ty + 16 * y;
    if (c >= n) continue;
    double* ac = a + (int64_t)c * n;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      const int r = r0 + tx + 16 * x;
      if (r < n) ac[r] -= acc[x][y];
    }
  }
}

// ---------------------------------- blocked solve of large nodes' ancestor columns
// y = S^-1 Z for the N.coff ancestor columns of a node with sd >= SCHUR_BIG_SOLVE_SD
// (the factorization's schur solve, src/HODLR_Matrix.cpp:682): the LU's row
// interchanges, then the unit-lower and the upper solves by 32-row diagonal
// blocks, each a register-resident triangular solve (one thread per column)
// followed by a 64 x 64-tiled update of the remaining rows over all SMs.  The
// one-CTA-per-column-tile kernel would read the whole LU again for every 16
// columns; here each block of the LU is read once per 64 columns.
__global__ void __launch_bounds__(256) big_rhs_perm_kernel(SchurLaunch L, BigNodes B) {
  const SchurNode N = L.nodes[B.idx[blockIdx.y]];
  const int n = N.kb + N.kt;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N.coff) return;
  double* x = L.R + N.r_off + (int64_t)c * n;
  const int* piv = L.piv + N.p_off;
  for (int p = 0; p < n; ++p) {
    const int q = __ldg(piv + p);
    if (q < p || q >= n) {  // not an LU interchange: skip and report
      atomicOr(L.err, DEV_ERR_INDEX | DEV_ERR_AT_BLOCKED_PIV);
      continue;
    }
    if (q != p) {
      const double t = x[p];
      x[p] = x[q];
      x[q] = t;
    }
  }
}

template <bool LOWER>
__global__ void __launch_bounds__(256) big_rhs_diag_kernel(SchurLaunch L, BigNodes B, int j0) {
  __shared__ double t11[BNB][BNB + 1];
  const SchurNode N = L.nodes[B.idx[blockIdx.y]];
  const int n = N.kb + N.kt;
  if (j0 >= n) return;
  const int nb = min(BNB, n - j0);
  const double* a = L.S + N.s_off;
  for (int e = threadIdx.x; e < BNB * BNB; e += blockDim.x) {
    const int i = e % BNB, p = e / BNB;
    t11[i][p] = (i < nb && p < nb) ? a[(int64_t)(j0 + p) * n + j0 + i] : (i == p ? 1.0 : 0.0);
  }
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N.coff) return;
  double* x = L.R + N.r_off + (int64_t)c * n + j0;
  double u[BNB];
#pragma unroll
  for (int i = 0; i < BNB; ++i) u[i] = i < nb ? x[i] : 0.0;
  if (LOWER) {  // unit lower, rows in order
#pragma unroll
    for (int i = 1; i < BNB; ++i)
#pragma unroll
      for (int p = 0; p < i; ++p) u[i] = fma(-t11[i][p], u[p], u[i]);
  } else {  // upper, rows in reverse order
#pragma unroll
    for (int i = BNB - 1; i >= 0; --i) {
      u[i] = u[i] / t11[i][i];
#pragma unroll
      for (int p = 0; p < i; ++p) u[p] = fma(-t11[p][i], u[i], u[p]);
    }
  }
#pragma unroll
  for (int i = 0; i < BNB; ++i)
    if (i < nb) x[i] = u[i];
}

// Rows below the block (LOWER) or above it (!LOWER) of the node's ancestor
// columns -= S[those rows, block columns] * the block's solved rows.
template <bool LOWER>
__global__ void __launch_bounds__(256) big_rhs_update_kernel(SchurLaunch L, BigNodes B, int j0) {
  __shared__ double ls[BNB][BT + 1];  // S tile, [p][row]
  __shared__ double us[BNB][BT + 1];  // solved block rows, [p][col]
  const SchurNode N = L.nodes[B.idx[blockIdx.z]];
  const int n = N.kb + N.kt;
  if (j0 >= n) return;
  const int nb = min(BNB, n - j0);
  const int rlo = LOWER ? j0 + nb : 0, rhi = LOWER ? n : j0;
  const int r0 = rlo + blockIdx.x * BT, c0 = blockIdx.y * BT;
  if (r0 >= rhi || c0 >= N.coff) return;
  const double* a = L.S + N.s_off;
  double* x = L.R + N.r_off;
  for (int e = threadIdx.x; e < BNB * BT; e += blockDim.x) {
    const int i = e % BT, p = e / BT;
    ls[p][i] = (p < nb && r0 + i < rhi) ? a[(int64_t)(j0 + p) * n + r0 + i] : 0.0;
    us[p][i] = (p < nb && c0 + i < N.coff) ? x[(int64_t)(c0 + i) * n + j0 + p] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int y = 0; y < 4; ++y) acc[q][y] = 0.0;
#pragma unroll 8
  for (int p = 0; p < BNB; ++p) {
    double l[4], u[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) l[q] = ls[p][tx + 16 * q];
#pragma unroll
    for (int y = 0; y < 4; ++y) u[y] = us[p][ty + 16 * y];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[q][y] = fma(l[q], u[y], acc[q][y]);
  }
#pragma unroll
  for (int y = 0; y < 4; ++y) {
    const int c = c0 + ty + 16 * y;
    if (c >= N.coff) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + tx + 16 * q;
      if (r < rhi) x[(int64_t)c * n + r] -= acc[q][y];
    }
  }
}

// x <- U^-1 L^-1 x for `ncol` columns in shared memory (x[c*ldx+i]) with the
// packed LU of an n x n matrix in global memory (column-major, ld n): the
// capacitance matrices, up to a few thousand rows, with few columns per CTA.
// Diagonal blocks of GB rows: one warp per column substitutes with the
// block's row of A in registers (lane = row) and each solved value broadcast
// by a shuffle, so the sequential chain is shuffles and FMAs, not memory
// loads.  Rows outside the block: one thread per row loads its GB entries of
// A once and updates every column.  The forward sweep performs exactly the
// operations of a row-by-row substitution, in the same order (ascending
// column); the backward sweep subtracts within a diagonal block in
// descending column order.
constexpr int GB = 32;

__device__ void lu_solve_global(const double* __restrict__ a, int n, double* x, int ldx,
                                int ncol) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, NW = NT >> 5;
  for (int b0 = 0; b0 < n; b0 += GB) {  // forward, unit lower
    const int nb = min(GB, n - b0), be = b0 + nb;
    if (wid < ncol) {
      double ar[GB];  // A(b0 + lane, b0 + p), p < lane
#pragma unroll
      for (int p = 0; p < GB; ++p)
        ar[p] = (p < lane && lane < nb) ? __ldg(a + (int64_t)(b0 + p) * n + b0 + lane) : 0.0;
      for (int c = wid; c < ncol; c += NW) {
        double* xc = x + c * ldx + b0;
        double t = lane < nb ? xc[lane] : 0.0;
#pragma unroll
        for (int p = 0; p < GB - 1; ++p) {
          const double xp = __shfl_sync(0xffffffffu, t, p);
          if (p < lane) t = fma(-ar[p], xp, t);
        }
        if (lane < nb) xc[lane] = t;
      }
    }
    __syncthreads();
    for (int r = be + tid; r < n; r += NT) {
      double ar[GB];  // A(r, b0 + p)
#pragma unroll
      for (int p = 0; p < GB; ++p) ar[p] = p < nb ? __ldg(a + (int64_t)(b0 + p) * n + r) : 0.0;
      for (int c = 0; c < ncol; ++c) {
        double* xc = x + c * ldx;
        double t = xc[r];
#pragma unroll
        for (int p = 0; p < GB; ++p)
          if (p < nb) t = fma(-ar[p], xc[b0 + p], t);
        xc[r] = t;
      }
    }
    __syncthreads();
  }
  for (int be = n; be > 0; be -= GB) {  // backward, upper
    const int b0 = max(0, be - GB), nb = be - b0;
    if (wid < ncol) {
      double ar[GB];  // A(b0 + lane, b0 + p), p > lane
#pragma unroll
      for (int p = 0; p < GB; ++p)
        ar[p] = (lane < p && p < nb) ? __ldg(a + (int64_t)(b0 + p) * n + b0 + lane) : 0.0;
      const double ad = lane < nb ? __ldg(a + (int64_t)(b0 + lane) * n + b0 + lane) : 1.0;
      for (int c = wid; c < ncol; c += NW) {
        double* xc = x + c * ldx + b0;
        double t = lane < nb ? xc[lane] : 0.0;
#pragma unroll
        for (int p = GB - 1; p >= 0; --p) {
          if (p >= nb) continue;  // the same for every lane
          if (lane == p) t = t / ad;
          const double xp = __shfl_sync(0xffffffffu, t, p);
          if (lane < p) t = fma(-ar[p], xp, t);
        }
        if (lane < nb) xc[lane] = t;
      }
    }
    __syncthreads();
    for (int r = tid; r < b0; r += NT) {
      double ar[GB];  // A(r, b0 + p)
#pragma unroll
      for (int p = 0; p < GB; ++p) ar[p] = p < nb ? __ldg(a + (int64_t)(b0 + p) * n + r) : 0.0;
      for (int c = 0; c < ncol; ++c) {
        double* xc = x + c * ldx;
        double t = xc[r];
#pragma unroll
        for (int p = 0; p < GB; ++p)
          if (p < nb) t = fma(-ar[p], xc[b0 + p], t);
        xc[r] = t;
      }
    }
    __syncthreads();
  }
}

// y = S^-1 rhs for `ncols` right-hand sides stored in R (ld sd) at r_off
// (ncols < 0: N.coff columns); one CTA per (node, tile of STC columns).
// WARP_SUBST selects lu_solve_global, whose short sequential chains suit the
// solve (one CTA per node, latency-bound at the top levels); the ancestor
// columns of the factorization (many CTAs per node, throughput-bound) keep
// the 32-register blocked tile solve.
constexpr int STC = 16;

// tc columns per CTA (STC, or fewer where a column tile would not fit in
// shared memory); in_smem == false: the columns are solved in place in
// global memory (capacitance matrices too large for even one column).
template <bool WARP_SUBST>
__global__ void __launch_bounds__(256) schur_solve_kernel(SchurLaunch L, int ncols, int tc,
                                                          bool in_smem, int skip_sd) {
  extern __shared__ double xs_smem[];
  const int node = blockIdx.y;
  const SchurNode N = L.nodes[node];
  const int n = N.kb + N.kt;
  if (n >= skip_sd) return;  // left to the blocked solve
  const int cols = ncols < 0 ? N.coff : ncols;
  const int c0 = blockIdx.x * tc;
  if (c0 >= cols) return;
  const int nc = min(tc, cols - c0);
  const double* a = L.S + N.s_off;
  const int* piv = L.piv + N.p_off;
  double* R = L.R + N.r_off;
  const int ldx = in_smem ? (n | 1) : n;
  double* xs = in_smem ? xs_smem : R + (int64_t)c0 * n;
  if (in_smem) {
    for (int e = threadIdx.x; e < n * nc; e += blockDim.x) {
      int i = e % n, c = e / n;
      xs[c * ldx + i] = R[(int64_t)(c0 + c) * n + i];
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    double* xc = xs + c * ldx;
    for (int p = 0; p < n; ++p) {
      int q = piv[p];
      if (q < p || q >= n) {  // not an LU interchange: skip and report
        atomicOr(L.err, DEV_ERR_INDEX | DEV_ERR_AT_SOLVE_PIV);
        continue;
      }
      if (q != p) {
        double t = xc[p];
        xc[p] = xc[q];
        xc[q] = t;
      }
    }
  }
  __syncthreads();
  if (WARP_SUBST)
    lu_solve_global(a, n, xs, ldx, nc);
  else
    lu_solve_tile(GlobalLU{a, n}, n, xs, ldx, nc);
  if (in_smem) {
    for (int e = threadIdx.x; e < n * nc; e += blockDim.x) {
      int i = e % n, c = e / n;
      R[(int64_t)(c0 + c) * n + i] = xs[c * ldx + i];
    }
  }
}

// Launch helpers return the first CUDA error at once.
#define LCK(call)                             \
  do {                                        \
    cudaError_t e__ = (call);                 \
    if (e__ != cudaSuccess) return (int)e__;  \
  } while (0)

}  // namespace

int leaf_lu_launch(const LeafLULaunch& L, int nleaves, int smax, cudaStream_t s) {
  size_t smem = sizeof(double) * (size_t)smax * (smax | 1);
  LCK(smem_opt_in((const void*)leaf_lu_kernel, smem));
  leaf_lu_kernel<<<nleaves, LNT, smem, s>>>(L);
  return (int)cudaGetLastError();
}

int leaf_solve_launch(const LeafSolveLaunch& L, int nleaves, int smax, cudaStream_t s) {
  if (L.ncols <= 0) return 0;
  if (L.ncols <= 16) {
    constexpr int TC = 16;
    size_t smem = sizeof(double) * (size_t)(smax | 1) * (smax + TC);
    LCK(smem_opt_in((const void*)leaf_solve_kernel<TC>, smem));
    leaf_solve_kernel<TC><<<dim3((L.ncols + TC - 1) / TC, nleaves), LNT, smem, s>>>(L);
  } else {
    constexpr int TC = 64;
    size_t smem = sizeof(double) * (size_t)(smax | 1) * (smax + TC);
    LCK(smem_opt_in((const void*)leaf_solve_kernel<TC>, smem));
    leaf_solve_kernel<TC><<<dim3((L.ncols + TC - 1) / TC, nleaves), LNT, smem, s>>>(L);
  }
  return (int)cudaGetLastError();
}

// Inner panel width for rows x pnb doubles of shared memory (<= 200 KB).
static int panel_width(int rows) {
  int pnb = 16;
  while (pnb > 1 && (size_t)rows * pnb * sizeof(double) > 200 * 1024) pnb >>= 1;
  return pnb;
}

int schur_factor_launch(const SchurLaunch& L, int nnodes, const int* sd, cudaStream_t s) {
  if (nnodes == 0) return 0;
  int form_y = 1;  // CTAs per node for forming S: about 64K entries each
  for (int i = 0; i < nnodes; ++i)
    form_y = std::max(form_y, (int)std::min<int64_t>(256, (int64_t)sd[i] * sd[i] / 65536 + 1));
  schur_form_kernel<<<dim3(nnodes, form_y), 256, 0, s>>>(L);
  LCK(cudaGetLastError());
  int small_max = 0, big_max = 0;
  std::vector<int> big;
  for (int i = 0; i < nnodes; ++i) {
    if (sd[i] >= SCHUR_BIG_SD) {
      big.push_back(i);
      big_max = std::max(big_max, sd[i]);
    } else {
      small_max = std::max(small_max, sd[i]);
    }
  }
  if (small_max > 0) {
    const int pnb = panel_width(small_max);
    size_t smem = (size_t)small_max * pnb * sizeof(double);
    LCK(smem_opt_in((const void*)schur_lu_kernel, smem));
    schur_lu_kernel<<<nnodes, SNT, smem, s>>>(L, pnb, SCHUR_BIG_SD);
    LCK(cudaGetLastError());
  }
  for (size_t b0 = 0; b0 < big.size(); b0 += BIG_MAX) {
    BigNodes B;
    B.count = (int)std::min<size_t>(BIG_MAX, big.size() - b0);
    int mx = 0;
    for (int i = 0; i < B.count; ++i) {
      B.idx[i] = big[b0 + i];
      mx = std::max(mx, sd[big[b0 + i]]);
    }
    const int pnb = std::min(BNB, panel_width(mx));
    const size_t smem = (size_t)mx * pnb * sizeof(double);
    LCK(smem_opt_in((const void*)big_panel_kernel, smem));
    for (int j0 = 0; j0 < mx; j0 += BNB) {
      big_panel_kernel<<<B.count, SNT, smem, s>>>(L, B, j0, pnb);
      LCK(cudaGetLastError());
      big_swap_trsm_kernel<<<dim3((mx + 255) / 256, B.count), 256, 0, s>>>(L, B, j0);
      LCK(cudaGetLastError());
      const int rest = mx - j0 - BNB;
      if (rest > 0) {
        const int t = (rest + BT - 1) / BT;
        big_update_kernel<<<dim3(t, t, B.count), 256, 0, s>>>(L, B, j0);
        LCK(cudaGetLastError());
      }
    }
  }
  return (int)cudaGetLastError();
}

int schur_factor_launches(const int* sd, int nnodes) {
  int n = 1, small = 0, mx = 0, big = 0;
  for (int i = 0; i < nnodes; ++i) {
    if (sd[i] >= SCHUR_BIG_SD) {
      ++big;
      mx = std::max(mx, sd[i]);
    } else {
      small = 1;
    }
  }
  n += small;
  if (big) {
    const int batches = (big + BIG_MAX - 1) / BIG_MAX;
    for (int j0 = 0; j0 < mx; j0 += BNB) n += batches * (mx - j0 - BNB > 0 ? 3 : 2);
  }
  return n;
}

int schur_solve_factor_launch(const SchurLaunch& L, int nnodes, const int* sd, int coff,
                              cudaStream_t s, int* launches) {
  *launches = 0;
  if (nnodes == 0 || coff <= 0) return 0;
  std::vector<int> big;
  int small_max = 0;
  for (int i = 0; i < nnodes; ++i) {
    if (sd[i] >= SCHUR_BIG_SOLVE_SD)
      big.push_back(i);
    else
      small_max = std::max(small_max, sd[i]);
  }
  if (small_max > 0) {
    const size_t col_bytes = sizeof(double) * (size_t)(small_max | 1);
    const int tc = (int)std::max<size_t>(1, std::min<size_t>(STC, 200 * 1024 / col_bytes));
    const size_t smem = col_bytes * tc;
    LCK(smem_opt_in((const void*)schur_solve_kernel<false>, smem));
    schur_solve_kernel<false><<<dim3((coff + tc - 1) / tc, nnodes), 256, smem, s>>>(
        L, -1, tc, true, SCHUR_BIG_SOLVE_SD);
    LCK(cudaGetLastError());
    ++*launches;
  }
  const int ctiles = (coff + BT - 1) / BT, cblocks = (coff + 255) / 256;
  for (size_t b0 = 0; b0 < big.size(); b0 += BIG_MAX) {
    BigNodes B;
    B.count = (int)std::min<size_t>(BIG_MAX, big.size() - b0);
    int mx = 0;
    for (int i = 0; i < B.count; ++i) {
      B.idx[i] = big[b0 + i];
      mx = std::max(mx, sd[big[b0 + i]]);
    }
    big_rhs_perm_kernel<<<dim3(cblocks, B.count), 256, 0, s>>>(L, B);
    LCK(cudaGetLastError());
    ++*launches;
    for (int j0 = 0; j0 < mx; j0 += BNB) {
      big_rhs_diag_kernel<true><<<dim3(cblocks, B.count), 256, 0, s>>>(L, B, j0);
      LCK(cudaGetLastError());
      const int rows = mx - j0 - BNB;
      if (rows > 0) {
        big_rhs_update_kernel<true><<<dim3((rows + BT - 1) / BT, ctiles, B.count), 256, 0, s>>>(
            L, B, j0);
        LCK(cudaGetLastError());
      }
      *launches += 1 + (rows > 0);
    }
    for (int j0 = (mx - 1) / BNB * BNB; j0 >= 0; j0 -= BNB) {
      big_rhs_diag_kernel<false><<<dim3(cblocks, B.count), 256, 0, s>>>(L, B, j0);
      LCK(cudaGetLastError());
      if (j0 > 0) {
        big_rhs_update_kernel<false><<<dim3((j0 + BT - 1) / BT, ctiles, B.count), 256, 0, s>>>(
            L, B, j0);
        LCK(cudaGetLastError());
      }
      *launches += 1 + (j0 > 0);
    }
  }
  return (int)cudaGetLastError();
}

int schur_solve_launch(const SchurLaunch& L, int nnodes, int ncols, int max_cols, int max_sd,
                       cudaStream_t s) {
  if (nnodes == 0 || max_cols <= 0) return 0;
  // columns per CTA: STC, fewer when a tile of them would exceed the
  // shared-memory budget, none (in place in global memory) past one column
  const size_t col_bytes = sizeof(double) * (size_t)(max_sd | 1);
  constexpr size_t kBudget = 200 * 1024;
  const int tc = (int)std::max<size_t>(1, std::min<size_t>(STC, kBudget / col_bytes));
  const bool in_smem = col_bytes <= kBudget;
  const size_t smem = in_smem ? col_bytes * tc : 0;
  const dim3 grid((max_cols + tc - 1) / tc, nnodes);
  if (ncols >= 0) {
    LCK(smem_opt_in((const void*)schur_solve_kernel<true>, smem));
    schur_solve_kernel<true><<<grid, 256, smem, s>>>(L, ncols, tc, in_smem, INT_MAX);
  } else {
    LCK(smem_opt_in((const void*)schur_solve_kernel<false>, smem));
    schur_solve_kernel<false><<<grid, 256, smem, s>>>(L, ncols, tc, in_smem, INT_MAX);
  }
  return (int)cudaGetLastError();
}
