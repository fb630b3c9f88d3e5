// Full-kernel product Y = K X in FP64 with every entry generated on the fly.
// Replaces kernelMatrix::operator* (src/kernel.cpp:27-35), which the
// reference uses for the residual ||K x - b|| / ||b|| (src/HODLR_Matrix.cpp:
// 785-787), and supplies the residual of iterative refinement and GMRES.
//
// Bound by the FP64 units: the distance, square root and Tang exp from
// kfast.cuh (specialised per kernel family at compile time, no dispatch) and
// two products per right-hand side and evaluated entry.  Four forms:
//   kmatvec_kernel          row by row (dense input, the no-alloc entry, up to
//                           16 right-hand sides); column ranges split over
//                           gridDim.y, partial sums added in a fixed order;
//   kmatvec_sym_kernel      each entry evaluated once for K_ij and K_ji,
//                           1 to 4 right-hand sides, FMAs;
//   kmatvec_sym_mma_kernel  the same for 5 to 8 right-hand sides with the
//                           products on mma.m8n8k4.f64;
//   kmatvec_forest_kernel   block-diagonal product over a forest of systems.
#include "common.cuh"
#include "kfast.cuh"
#include "kmatvec.h"

namespace {

constexpr int KT = 128;
constexpr int RPT = 2;  // rows per thread

__constant__ double c_tang[HX_TANG_TABLE_SIZE] = HX_TANG_TABLE_INIT;

template <int NR, int KTYPE, int DIM>
__global__ void __launch_bounds__(KT) kmatvec_kernel(KmatvecLaunch L) {
  __shared__ double xs[DIM > 0 ? DIM : 1][KT];
  __shared__ double vs[NR][KT];
  __shared__ double tab[HX_TANG_TABLE_SIZE];
  const int n = L.n;
  const int nsplit = gridDim.y;
  const int per = ((n + nsplit - 1) / nsplit + KT - 1) / KT * KT;
  const int jb = blockIdx.y * per, je = min(n, jb + per);
  for (int i = threadIdx.x; i < HX_TANG_TABLE_SIZE; i += blockDim.x) tab[i] = c_tang[i];
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


// ------------------------------------------------------------ symmetric form
// K is symmetric entry for entry (the squared distance of i, j and of j, i
// are the same sums of the same rounded squares), so one evaluation of K_ij
// serves both y_i += K_ij x_j and y_j += K_ij x_i.  The points are cut into
// 256-point tiles and the tiles into S splits; CTA (a, b), a <= b, takes every
// tile pair (I in split a, J in split b), J >= I when a == b.  Its row sums
// (rows of a) go to slice b of the workspace, its column sums (rows of b) to
// slice a: every (slice, row) is written by exactly one CTA, in a fixed order,
// and Y = sum over slices (kmatvec_reduce) is deterministic.  Diagonal tile
// pairs (J == I) are evaluated in full with row sums only.
//
// Column sums without a cross-lane reduction per column: within a group of 32
// columns, lane L handles column (s + L) mod 32 at step s and then hands its
// column accumulator to lane L - 1, so each accumulator follows one column
// around the warp and ends, after 32 steps, in the lane of that column.  The
// four warps' group sums are added through shared memory (double-buffered
// per group) and accumulated into the workspace.
constexpr int ST = 256;  // tile edge (rows = columns)
constexpr int SG = 32;   // rotation group
// 1 to 4 right-hand sides (more go to kmatvec_sym_mma_kernel): 2 rows per
// thread, 128 threads
template <int NR>
struct SymCfg {
  static_assert(NR == 1 || NR == 4, "the FMA form serves 1 to 4 right-hand sides");
  static constexpr int RPT = 2;
  static constexpr int NT = ST / RPT;
  static constexpr int NW = NT / 32;
  static constexpr int MINB = 3;
};

template <int NR>
struct SymPad {  // row stride of the staged X tile: an odd number of 16-byte units
  static constexpr int VS = NR == 1 ? 1 : NR + 2;
};

template <int NR, int KTYPE, int DIM>
__global__ void __launch_bounds__(SymCfg<NR>::NT, SymCfg<NR>::MINB)
    kmatvec_sym_kernel(KmatvecLaunch L, int S, int tps) {
  constexpr int SYM_RPT = SymCfg<NR>::RPT, SYM_NT = SymCfg<NR>::NT, SYM_NW = SymCfg<NR>::NW;
  constexpr int VS = SymPad<NR>::VS;
  __shared__ double xs[DIM][ST];
  __shared__ __align__(16) double vs[ST][VS];
  __shared__ __align__(16) double colw[2][SYM_NW][SG][VS];
  __shared__ double tab[HX_TANG_TABLE_SIZE];
  const int n = L.n;
  const int nT = (n + ST - 1) / ST;
  int a, b;
  {
    const int nup = S * (S - 1) / 2;
    int p = blockIdx.x;
    if (p < nup) {
      a = 0;
      while (p >= S - 1 - a) {
        p -= S - 1 - a;
        ++a;
      }
      b = a + 1 + p;
    } else {
      a = b = p - nup;
    }
  }
  const int ia0 = a * tps, ia1 = min(nT, ia0 + tps);
  const int jb1 = min(nT, b * tps + tps);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < HX_TANG_TABLE_SIZE; i += blockDim.x) tab[i] = c_tang[i];
  const double cs = hx_point_scale<KTYPE>(L.src.kp.a);  // coordinates scaled once
  const int64_t slice = (int64_t)L.nrhs * n;
  double* __restrict__ wsA = L.ws + (int64_t)a * slice;  // column sums (rows of split b)
  double* __restrict__ wsB = L.ws + (int64_t)b * slice;  // row sums (rows of split a)
  const hx_kparams kp = L.src.kp;
  const double dcorr = kp.diag_replace ? kp.diag_value - 1.0 : kp.shift;

  for (int I = ia0; I < ia1; ++I) {
    int row[SYM_RPT];
    bool live[SYM_RPT];
    double xi[SYM_RPT][DIM];
    double xv[SYM_RPT][NR];
    double acc[SYM_RPT][NR];
#pragma unroll
    for (int q = 0; q < SYM_RPT; ++q) {
      row[q] = I * ST + q * SYM_NT + threadIdx.x;
      live[q] = row[q] < n;
#pragma unroll
      for (int d = 0; d < DIM; ++d) xi[q][d] = live[q] ? cs * L.src.pts[d * L.src.ld + row[q]] : 0.0;
#pragma unroll
      for (int c = 0; c < NR; ++c) {
        xv[q][c] = (live[q] && c < L.nrhs) ? L.X[(int64_t)c * L.ldx + row[q]] : 0.0;
        acc[q][c] = 0.0;
      }
    }
    const int jstart = a == b ? I : b * tps;
    for (int J = jstart; J < jb1; ++J) {
      __syncthreads();  // every thread is done with the previous tile
      for (int t = threadIdx.x; t < ST; t += SYM_NT) {
        const int j = J * ST + t;
        const bool ok = j < n;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xs[d][t] = ok ? cs * L.src.pts[d * L.src.ld + j] : 0.0;
#pragma unroll
        for (int c = 0; c < NR; ++c)
          vs[t][c] = (ok && c < L.nrhs) ? L.X[(int64_t)c * L.ldx + j] : 0.0;
      }
      __syncthreads();
      if (J == I) {  // diagonal tile pair: all entries, row sums only
#pragma unroll 2
        for (int t = 0; t < ST; ++t) {
#pragma unroll
          for (int q = 0; q < SYM_RPT; ++q) {
            double r2 = HX_R2_FLOOR;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
              const double dd = xi[q][d] - xs[d][t];
              r2 = fma(dd, dd, r2);
            }
            const double k = hx_kernel_unit_t<KTYPE>(r2, tab);
#pragma unroll
            for (int c = 0; c < NR; ++c) acc[q][c] = fma(k, vs[t][c], acc[q][c]);
          }
        }
        continue;
      }
      for (int g = 0; g < ST / SG; ++g) {
        double cacc[NR];
#pragma unroll
        for (int c = 0; c < NR; ++c) cacc[c] = 0.0;
#pragma unroll 2
        for (int s = 0; s < SG; ++s) {
          const int t = g * SG + ((s + lane) & (SG - 1));
          double xj[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d) xj[d] = xs[d][t];
          double vj[NR];
          if (NR == 1) {
            vj[0] = vs[t][0];
          } else {
#pragma unroll
            for (int c = 0; c < NR; c += 2) {
              const double2 v2 = *reinterpret_cast<const double2*>(&vs[t][c]);
              vj[c] = v2.x;
              vj[c + 1] = v2.y;
            }
          }
#pragma unroll
          for (int q = 0; q < SYM_RPT; ++q) {
            double r2 = HX_R2_FLOOR;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
              const double dd = xi[q][d] - xj[d];
              r2 = fma(dd, dd, r2);
            }
            const double k = hx_kernel_unit_t<KTYPE>(r2, tab);
#pragma unroll
            for (int c = 0; c < NR; ++c) {
              acc[q][c] = fma(k, vj[c], acc[q][c]);
              cacc[c] = fma(k, xv[q][c], cacc[c]);
            }
          }
#pragma unroll
          for (int c = 0; c < NR; ++c) cacc[c] = __shfl_sync(0xffffffffu, cacc[c], (lane + 1) & 31);
        }
        // lane L holds column g * SG + L of this warp's rows
        double* cw = &colw[g & 1][w][lane][0];
        if (NR == 1) {
          cw[0] = cacc[0];
        } else {
#pragma unroll
          for (int c = 0; c < NR; c += 2)
            *reinterpret_cast<double2*>(&cw[c]) = make_double2(cacc[c], cacc[c + 1]);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < SG * NR; e += SYM_NT) {
          const int tl = e % SG, c = e / SG;
          const int j = J * ST + g * SG + tl;
          if (c < L.nrhs && j < n) {
            double sum = colw[g & 1][0][tl][c];
#pragma unroll
            for (int ww = 1; ww < SYM_NW; ++ww) sum += colw[g & 1][ww][tl][c];
            double* dst = wsA + (int64_t)c * n + j;
            *dst = I == ia0 ? sum : *dst + sum;
          }
        }
      }
    }
    // row sums of tile I; in a diagonal block the earlier tiles' column sums
    // are already there, and K_ii = f(0) + shift (or the replaced value)
#pragma unroll
    for (int q = 0; q < SYM_RPT; ++q) {
      if (!live[q]) continue;
#pragma unroll
      for (int c = 0; c < NR; ++c) {
        if (c >= L.nrhs) continue;
        double v = acc[q][c];
        if (a == b) v = fma(dcorr, xv[q][c], v);
        double* dst = wsB + (int64_t)c * n + row[q];
        *dst = (a == b && I != ia0) ? *dst + v : v;
      }
    }
  }
}

// ---------------------------------------- symmetric form, 8 right-hand sides
// The same tile-pair schedule and workspace ownership as kmatvec_sym_kernel,
// with the per-entry products on the FP64 tensor-core instruction
// mma.m8n8k4.f64 (D[8x8] += A[8x4] B[4x8]; lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) .. +1]).  Warp w of 8 owns rows
// 32w .. 32w+31 of tile I as four 8-row chunks and walks tile J in 8-column
// chunks.  In a chunk lane (g, t) evaluates e0 = K[g][t] and e1 = K[g][t+4]:
//   row sums    Y_I[rows][rhs] += K[rows][cols] X_J[cols][rhs]: A = e0, e1;
//   column sums Y_J[cols][rhs] += K^T[cols][rows] X_I[rows][rhs]: A needs
//               K[t][g], K[t+4][g], the transpose, which goes through a
//               per-warp shared-memory buffer (two 8-byte stores, one 16-byte
//               load per lane).
// The chunks are software-pipelined: the column MMAs of chunk c - 1 (its
// transpose written and warp-synchronised in the previous step) are issued
// beside the entries of chunk c, so their dependent chain hides under the
// entry arithmetic; two transpose buffers suffice because a step reads the
// previous buffer before its own warp barrier.  Each warp's column sums of a
// chunk are stored per warp; after every 32 columns the CTA adds the eight
// warps' sums in warp order into the workspace slice, so every (slice, row)
// still has one writer in a fixed order.  The FP64 work per entry is the
// entry itself plus 16 FMAs inside the MMAs, as in the FMA form, with half
// the instructions and half the registers.
constexpr int MMA_NT = 256;  // 8 warps
constexpr int MMA_VSP = ST + 8;  // padded row stride of the staged X tile

__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// staged position of tile column u: chunk c = u / 8 keeps its 8 columns, and
// columns t and t + 4 of a chunk sit side by side (one 16-byte load per lane)
__device__ __forceinline__ int mma_pos(int u) { return (u & ~7) + 2 * (u & 3) + ((u >> 2) & 1); }

// dynamic shared memory of the kernel, in doubles
template <int DIM>
struct MmaSmem {
  static constexpr int XS = 0;                        // [DIM][ST] column coordinates
  static constexpr int VS = XS + DIM * ST;            // [8][MMA_VSP] X_J by rhs
  static constexpr int TR = VS + 8 * MMA_VSP;         // [8 warps][2][4 row chunks][64]
  static constexpr int CW = TR + 8 * 2 * 4 * 64;      // [2][8 warps][8 rhs][34]
  static constexpr int TAB = CW + 2 * 8 * 8 * 34;     // [HX_TANG_TABLE_SIZE]
  static constexpr size_t BYTES = (size_t)(TAB + HX_TANG_TABLE_SIZE) * sizeof(double);
};

template <int KTYPE, int DIM>
__global__ void __launch_bounds__(MMA_NT, 2)
    kmatvec_sym_mma_kernel(KmatvecLaunch L, int S, int tps) {
  extern __shared__ __align__(16) double mma_smem[];
  using M = MmaSmem<DIM>;
  double(*xs)[ST] = reinterpret_cast<double(*)[ST]>(mma_smem + M::XS);
  double(*vsT)[MMA_VSP] = reinterpret_cast<double(*)[MMA_VSP]>(mma_smem + M::VS);
  double(*tr)[2][4][64] = reinterpret_cast<double(*)[2][4][64]>(mma_smem + M::TR);
  double(*colw)[8][8][34] = reinterpret_cast<double(*)[8][8][34]>(mma_smem + M::CW);
  double* tab = mma_smem + M::TAB;
  const int n = L.n;
  const int nT = (n + ST - 1) / ST;
  int a, b;
  {
    const int nup = S * (S - 1) / 2;
    int p = blockIdx.x;
    if (p < nup) {
      a = 0;
      while (p >= S - 1 - a) {
        p -= S - 1 - a;
        ++a;
      }
      b = a + 1 + p;
    } else {
      a = b = p - nup;
    }
  }
  const int ia0 = a * tps, ia1 = min(nT, ia0 + tps);
  const int jb1 = min(nT, b * tps + tps);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int i = threadIdx.x; i < HX_TANG_TABLE_SIZE; i += blockDim.x) tab[i] = c_tang[i];
  const double cs = hx_point_scale<KTYPE>(L.src.kp.a);
  const int64_t slice = (int64_t)L.nrhs * n;
  double* __restrict__ wsA = L.ws + (int64_t)a * slice;
  double* __restrict__ wsB = L.ws + (int64_t)b * slice;
  const hx_kparams kp = L.src.kp;
  const double dcorr = kp.diag_replace ? kp.diag_value - 1.0 : kp.shift;
  const int wsl = 8 * t + 2 * (g & 3) + (g >> 2);  // where this lane's K[g][t] goes

  for (int I = ia0; I < ia1; ++I) {
    const int rbase = I * ST + 32 * w;
    double xr[4][DIM];        // coordinates of row g of each chunk
    double xi0[4], xi1[4];    // X_I[row t][rhs g], X_I[row t + 4][rhs g]
    double accR[4][2];        // Y_I[row g][rhs 2t, 2t + 1]
#pragma unroll
    for (int rc = 0; rc < 4; ++rc) {
      const int r = rbase + 8 * rc + g;
#pragma unroll
      for (int d = 0; d < DIM; ++d) xr[rc][d] = r < n ? cs * L.src.pts[d * L.src.ld + r] : 0.0;
      const int r0 = rbase + 8 * rc + t, r1 = r0 + 4;
      const bool cg = g < L.nrhs;
      xi0[rc] = (cg && r0 < n) ? L.X[(int64_t)g * L.ldx + r0] : 0.0;
      xi1[rc] = (cg && r1 < n) ? L.X[(int64_t)g * L.ldx + r1] : 0.0;
      accR[rc][0] = accR[rc][1] = 0.0;
    }
    const int jstart = a == b ? I : b * tps;
    for (int J = jstart; J < jb1; ++J) {
      __syncthreads();  // every thread is done with the previous tile
      {
        const int u = threadIdx.x, j = J * ST + u, pu = mma_pos(u);
        const bool ok = j < n;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xs[d][pu] = ok ? cs * L.src.pts[d * L.src.ld + j] : 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) vsT[c][pu] = (ok && c < L.nrhs) ? L.X[(int64_t)c * L.ldx + j] : 0.0;
      }
      __syncthreads();
      // entries of chunk cc and their row sums
      auto chunk = [&](int cc, double (&e0)[4], double (&e1)[4]) {
        const int p0 = 8 * cc + 2 * t;
        double xc0[DIM], xc1[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const double2 v = *reinterpret_cast<const double2*>(&xs[d][p0]);
          xc0[d] = v.x;
          xc1[d] = v.y;
        }
        const double2 xb = *reinterpret_cast<const double2*>(&vsT[g][p0]);
#pragma unroll
        for (int rc = 0; rc < 4; ++rc) {
          double s0 = HX_R2_FLOOR, s1 = HX_R2_FLOOR;
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            const double d0 = xr[rc][d] - xc0[d], d1 = xr[rc][d] - xc1[d];
            s0 = fma(d0, d0, s0);
            s1 = fma(d1, d1, s1);
          }
          e0[rc] = hx_kernel_unit_t<KTYPE>(s0, tab);
          e1[rc] = hx_kernel_unit_t<KTYPE>(s1, tab);
          dmma_884(accR[rc], e0[rc], xb.x);
          dmma_884(accR[rc], e1[rc], xb.y);
        }
      };
      auto put_tr = [&](int buf, const double (&e0)[4], const double (&e1)[4]) {
        double* tb = &tr[w][buf][0][0];
#pragma unroll
        for (int rc = 0; rc < 4; ++rc) {
          tb[rc * 64 + wsl] = e0[rc];
          tb[rc * 64 + 32 + wsl] = e1[rc];
        }
      };
      auto get_tr = [&](int buf, double2 (&v)[4]) {
        const double* tb = &tr[w][buf][0][0];
#pragma unroll
        for (int rc = 0; rc < 4; ++rc) v[rc] = *reinterpret_cast<const double2*>(&tb[rc * 64 + 8 * g + 2 * t]);
      };
      // column sums of chunk cc over this warp's rows, into the group buffer
      auto col_sums = [&](int cc, const double2 (&v)[4]) {
        double accC[2] = {0.0, 0.0};
#pragma unroll
        for (int rc = 0; rc < 4; ++rc) {
          dmma_884(accC, v[rc].x, xi0[rc]);
          dmma_884(accC, v[rc].y, xi1[rc]);
        }
        colw[(cc >> 2) & 1][w][2 * t][8 * (cc & 3) + g] = accC[0];
        colw[(cc >> 2) & 1][w][2 * t + 1][8 * (cc & 3) + g] = accC[1];
      };
      auto reduce_group = [&](int grp) {
        const int col = threadIdx.x & 31, c = threadIdx.x >> 5;
        const int j = J * ST + grp * 32 + col;
        if (c < L.nrhs && j < n) {
          double sum = colw[grp & 1][0][c][col];
#pragma unroll
          for (int ww = 1; ww < 8; ++ww) sum += colw[grp & 1][ww][c][col];
          double* dst = wsA + (int64_t)c * n + j;
          *dst = I == ia0 ? sum : *dst + sum;
        }
      };
      if (J == I) {  // diagonal tile pair: all entries, row sums only
#pragma unroll 1
        for (int cc = 0; cc < ST / 8; ++cc) {
          double e0[4], e1[4];
          chunk(cc, e0, e1);
        }
        continue;
      }
      // software pipeline: the column sums of chunk cc - 1 (entries already
      // transposed) run beside the entries of chunk cc
      {
        double e0[4], e1[4];
        chunk(0, e0, e1);
        put_tr(0, e0, e1);
        __syncwarp();
      }
#pragma unroll 1
      for (int cc = 1; cc < ST / 8; ++cc) {
        double2 v[4];
        get_tr((cc - 1) & 1, v);
        double e0[4], e1[4];
        chunk(cc, e0, e1);
        col_sums(cc - 1, v);
        put_tr(cc & 1, e0, e1);
        __syncwarp();
        if ((cc & 3) == 0) {
          __syncthreads();
          reduce_group((cc >> 2) - 1);
        }
      }
      {
        double2 v[4];
        get_tr(1, v);
        col_sums(ST / 8 - 1, v);
      }
      __syncthreads();
      reduce_group(ST / 32 - 1);
    }
    // row sums of tile I; in a diagonal block the earlier tiles' column sums
    // are already there, and K_ii = f(0) + shift (or the replaced value)
#pragma unroll
    for (int rc = 0; rc < 4; ++rc) {
      const int r = rbase + 8 * rc + g;
      if (r >= n) continue;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int c = 2 * t + q;
        if (c >= L.nrhs) continue;
        double v = accR[rc][q];
        if (a == b) v = fma(dcorr, L.X[(int64_t)c * L.ldx + r], v);
        double* dst = wsB + (int64_t)c * n + r;
        *dst = (a == b && I != ia0) ? *dst + v : v;
      }
    }
  }
}

template <int KTYPE, int DIM>
void launch_sym_mma_dim(const KmatvecLaunch& L, int S, int tps, cudaStream_t s) {
  // the opt-in above 48 KB of shared memory, for the current device (set on
  // every launch, as the attribute is per device); a failure shows as the
  // launch's error
  cudaFuncSetAttribute(kmatvec_sym_mma_kernel<KTYPE, DIM>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MmaSmem<DIM>::BYTES);
  const int grid = S * (S + 1) / 2;
  kmatvec_sym_mma_kernel<KTYPE, DIM><<<grid, MMA_NT, MmaSmem<DIM>::BYTES, s>>>(L, S, tps);
}

template <int KTYPE>
void launch_sym_mma(const KmatvecLaunch& L, int S, int tps, cudaStream_t s) {
  if (L.src.kp.dim == 1)
    launch_sym_mma_dim<KTYPE, 1>(L, S, tps, s);
  else if (L.src.kp.dim == 2)
    launch_sym_mma_dim<KTYPE, 2>(L, S, tps, s);
  else
    launch_sym_mma_dim<KTYPE, 3>(L, S, tps, s);
}

void launch_sym_mma_type(const KmatvecLaunch& L, int S, int tps, cudaStream_t s) {
  switch (L.src.kp.type) {
    case HX_KERNEL_GAUSSIAN: launch_sym_mma<HX_KERNEL_GAUSSIAN>(L, S, tps, s); break;
    case HX_KERNEL_MATERN32: launch_sym_mma<HX_KERNEL_MATERN32>(L, S, tps, s); break;
    case HX_KERNEL_INV_MULTIQUADRIC: launch_sym_mma<HX_KERNEL_INV_MULTIQUADRIC>(L, S, tps, s); break;
    case HX_KERNEL_QUADRATIC: launch_sym_mma<HX_KERNEL_QUADRATIC>(L, S, tps, s); break;
    default: launch_sym_mma<HX_KERNEL_EXPONENTIAL>(L, S, tps, s); break;
  }
}

template <int NR, int KTYPE>
void launch_sym_dim(const KmatvecLaunch& L, int S, int tps, cudaStream_t s) {
  const int grid = S * (S + 1) / 2;
  if (L.src.kp.dim == 1)
    kmatvec_sym_kernel<NR, KTYPE, 1><<<grid, SymCfg<NR>::NT, 0, s>>>(L, S, tps);
  else if (L.src.kp.dim == 2)
    kmatvec_sym_kernel<NR, KTYPE, 2><<<grid, SymCfg<NR>::NT, 0, s>>>(L, S, tps);
  else
    kmatvec_sym_kernel<NR, KTYPE, 3><<<grid, SymCfg<NR>::NT, 0, s>>>(L, S, tps);
}

template <int NR>
void launch_sym_type(const KmatvecLaunch& L, int S, int tps, cudaStream_t s) {
  switch (L.src.kp.type) {
    case HX_KERNEL_GAUSSIAN: launch_sym_dim<NR, HX_KERNEL_GAUSSIAN>(L, S, tps, s); break;
    case HX_KERNEL_MATERN32: launch_sym_dim<NR, HX_KERNEL_MATERN32>(L, S, tps, s); break;
    case HX_KERNEL_INV_MULTIQUADRIC: launch_sym_dim<NR, HX_KERNEL_INV_MULTIQUADRIC>(L, S, tps, s); break;
    case HX_KERNEL_QUADRATIC: launch_sym_dim<NR, HX_KERNEL_QUADRATIC>(L, S, tps, s); break;
    default: launch_sym_dim<NR, HX_KERNEL_EXPONENTIAL>(L, S, tps, s); break;
  }
}

// Tiles per split: about 96 splits (4656 CTAs) once there are enough tiles.
int sym_tps(int n) {
  const int nT = (n + ST - 1) / ST;
  return nT <= 96 ? 1 : (nT + 95) / 96;
}

// ------------------------------------------------------------ forest form
// Block-diagonal product over a forest of independent systems.  Work item
// (x, y, z, w) = rows [x, min(x + 2*KT, z)) of system w against its columns
// [y, z), with system w's kernel (L.src.kps[w]); one launch per kernel family
// present, items largest system first.  Every row is owned by one CTA and
// written once: no workspace, deterministic.
template <int NR, int KTYPE, int DIM>
__global__ void __launch_bounds__(KT) kmatvec_forest_kernel(KmatvecLaunch L,
                                                            const int4* __restrict__ items) {
  __shared__ double xs[DIM][KT];
  __shared__ double vs[NR][KT];
  __shared__ double tab[HX_TANG_TABLE_SIZE];
  const int4 it = items[blockIdx.x];
  if (L.skip && L.skip[it.w]) return;  // a converged system of a refinement
  const hx_kparams kp = L.src.kps[it.w];
  for (int i = threadIdx.x; i < HX_TANG_TABLE_SIZE; i += blockDim.x) tab[i] = c_tang[i];
  int row[RPT];
  bool live[RPT];
  double xi[RPT][DIM];
  double acc[RPT][NR];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    row[q] = it.x + q * KT + threadIdx.x;
    live[q] = row[q] < it.z;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[q][d] = live[q] ? L.src.pts[d * L.src.ld + row[q]] : 0.0;
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[q][c] = 0.0;
  }
  for (int j0 = it.y; j0 < it.z; j0 += KT) {
    const int jn = min(KT, it.z - j0);
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
        double r2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const double dd = xi[q][d] - xs[d][t];
          r2 = fma(dd, dd, r2);
        }
        const double kij = hx_kernel_r2_fast_t<KTYPE>(kp.a, r2, tab);
#pragma unroll
        for (int c = 0; c < NR; ++c) acc[q][c] = fma(kij, vs[c][t], acc[q][c]);
      }
    }
  }
  const double dcorr = kp.diag_replace ? kp.diag_value - 1.0 : kp.shift;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    if (!live[q]) continue;
#pragma unroll
    for (int c = 0; c < NR; ++c)
      if (c < L.nrhs)
        L.Y[(int64_t)c * L.ldy + row[q]] =
            fma(dcorr, L.X[(int64_t)c * L.ldx + row[q]], acc[q][c]);
  }
}

template <int NR, int KTYPE>
void launch_forest_dim(const KmatvecLaunch& L, const int4* items, int count, cudaStream_t s) {
  if (L.src.kp.dim == 1)
    kmatvec_forest_kernel<NR, KTYPE, 1><<<count, KT, 0, s>>>(L, items);
  else if (L.src.kp.dim == 2)
    kmatvec_forest_kernel<NR, KTYPE, 2><<<count, KT, 0, s>>>(L, items);
  else
    kmatvec_forest_kernel<NR, KTYPE, 3><<<count, KT, 0, s>>>(L, items);
}

template <int NR>
void launch_forest_type(const KmatvecLaunch& L, int type, const int4* items, int count,
                        cudaStream_t s) {
  switch (type) {
    case HX_KERNEL_GAUSSIAN: launch_forest_dim<NR, HX_KERNEL_GAUSSIAN>(L, items, count, s); break;
    case HX_KERNEL_MATERN32: launch_forest_dim<NR, HX_KERNEL_MATERN32>(L, items, count, s); break;
    case HX_KERNEL_INV_MULTIQUADRIC:
      launch_forest_dim<NR, HX_KERNEL_INV_MULTIQUADRIC>(L, items, count, s);
      break;
    case HX_KERNEL_QUADRATIC: launch_forest_dim<NR, HX_KERNEL_QUADRATIC>(L, items, count, s); break;
    default: launch_forest_dim<NR, HX_KERNEL_EXPONENTIAL>(L, items, count, s); break;
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

int kmatvec_sym_slices(int n, int nrhs, bool dense) {
  if (dense || nrhs > 8 || n < 1) return 0;
  const int nT = (n + ST - 1) / ST;
  const int tps = sym_tps(n);
  return (nT + tps - 1) / tps;
}

int kmatvec_sym_launch(const KmatvecLaunch& L, int S, cudaStream_t s) {
  const int tps = sym_tps(L.n);
  if (S != kmatvec_sym_slices(L.n, L.nrhs, L.src.dense) || S < 1) return (int)cudaErrorInvalidValue;
  if (L.nrhs <= 1)
    launch_sym_type<1>(L, S, tps, s);
  else if (L.nrhs <= 4)
    launch_sym_type<4>(L, S, tps, s);
  else
    launch_sym_mma_type(L, S, tps, s);
  kmatvec_reduce<<<1024, 256, 0, s>>>(L, S);
  return (int)cudaGetLastError();
}

int kmatvec_forest_launch(const KmatvecLaunch& L, const int4* d_items, const int* type_off,
                          cudaStream_t s) {
  if (L.nrhs < 1 || L.nrhs > 16) return (int)cudaErrorInvalidValue;
  for (int t = 0; t < HX_FOREST_TYPES; ++t) {
    const int count = type_off[t + 1] - type_off[t];
    if (count <= 0) continue;
    const int4* items = d_items + type_off[t];
    if (L.nrhs <= 1)
      launch_forest_type<1>(L, t, items, count, s);
    else if (L.nrhs <= 4)
      launch_forest_type<4>(L, t, items, count, s);
    else if (L.nrhs <= 8)
      launch_forest_type<8>(L, t, items, count, s);
    else
      launch_forest_type<16>(L, t, items, count, s);
  }
  return (int)cudaGetLastError();
}
