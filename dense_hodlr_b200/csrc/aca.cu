// Batched partial-pivot ACA: every off-diagonal block of a tree level (or of
// several levels) is compressed in one launch.
//
// Restates partialPivACA_LowRankApprox (src/lowRank.cpp:117-279) and
// chooseNextRowCol (src/lowRank.cpp:291-298).  The values that decide pivots
// are bit-identical to the CPU oracle: entries come from kfun.h, the residual
// row/column are accumulated in l order with separately rounded products and
// sums (src/lowRank.cpp:164-168, 211-215), the pivot is 1/r then multiplied
// (src/lowRank.cpp:208,230), and every argmax returns the first maximum.
// Only the Frobenius-norm dots of the stopping test (src/lowRank.cpp:234-241)
// are summed in a GPU order; they change epsilon in its last bits and thus
// the rank only when epsilon sits within rounding of the tolerance.  Each
// block records its smallest |eps - tol| / tol so such near ties are visible.
//
// Work decomposition.  A block is processed by a group of G CTAs.  CTA g owns
// a contiguous slice of the block's rows (for W, the column pass) and of its
// columns (for V, the row pass).  One ACA step is two group phases:
//   A  row residual on the column slice, slice argmax   -> barrier
//   B  pick pivot column, column residual on the row slice, slice argmax,
//      slice partial dots for the norm estimate          -> barrier
//   C  (redundant in every CTA) combine partials, epsilon, next row.
// G = 1 for levels with many blocks (barriers are __syncthreads); G > 1 runs
// under a cooperative launch so that a group's CTAs are co-resident, and its
// barrier is a counter in global memory polled with a bounded spin.
#include "common.cuh"
#include "hodlr_internal.h"

namespace {

struct Shared {
  double red_v[32];
  int red_i[32];
  int red_c[32];
  double bcast_d[8];
  int bcast_i[8];
};

// Group barrier.  gen counts the barriers this CTA has passed.
__device__ bool group_sync(unsigned* bar, int G, unsigned& gen, unsigned* err) {
  __syncthreads();
  if (G == 1) return true;
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_fail = 0;
    __threadfence();
    atomicAdd(bar, 1u);
    unsigned target = (gen + 1) * (unsigned)G;
    unsigned polls = 0;
    while (ld_acquire_u32(bar) < target) {
      if (++polls > HODLR_SPIN_LIMIT || *(volatile unsigned*)err) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        s_fail = 1;
        break;
      }
      __nanosleep(128);
    }
    __threadfence();
  }
  ++gen;
  __syncthreads();
  return s_fail == 0;
}

template <int NT>
__device__ void block_argmax(Shared& sh, double& v, int& i) {
  warp_argmax(v, i);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh.red_v[w] = v;
    sh.red_i[w] = i;
  }
  __syncthreads();
  if (w == 0) {
    v = lane < NT / 32 ? sh.red_v[lane] : -1.0;
    i = lane < NT / 32 ? sh.red_i[lane] : INT_MAX;
    warp_argmax(v, i);
  }
  __syncthreads();
}

template <int NT>
__device__ int block_min_int(Shared& sh, int x) {
  x = warp_min_int(x);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh.red_c[w] = x;
  __syncthreads();
  int r = INT_MAX;
  if (w == 0) {
    r = lane < NT / 32 ? sh.red_c[lane] : INT_MAX;
    r = warp_min_int(r);
    if (lane == 0) sh.bcast_i[7] = r;
  }
  __syncthreads();
  r = sh.bcast_i[7];
  __syncthreads();
  return r;
}

// Deterministic block sum (fixed tree); result valid in every thread.
template <int NT>
__device__ double block_sum(Shared& sh, double x) {
  x = warp_sum(x);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh.red_v[w] = x;
  __syncthreads();
  if (w == 0) {
    double y = lane < NT / 32 ? sh.red_v[lane] : 0.0;
    y = warp_sum(y);
    if (lane == 0) sh.bcast_d[7] = y;
  }
  __syncthreads();
  double r = sh.bcast_d[7];
  __syncthreads();
  return r;
}

// Combine the G slice partials (value, index, chosen-flag, candidate) stored
// at part[g * stride + off .. off+3].  Slices are in index order, so the
// lowest index among equal maxima is the first maximum of the block.
__device__ void reduce_partials(Shared& sh, const double* part, int64_t stride, int G,
                                int off, double& v, int& idx, int& flag, int& cand) {
  if (threadIdx.x < 32) {
    double bv = -1.0;
    int bi = INT_MAX, bf = 0, bc = INT_MAX;
    for (int g = threadIdx.x; g < G; g += 32) {
      const double* p = part + g * stride + off;
      double pv = __ldcg(p);
      int pi = (int)__ldcg(p + 1);
      int pf = (int)__ldcg(p + 2);
      int pc = (int)__ldcg(p + 3);
      if (pv > bv || (pv == bv && pi < bi)) {
        bv = pv;
        bi = pi;
        bf = pf;
      }
      bc = min(bc, pc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double v2 = __shfl_down_sync(0xffffffffu, bv, o);
      int i2 = __shfl_down_sync(0xffffffffu, bi, o);
      int f2 = __shfl_down_sync(0xffffffffu, bf, o);
      int c2 = __shfl_down_sync(0xffffffffu, bc, o);
      if (v2 > bv || (v2 == bv && i2 < bi)) {
        bv = v2;
        bi = i2;
        bf = f2;
      }
      bc = min(bc, c2);
    }
    if (threadIdx.x == 0) {
      sh.bcast_d[0] = bv;
      sh.bcast_i[0] = bi;
      sh.bcast_i[1] = bf;
      sh.bcast_i[2] = bc;
    }
  }
  __syncthreads();
  v = sh.bcast_d[0];
  idx = sh.bcast_i[0];
  flag = sh.bcast_i[1];
  cand = sh.bcast_i[2];
  __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT) aca_kernel(AcaLaunch L) {
  extern __shared__ double dyn[];  // wrow[kcap], vrow[kcap]
  __shared__ Shared sh;
  const int G = L.G;
  const int b = blockIdx.x / G, g = blockIdx.x % G;
  const int tid = threadIdx.x;
  if (b >= L.nblocks) return;
  const AcaBlock B = L.blocks[b];
  AcaState* st = B.st;
  if (st->status != ACA_RUNNING && st->status != ACA_POST) return;

  const int64_t ld = L.ld;
  const int m = B.m, n = B.n, ub = min(m, n);
  const double tol = L.tol, minPiv = L.minPivot;
  double* wrow = dyn;
  double* vrow = dyn + B.kcap;
  double* part_me = L.part + (int64_t)blockIdx.x * L.part_stride;
  const double* part_grp = L.part + (int64_t)(b * G) * L.part_stride;
  unsigned* bar = L.bar + b;
  unsigned gen = 0;

  const int sm = (m + G - 1) / G, sn = (n + G - 1) / G;
  const int i_lo = min(m, g * sm), i_hi = min(m, i_lo + sm);
  const int j_lo = min(n, g * sn), j_hi = min(n, j_lo + sn);

  int k = st->k, cur = st->cur, iters = st->iters, status = st->status;
  double frob2 = st->frob2, eps = st->eps, margin = st->margin;
  int near = st->near;
  bool nonfinite = false;

  while (status == ACA_RUNNING) {
    // while ((eps > tol || k < minRank) && k < ub), minRank = -1 on the default tree
    if (!(eps > tol) || k >= ub) {
      status = ACA_POST;
      break;
    }
    if (k >= B.kcap) {  // paused: the host grows the capacity and resumes
      status = ACA_NEED_CAP;
      break;
    }
    ++iters;
    // ---------------- phase A: residual row on this CTA's column slice
    if (g == 0 && tid == 0) B.cR[cur] = 1;
    for (int l = tid; l < k; l += NT) wrow[l] = __ldcg(B.W + cur + (int64_t)l * ld);
    __syncthreads();
    const int gi = B.r0 + cur;
    double xi[3] = {0.0, 0.0, 0.0};
    if (!L.src.dense)
      #pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < L.src.kp.dim) xi[d] = __ldg(L.src.pts + d * L.src.ld + gi);
    double bv = -1.0;
    int bi = INT_MAX, cand = INT_MAX;
    for (int j0 = j_lo + tid; j0 < j_hi; j0 += 4 * NT) {
      int jj[4];
      double s[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        jj[e] = j0 + e * NT;
        s[e] = 0.0;
      }
      const double* vp = B.V;
      for (int l = 0; l < k; ++l, vp += ld) {
        const double w = wrow[l];
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (jj[e] < j_hi) s[e] = __dadd_rn(s[e], __dmul_rn(w, vp[jj[e]]));
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = jj[e];
        if (j < j_hi) {
          double v = __dsub_rn(src_entry_xi(L.src, xi, gi, B.c0 + j), s[e]);
          B.V[j + (int64_t)k * ld] = v;
          double a = fabs(v);
          nonfinite |= !isfinite(v);
          if (a > bv) {  // increasing j per thread: keeps the first maximum
            bv = a;
            bi = j;
          }
          if (cand == INT_MAX && a > minPiv && __ldcg(B.cC + j) == 0) cand = j;
        }
      }
    }
    block_argmax<NT>(sh, bv, bi);
    cand = block_min_int<NT>(sh, cand);
    if (tid == 0) {
      part_me[0] = bv;
      part_me[1] = (double)bi;
      part_me[2] = (bi != INT_MAX) ? (double)__ldcg(B.cC + bi) : 0.0;
      part_me[3] = (double)cand;
    }
    if (!group_sync(bar, G, gen, L.err)) { status = ACA_ERROR; break; }

    // ---------------- phase B: pivot column, residual column on the row slice
    double mv;
    int mi, mflag, mcand;
    reduce_partials(sh, part_grp, L.part_stride, G, 0, mv, mi, mflag, mcand);
    if (mv <= minPiv) {
      // zero residual row: move to the first unchosen row (src/lowRank.cpp:187-195)
      int f = INT_MAX;
      for (int i = tid; i < m; i += NT)
        if (__ldcg(B.cR + i) == 0) { f = i; break; }
      f = block_min_int<NT>(sh, f);
      if (f == INT_MAX) { status = ACA_POST; break; }
      cur = f;
      if (!group_sync(bar, G, gen, L.err)) { status = ACA_ERROR; break; }
      continue;
    }
    int cc;
    if (!mflag) {
      cc = mi;
    } else {
      if (mcand == INT_MAX) { status = ACA_POST; break; }
      cc = mcand;
    }
    if (g == 0 && tid == 0) B.cC[cc] = 1;
    const double piv = __ddiv_rn(1.0, __ldcg(B.V + cc + (int64_t)k * ld));
    for (int l = tid; l < k; l += NT) vrow[l] = __ldcg(B.V + cc + (int64_t)l * ld);
    __syncthreads();
    const int gj = B.c0 + cc;
    double xj[3] = {0.0, 0.0, 0.0};
    if (!L.src.dense)
      #pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < L.src.kp.dim) xj[d] = __ldg(L.src.pts + d * L.src.ld + gj);
    bv = -1.0;
    bi = INT_MAX;
    cand = INT_MAX;
    double sw = 0.0;
    for (int i0 = i_lo + tid; i0 < i_hi; i0 += 4 * NT) {
      int ii[4];
      double s[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        ii[e] = i0 + e * NT;
        s[e] = 0.0;
      }
      const double* wp = B.W;
      for (int l = 0; l < k; ++l, wp += ld) {
        const double v = vrow[l];
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (ii[e] < i_hi) s[e] = __dadd_rn(s[e], __dmul_rn(v, wp[ii[e]]));
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int i = ii[e];
        if (i < i_hi) {
          double c = __dsub_rn(src_entry_xj(L.src, xj, B.r0 + i, gj), s[e]);
          double w = __dmul_rn(piv, c);
          B.W[i + (int64_t)k * ld] = w;
          sw = fma(w, w, sw);
          double a = fabs(c);
          nonfinite |= !isfinite(c);
          if (a > bv) {
            bv = a;
            bi = i;
          }
          if (cand == INT_MAX && a > minPiv && __ldcg(B.cR + i) == 0) cand = i;
        }
      }
    }
    block_argmax<NT>(sh, bv, bi);
    cand = block_min_int<NT>(sh, cand);
    if (tid == 0) {
      part_me[4] = bv;
      part_me[5] = (double)bi;
      part_me[6] = (bi != INT_MAX) ? (double)__ldcg(B.cR + bi) : 0.0;
      part_me[7] = (double)cand;
    }
    // partial dots of the norm update over this CTA's slices
    sw = block_sum<NT>(sh, sw);
    double sv = 0.0;
    for (int j = j_lo + tid; j < j_hi; j += NT) {
      double v = B.V[j + (int64_t)k * ld];
      sv = fma(v, v, sv);
    }
    sv = block_sum<NT>(sh, sv);
    {
      const int w = tid >> 5, lane = tid & 31;
      const double* wk = B.W + (int64_t)k * ld;
      const double* vk = B.V + (int64_t)k * ld;
      for (int l = w; l < k; l += NT / 32) {
        const double* wl = B.W + (int64_t)l * ld;
        const double* vl = B.V + (int64_t)l * ld;
        double aw = 0.0, av = 0.0;
        for (int i = i_lo + lane; i < i_hi; i += 32) aw = fma(wk[i], wl[i], aw);
        for (int j = j_lo + lane; j < j_hi; j += 32) av = fma(vl[j], vk[j], av);
        aw = warp_sum(aw);
        av = warp_sum(av);
        if (lane == 0) {
          part_me[8 + l] = aw;
          part_me[8 + B.kcap + l] = av;
        }
      }
      if (tid == 0) {
        part_me[8 + 2 * B.kcap] = sw;
        part_me[9 + 2 * B.kcap] = sv;
      }
    }
    if (!group_sync(bar, G, gen, L.err)) { status = ACA_ERROR; break; }

    // ---------------- phase C: next row, norm estimate, epsilon
    int nflag, ncand, ni;
    double nv;
    reduce_partials(sh, part_grp, L.part_stride, G, 4, nv, ni, nflag, ncand);
    int nr;
    if (!nflag)
      nr = ni;
    else
      nr = ncand;
    if (nr == INT_MAX) {  // no admissible next row: stop before storing (src/lowRank.cpp:226-227)
      status = ACA_POST;
      break;
    }
    double sum_local = 0.0;
    for (int l = tid; l < k; l += NT) {
      double dw = 0.0, dv = 0.0;
      for (int q = 0; q < G; ++q) {
        dw += __ldcg(part_grp + q * L.part_stride + 8 + l);
        dv += __ldcg(part_grp + q * L.part_stride + 8 + B.kcap + l);
      }
      sum_local += dw * dv;
    }
    double sumNorm = block_sum<NT>(sh, sum_local);
    double swt = 0.0, svt = 0.0;
    for (int q = 0; q < G; ++q) {
      swt += __ldcg(part_grp + q * L.part_stride + 8 + 2 * B.kcap);
      svt += __ldcg(part_grp + q * L.part_stride + 9 + 2 * B.kcap);
    }
    frob2 += 2 * sumNorm + swt * svt;
    eps = sqrt(swt) * sqrt(svt) / sqrt(frob2);
    if (g == 0 && tid == 0) {
      B.prow[k] = cur;
      B.pcol[k] = cc;
    }
    cur = nr;
    ++k;
    if (k < ub) {
      double gap = fabs(eps - tol) / tol;
      margin = fmin(margin, gap);
      if (gap < 1e-10) ++near;
    }
    // No barrier needed here: the next writes to the row partials happen
    // after every CTA has passed barrier 2, and W(:,k) / V(:,k) are final.
  }

  // ---------------- post-processing (src/lowRank.cpp:250-277)
  int rank = k;
  if (status == ACA_POST) {
    if (k == 0) {
      for (int i = i_lo + tid; i < i_hi; i += NT) B.W[i] = 0.0;
      for (int j = j_lo + tid; j < j_hi; j += NT) B.V[j] = 0.0;
      rank = 1;
      status = ACA_DONE;
    } else if (k >= ub - 1) {
      const int full = (n <= m) ? n : m;
      if (B.kcap < full) {
        status = ACA_NEED_CAP_POST;  // the full representation needs more columns
        rank = full;
      } else if (n <= m) {  // W = block (m x n), V = I_n
        for (int l = 0; l < n; ++l) {
          double xj[3] = {0.0, 0.0, 0.0};
          if (!L.src.dense)
#pragma unroll
            for (int d = 0; d < 3; ++d)
              if (d < L.src.kp.dim) xj[d] = __ldg(L.src.pts + d * L.src.ld + B.c0 + l);
          for (int i = i_lo + tid; i < i_hi; i += NT)
            B.W[i + (int64_t)l * ld] = src_entry_xj(L.src, xj, B.r0 + i, B.c0 + l);
          for (int j = j_lo + tid; j < j_hi; j += NT)
            B.V[j + (int64_t)l * ld] = (j == l) ? 1.0 : 0.0;
        }
        rank = n;
        status = ACA_DONE;
      } else {  // W = I_m, V = block^T (n x m)
        for (int l = 0; l < m; ++l) {
          double xi[3] = {0.0, 0.0, 0.0};
          if (!L.src.dense)
#pragma unroll
            for (int d = 0; d < 3; ++d)
              if (d < L.src.kp.dim) xi[d] = __ldg(L.src.pts + d * L.src.ld + B.r0 + l);
          for (int j = j_lo + tid; j < j_hi; j += NT)
            B.V[j + (int64_t)l * ld] = src_entry_xi(L.src, xi, B.r0 + l, B.c0 + j);
          for (int i = i_lo + tid; i < i_hi; i += NT)
            B.W[i + (int64_t)l * ld] = (i == l) ? 1.0 : 0.0;
        }
        rank = m;
        status = ACA_DONE;
      }
    } else {
      status = ACA_DONE;
    }
  }
  if (nonfinite) atomicOr(L.err, DEV_ERR_NONFINITE);
  // Every CTA of the group reached the same state; CTA 0 records it after a
  // last barrier, so that no CTA of the group can still be about to read the
  // entry state (a block that starts in post-processing has no barrier before).
  if (status != ACA_ERROR && !group_sync(bar, G, gen, L.err)) status = ACA_ERROR;
  if (g == 0 && tid == 0) {
    st->k = k;
    st->cur = cur;
    st->iters = iters;
    st->status = status;
    st->frob2 = frob2;
    st->eps = eps;
    st->margin = margin;
    st->near = near;
    st->rank = rank;
  }
}

}  // namespace

int aca_launch(const AcaLaunch& L, int nt, int kcap_max, bool cooperative, cudaStream_t s) {
  size_t smem = sizeof(double) * 2 * (size_t)kcap_max;
  dim3 grid(L.nblocks * L.G), block(nt);
  void* args[] = {(void*)&L};
  cudaError_t e;
  if (nt == 256) {
    auto fn = aca_kernel<256>;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    e = cooperative ? cudaLaunchCooperativeKernel((void*)fn, grid, block, args, smem, s)
                    : cudaLaunchKernel((void*)fn, grid, block, args, smem, s);
  } else {
    auto fn = aca_kernel<128>;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    e = cooperative ? cudaLaunchCooperativeKernel((void*)fn, grid, block, args, smem, s)
                    : cudaLaunchKernel((void*)fn, grid, block, args, smem, s);
  }
  return e == cudaSuccess ? 0 : (int)e;
}

int aca_max_coresident(int nt, int kcap_max, int* per_sm) {
  size_t smem = sizeof(double) * 2 * (size_t)kcap_max;
  int nb = 0;
  cudaError_t e;
  if (nt == 256) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(aca_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, aca_kernel<256>, nt, smem);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(aca_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, aca_kernel<128>, nt, smem);
  }
  *per_sm = nb;
  return e == cudaSuccess ? 0 : (int)e;
}
