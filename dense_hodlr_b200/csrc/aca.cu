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
//   B  pick pivot column, column residual on the row slice, slice argmax
//                                                        -> barrier
//   C  (redundant in every CTA) combine partials, next row.
// Each step streams the W and V panels once.  The stopping test of step k-1
// needs dots of its new columns with all earlier ones; they are accumulated
// while step k streams the same panels for its residuals, and step k is run
// speculatively: if epsilon_{k-1} <= tol it is discarded, so pivots and ranks
// are those of the reference's loop.  Where step k cannot stream the panels
// (a zero residual row, the capacity limit) the dots take a pass of their own.
// G = 1 for levels with many blocks (barriers are __syncthreads); G > 1 runs
// under a cooperative launch so that a group's CTAs are co-resident, and its
// barrier is a counter in global memory polled with a bounded spin.  Groups
// are either all of size L.G (CTA c works on block c / G) or, with a CTA
// table, of per-block size B.G starting at CTA B.g0 (sized from predicted
// ranks so that a level's blocks finish together).
#include "common.cuh"
#include "hodlr_internal.h"

namespace {

// The block's W or V panel in the launch's element type (FP64 panels).
template <typename T>
__device__ __forceinline__ T* panel_of(double* d) { return d; }

struct Shared {
  double red_v[32];
  int red_i[32];
  int red_c[32];
  double bcast_d[8];
  int bcast_i[8];
};

// Group barrier.  gen counts the barriers this CTA has passed.  It gives up
// after L.spin_limit polls (or once another CTA has raised the error word).
__device__ bool group_sync(const AcaLaunch& L, unsigned* bar, int G, unsigned& gen,
                           unsigned* err) {
  __syncthreads();
  if (G == 1) return true;
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_fail = 0;
    __threadfence();
    atomicAdd(bar, 1u);
    unsigned target = (gen + 1) * (unsigned)G + L.bar_extra;
    unsigned polls = 0;
    while (ld_acquire_u32(bar) < target) {
      if (++polls > L.spin_limit || *(volatile unsigned*)err) {
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

// One residual pass over a slice [lo, hi) of a panel P (column l at P + l*ld):
//   r[j] = entry(j) - sum_{l<k} coef[l] * P(j, l)     (l order, unfused: bit-exact)
//   written to P(j, k) * scale (scale = 1 for V, the pivot reciprocal for W),
// and, if `dots`, the per-warp partial dots  sum_j P(j, l) * P(j, k-1)  for
// l < k-1 accumulated into dotw[warp * ldd + l] (the norm update of step k-1,
// computed while the panel streams through for step k).  Returns the slice
// argmax of |r| (first maximum), the first admissible candidate (unchosen,
// |r| > minPiv) and the partial sum of squares of the stored column.
template <int NT, int E, bool ROW, typename T>
__device__ void residual_pass(const AcaLaunch& L, const AcaBlock& B, T* P, int lo, int hi,
                              int k, const double* __restrict__ coef, bool dots,
                              double* __restrict__ dotw, int ldd, int fixed, const double* xfix,
                              double scale, const unsigned char* chosen, double& bv, int& bi,
                              int& cand, double& sq, bool& nonfinite, const EntrySrc& S) {
  constexpr int U = 16 / E;  // panel columns per chunk: 16 loads in flight per thread
  const int64_t ld = L.ld;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const double minPiv = L.minPivot;
  const T* __restrict__ Pr = P;  // columns < k are only read here
  const int kd = dots ? k - 1 : 0;
  bool first = true;
  for (int jb = lo; jb < hi; jb += E * NT, first = false) {
    int jj[E];
    bool ok[E];
    double s[E], vp[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      jj[e] = jb + tid + e * NT;
      ok[e] = jj[e] < hi;
      if (!ok[e]) jj[e] = lo;  // safe address; its products use vp = 0
      s[e] = 0.0;
      vp[e] = (dots && ok[e]) ? (double)Pr[jj[e] + (int64_t)(k - 1) * ld] : 0.0;
    }
    int l = 0;
    for (; l + U <= k; l += U) {
      double v[U][E];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int e = 0; e < E; ++e) v[u][e] = (double)Pr[jj[e] + (int64_t)(l + u) * ld];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const double c = coef[l + u];
#pragma unroll
        for (int e = 0; e < E; ++e) s[e] = __dadd_rn(s[e], __dmul_rn(c, v[u][e]));
      }
      if (dots) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (l + u >= kd) break;
          double d = 0.0;
#pragma unroll
          for (int e = 0; e < E; ++e) d = fma(v[u][e], vp[e], d);
          d = warp_sum(d);
          if (lane == 0) {
            if (first)
              dotw[w * ldd + l + u] = d;
            else
              dotw[w * ldd + l + u] += d;
          }
        }
      }
    }
    for (; l < k; ++l) {
      const double c = coef[l];
      double d = 0.0;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const double v = (double)Pr[jj[e] + (int64_t)l * ld];
        s[e] = __dadd_rn(s[e], __dmul_rn(c, v));
        d = fma(v, vp[e], d);
      }
      if (dots && l < kd) {
        d = warp_sum(d);
        if (lane == 0) {
          if (first)
            dotw[w * ldd + l] = d;
          else
            dotw[w * ldd + l] += d;
        }
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if (!ok[e]) continue;
      const int j = jj[e];
      double ent = ROW ? src_entry_xi(S, xfix, fixed, B.c0 + j)
                       : src_entry_xj(S, xfix, B.r0 + j, fixed);
      double r = __dsub_rn(ent, s[e]);
      // the panel keeps the value rounded to its type (no rounding for FP64),
      // and the norms of the stopping test use what it keeps
      const T kept = (T)(ROW ? r : __dmul_rn(scale, r));
      const double stored = (double)kept;
      P[j + (int64_t)k * ld] = kept;
      sq = fma(stored, stored, sq);
      double a = fabs(r);
      nonfinite |= !isfinite(r);
      if (a > bv) {  // increasing j per thread: the first maximum
        bv = a;
        bi = j;
      }
      if (cand == INT_MAX && a > minPiv && __ldcg(chosen + j) == 0) cand = j;
    }
  }
}

// ---------------------------------------------------------------- bulk-copy rings
// With streaming on, the group levels run 16 warps per CTA, and every warp
// streams its own contiguous part of the CTA's slice through a private ring
// of WR_S stages in shared memory, each WR_BC panel columns x WR_ROWS rows,
// filled by cp.async.bulk copies (one per column) that complete on the
// stage's mbarrier.  Lane 0 refills a stage as soon as its own warp is done
// with it: no warp waits for another.  Rows start on an even global index so
// that every copy is 16-byte aligned (requires an even N).
constexpr int WR_NT = 512, WR_E = 4, WR_ROWS = 32 * WR_E;
constexpr int WR_BC = 4, WR_SMAX = 3;
constexpr int WR_NW = WR_NT / 32;
// ring bytes of one CTA with `stages` stages (192 KB with 3)
constexpr size_t wring_bytes(int stages) {
  return sizeof(double) * (size_t)WR_NW * stages * WR_BC * WR_ROWS;
}

struct WRing {
  // [warp][stage][column u][row], WR_ROWS rows per column: a warp's stages
  // are `stages` apart (wring_bytes(stages) in all), not WR_SMAX
  double* buf;
  uint64_t* full;   // [warp][stage]: the stage's copies landed (1 arrival + bytes)
  int stages;
  uint32_t t;       // tiles this warp has consumed (the same in all its lanes)
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase.  On giving up it raises DEV_ERR_TIMEOUT
// and returns; once the error word is set, later waits give up at once, so a
// failed launch ends quickly (its next group barrier fails).
__device__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned* err) {
  for (uint32_t polls = 0;; ++polls) {
    if (mbar_try(bar, parity)) return;
    if (polls >= (1u << 20) || (polls >= 64 && *(volatile unsigned*)err)) {
      atomicOr(err, DEV_ERR_TIMEOUT);
      return;
    }
    if (polls >= 64) __nanosleep(64);
  }
}

// Lane 0: this warp's tile number tw into its stage tw % stages -- `nc`
// columns from l0 of P, `count` rows from row0 (count even, row0 on an even
// global row).  The stage was last read by this warp before a __syncwarp;
// the proxy fence orders those reads before the copies overwrite it.
__device__ void wring_issue(WRing& R, int w, uint32_t tw, const double* P, int64_t ld, int row0,
                            int count, int l0, int nc) {
  const int slot = (int)(tw % (uint32_t)R.stages);
  uint64_t* bar = R.full + w * WR_SMAX + slot;
  const uint32_t bytes = (uint32_t)count * (uint32_t)sizeof(double);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes * (uint32_t)nc)
               : "memory");
  double* dst = R.buf + ((size_t)(w * R.stages + slot) * WR_BC) * WR_ROWS;
  for (int u = 0; u < nc; ++u)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst + u * WR_ROWS)),
        "l"(P + row0 + (int64_t)(l0 + u) * ld), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Lane 0: the same tile as wring_issue, as one 2D tensor copy of the whole
// box (WR_ROWS rows from arena row x, WR_BC columns from column y).  Rows or
// columns past the slice land in the stage unread (the consumer masks them);
// past the arena they are zero-filled, and the transaction always counts the
// full box.  x is even by construction (16-byte aligned start) and every
// stage starts on a 128-byte boundary (the ring heads dynamic shared memory,
// stages are 4 KB); a copy breaking either rule would be invalid, so it is
// refused: the stage completes without data and the launch reports
// DEV_ERR_INDEX.
__device__ void wring_issue_tile(WRing& R, int w, uint32_t tw, const CUtensorMap* map, int x,
                                 int y, unsigned* err) {
  const int slot = (int)(tw % (uint32_t)R.stages);
  uint64_t* bar = R.full + w * WR_SMAX + slot;
  double* dst = R.buf + ((size_t)(w * R.stages + slot) * WR_BC) * WR_ROWS;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if ((x & 1) || (smem_addr(dst) & 127u)) {
    atomicOr(err, DEV_ERR_INDEX);
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
    return;
  }
  constexpr uint32_t bytes = (uint32_t)(sizeof(double) * WR_ROWS * WR_BC);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// Lane 0, before the CTA exits: every copy this warp issued has landed.
// In normal flow each issued tile was waited for; a wait that gave up (an
// error raised elsewhere in the launch) can leave copies in flight, and the
// CTA's shared memory must not be released under them.  A stage's tiles
// complete in issue order, so waiting for the last tile of each stage (the
// last `stages` tiles) suffices; each wait is bounded.
__device__ void wring_drain(const WRing& R, int w) {
  const uint32_t t0 = R.t > (uint32_t)R.stages ? R.t - (uint32_t)R.stages : 0u;
  for (uint32_t tw = t0; tw < R.t; ++tw) {
    uint64_t* bar = R.full + w * WR_SMAX + (int)(tw % (uint32_t)R.stages);
    const uint32_t parity = (tw / (uint32_t)R.stages) & 1u;
    for (uint32_t polls = 0; polls < (1u << 20) && !mbar_try(bar, parity); ++polls)
      __nanosleep(64);
  }
}

// residual_pass with every warp streaming its own rows through its ring.
// gbase: the global row of P[0] (the block's first column for V, first row
// for W).  The same arithmetic as residual_pass, element for element: the
// residual sums in l order with separately rounded products and sums, the
// argmax in increasing index per thread; the fused dots add their partials
// in a GPU order, as there.
template <int NT, int E, bool ROW>
__device__ void residual_pass_wring(const AcaLaunch& L, const AcaBlock& B, double* P, int lo,
                                    int hi, int k, const double* __restrict__ coef, bool dots,
                                    double* __restrict__ dotw, int ldd, int fixed,
                                    const double* xfix, double scale, const unsigned char* chosen,
                                    double& bv, int& bi, int& cand, double& sq, bool& nonfinite,
                                    const EntrySrc& S, WRing& R, int gbase) {
  static_assert(NT == WR_NT && E == WR_E, "the warp ring's geometry");
  constexpr int NW = NT / 32;
  const int64_t ld = L.ld;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const double minPiv = L.minPivot;
  const int kd = dots ? k - 1 : 0;
  // this warp's rows: an even-sized share of the slice from an even global row
  const int x0 = lo - ((gbase + lo) & 1);
  int rw = (hi - x0 + NW - 1) / NW;
  rw = (rw + 1) & ~1;
  const int wlo = x0 + w * rw, whi = min(hi, wlo + rw);
  if (lo >= hi || wlo >= whi) {  // no rows: zero partial dots from this warp
    if (dots)
      for (int l = lane; l < kd; l += 32) dotw[w * ldd + l] = 0.0;
    return;
  }
  const int tpc = (k + WR_BC - 1) / WR_BC;  // tiles per chunk
  if (lane == 0) {
    // this warp's earlier generic stores to these rows, then the copies
    asm volatile("fence.proxy.async.global;" ::: "memory");
  }
  const CUtensorMap* map = ROW ? &L.map_v : &L.map_w;  // the arena P lies in (ring_tile)
  bool first = true;
  for (int jb = wlo; jb < whi; jb += WR_ROWS, first = false) {
    const int count = (min(WR_ROWS, whi - jb) + 1) & ~1;
    // lane 0: tile q of this chunk into the warp's stage for tile number tw
    auto issue = [&](uint32_t tw, int q) {
      if (L.ring_tile)
        wring_issue_tile(R, w, tw, map, gbase + jb, q * WR_BC, L.err);
      else
        wring_issue(R, w, tw, P, ld, jb, count, q * WR_BC, min(WR_BC, k - q * WR_BC));
    };
    if (lane == 0)
      for (int q = 0; q < tpc && q < R.stages; ++q) issue(R.t + q, q);
    int jj[E];
    bool ok[E];
    double s[E], vp[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      jj[e] = jb + lane + 32 * e;
      ok[e] = jj[e] >= lo && jj[e] < whi;
      s[e] = 0.0;
      vp[e] = (dots && ok[e]) ? P[jj[e] + (int64_t)(k - 1) * ld] : 0.0;
    }
    for (int q = 0; q < tpc; ++q) {
      const uint32_t tw = R.t + q;
      const int slot = (int)(tw % (uint32_t)R.stages);
      mbar_wait_bounded(R.full + w * WR_SMAX + slot, (tw / (uint32_t)R.stages) & 1, L.err);
      const double* tile = R.buf + ((size_t)(w * R.stages + slot) * WR_BC) * WR_ROWS;
      const int l0 = q * WR_BC, nc = min(WR_BC, k - l0);
      double v[WR_BC][E];
#pragma unroll
      for (int u = 0; u < WR_BC; ++u)
#pragma unroll
        for (int e = 0; e < E; ++e)
          v[u][e] = (u < nc && ok[e]) ? tile[u * WR_ROWS + lane + 32 * e] : 0.0;
#pragma unroll
      for (int u = 0; u < WR_BC; ++u) {
        if (u >= nc) break;
        const double cf = coef[l0 + u];
#pragma unroll
        for (int e = 0; e < E; ++e) s[e] = __dadd_rn(s[e], __dmul_rn(cf, v[u][e]));
      }
      if (dots && l0 < kd) {
        // the tile's four column dots over the warp in one transposed
        // reduction: after the exchanges at offsets 16 and 8, lane group
        // q = lane / 8 holds partial sums of column q, then each group of 8
        // lanes sums its own (6 shuffles instead of 4 x 5)
        static_assert(WR_BC == 4, "transposed reduction of four columns");
        double d[WR_BC];
#pragma unroll
        for (int u = 0; u < WR_BC; ++u) {
          d[u] = 0.0;
#pragma unroll
          for (int e = 0; e < E; ++e) d[u] = fma(v[u][e], vp[e], d[u]);
        }
        const bool hi16 = (lane & 16) != 0, hi8 = (lane & 8) != 0;
        const double s0 = __shfl_xor_sync(0xffffffffu, hi16 ? d[0] : d[2], 16);
        const double s1 = __shfl_xor_sync(0xffffffffu, hi16 ? d[1] : d[3], 16);
        const double p0 = (hi16 ? d[2] : d[0]) + s0;
        const double p1 = (hi16 ? d[3] : d[1]) + s1;
        const double s2 = __shfl_xor_sync(0xffffffffu, hi8 ? p0 : p1, 8);
        double t = (hi8 ? p1 : p0) + s2;
        t += __shfl_xor_sync(0xffffffffu, t, 4);
        t += __shfl_xor_sync(0xffffffffu, t, 2);
        t += __shfl_xor_sync(0xffffffffu, t, 1);
        const int u = (hi16 ? 2 : 0) + (hi8 ? 1 : 0);  // the column this lane group summed
        if ((lane & 7) == 0 && l0 + u < kd) {
          if (first)
            dotw[w * ldd + l0 + u] = t;
          else
            dotw[w * ldd + l0 + u] += t;
        }
      }
      __syncwarp();
      if (lane == 0 && q + R.stages < tpc) issue(tw + R.stages, q + R.stages);
    }
    R.t += tpc;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if (!ok[e]) continue;
      const int j = jj[e];
      double ent = ROW ? src_entry_xi(S, xfix, fixed, B.c0 + j)
                       : src_entry_xj(S, xfix, B.r0 + j, fixed);
      double r = __dsub_rn(ent, s[e]);
      const double stored = ROW ? r : __dmul_rn(scale, r);
      P[j + (int64_t)k * ld] = stored;
      sq = fma(stored, stored, sq);
      double a = fabs(r);
      nonfinite |= !isfinite(r);
      if (a > bv) {
        bv = a;
        bi = j;
      }
      if (cand == INT_MAX && a > minPiv && __ldcg(chosen + j) == 0) cand = j;
    }
  }
}

// Partial dots of step k-1 over this CTA's slices when they could not be
// fused into a residual pass (a zero residual row, or the capacity limit).
template <int NT, typename T>
__device__ void dots_only_pass(const AcaLaunch& L, const T* BW, const T* BV, int k, int i_lo,
                               int i_hi, int j_lo, int j_hi, int kcap, double* bank) {
  const int64_t ld = L.ld;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T* wk = BW + (int64_t)(k - 1) * ld;
  const T* vk = BV + (int64_t)(k - 1) * ld;
  for (int l = w; l < k - 1; l += NT / 32) {
    const T* wl = BW + (int64_t)l * ld;
    const T* vl = BV + (int64_t)l * ld;
    double aw = 0.0, av = 0.0;
    for (int i = i_lo + lane; i < i_hi; i += 32) aw = fma((double)wk[i], (double)wl[i], aw);
    for (int j = j_lo + lane; j < j_hi; j += 32) av = fma((double)vl[j], (double)vk[j], av);
    aw = warp_sum(aw);
    av = warp_sum(av);
    if (lane == 0) {
      bank[l] = av;
      bank[kcap + l] = aw;
    }
  }
}

// epsilon of step k-1 from the G partial dots in the bank at offset bk
// (dotV at bk, dotW at bk + kcap):
// frobNormSq += 2 sum_l (w.W_l)(V_l.v) + |w|^2 |v|^2  (src/lowRank.cpp:234-241)
template <int NT>
__device__ double resolve_eps(Shared& sh, const AcaLaunch& L, const AcaBlock& B,
                              const double* part_grp, int G, int bk, int k, double swp,
                              double svp, double& frob2) {
  double sum_local = 0.0;
  for (int l = threadIdx.x; l < k - 1; l += NT) {
    double dv = 0.0, dw = 0.0;
    for (int q = 0; q < G; ++q) {
      dv += __ldcg(part_grp + q * L.part_stride + bk + l);
      dw += __ldcg(part_grp + q * L.part_stride + bk + B.kcap + l);
    }
    sum_local += dw * dv;
  }
  const double sumNorm = block_sum<NT>(sh, sum_local);
  frob2 += 2 * sumNorm + swp * svp;
  return sqrt(swp) * sqrt(svp) / sqrt(frob2);
}

// RING: the residual passes stream their panel slices through the warps'
// bulk-copy rings (group levels of an even N, 512 threads); the dynamic
// shared memory then starts with the rings' wring_bytes(L.ring_stages).
// T: the element type of the W/V panels (double).
template <int NT, int E, bool RING, typename T>
__global__ void __launch_bounds__(NT, (NT == 512 ? 1 : NT == 256 ? 2 : 4)) aca_kernel(const __grid_constant__ AcaLaunch L) {
  extern __shared__ __align__(128) double dyn_all[];
  __shared__ Shared sh;
  __shared__ __align__(8) uint64_t ring_full[RING ? WR_NW * WR_SMAX : 1];
  double* dyn = RING ? dyn_all + wring_bytes(L.ring_stages) / sizeof(double) : dyn_all;
  // dyn: row[kcap], then (unless L.dotg) per-warp dots[NT/32][kcap]
  constexpr int NW = NT / 32;
  const int b = L.cta_block ? (blockIdx.x < (unsigned)L.ncta ? L.cta_block[blockIdx.x] : L.nblocks)
                            : (int)(blockIdx.x / L.G);
  const int tid = threadIdx.x;
  if (b >= L.nblocks) return;
  const AcaBlock B = L.blocks[b];
  T* const BW = panel_of<T>(B.W);
  T* const BV = panel_of<T>(B.V);
  const int G = L.cta_block ? B.G : L.G;
  const int g = L.cta_block ? (int)blockIdx.x - B.g0 : (int)(blockIdx.x % L.G);
  const int64_t grp0 = L.cta_block ? B.g0 : (int64_t)b * G;
  AcaState* st = B.st;
  if (st->status != ACA_RUNNING && st->status != ACA_POST) return;
  const EntrySrc S = src_for(L.src, B.r0);  // the kernel of this block's system

  const int64_t ld = L.ld;
  const int m = B.m, n = B.n, ub = min(m, n);
  const double tol = L.tol, minPiv = L.minPivot;
  double* row = dyn;
  // per-warp dot partials: shared memory, or for large ranks this CTA's
  // slice of global memory (same writers and order: only the footprint moves)
  double* dotw = L.dotg ? L.dotg + (int64_t)blockIdx.x * L.dotg_stride : dyn + L.kcap_max;
  const int ldd = L.kcap_max;
  double* part_me = L.part + (int64_t)blockIdx.x * L.part_stride;
  const double* part_grp = L.part + grp0 * L.part_stride;
  unsigned* bar = L.bar + b;
  unsigned gen = 0;

  const int sm = (m + G - 1) / G, sn = (n + G - 1) / G;
  const int i_lo = min(m, g * sm), i_hi = min(m, i_lo + sm);
  const int j_lo = min(n, g * sn), j_hi = min(n, j_lo + sn);

  int k = st->k, cur = st->cur, iters = st->iters, status = st->status;
  double frob2 = st->frob2, eps = st->eps, margin = st->margin;
  double swp = st->swp, svp = st->svp;
  int near = st->near, pending = st->pending;
  bool nonfinite = false;
  WRing ring{dyn_all, ring_full, L.ring_stages, 0};
  if (RING) {
    if (tid == 0) {
      for (int q = 0; q < WR_NW * WR_SMAX; ++q)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&ring_full[q])));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }

  const int minR = B.minRank, maxR = B.maxRank;  // -1: none (src/lowRank.cpp:149,244-247)
  if (status == ACA_RUNNING && k == 0 && maxR == 0) status = ACA_POST;  // zero columns, rank 1
  auto note_margin = [&](int kcount) {
    if (kcount < ub && kcount >= minR) {
      double gap = fabs(eps - tol) / tol;
      margin = fmin(margin, gap);
      if (gap < 1e-10) ++near;
    }
  };

  while (status == ACA_RUNNING) {
    // loop test of the reference, with epsilon_{k-1} possibly still pending
    if (!pending && !(eps > tol) && k >= minR) { status = ACA_POST; break; }
    if (k >= ub) { status = ACA_POST; break; }
    if (k >= B.kcap) {
      if (pending) {
        const int bk0 = 8 + (k & 1) * (2 * B.kcap + 2);
        dots_only_pass<NT>(L, BW, BV, k, i_lo, i_hi, j_lo, j_hi, B.kcap, part_me + bk0);
        if (!group_sync(L, bar, G, gen, L.err)) { status = ACA_ERROR; break; }
        eps = resolve_eps<NT>(sh, L, B, part_grp, G, bk0, k, swp, svp, frob2);
        pending = 0;
        note_margin(k);
        if (!group_sync(L, bar, G, gen, L.err)) { status = ACA_ERROR; break; }
        if (!(eps > tol) && k >= minR) { status = ACA_POST; break; }
      }
      status = ACA_NEED_CAP;  // paused: the host grows the capacity and resumes
      break;
    }
    ++iters;
    const bool fuse = pending && k >= 2;
    // Dot and norm partials alternate between two banks by step parity: a
    // slow CTA may still read step k-1's bank in its phase C while a fast one
    // already writes step k's in phase A.
    const int bk = 8 + (k & 1) * (2 * B.kcap + 2);
    // ---------------- phase A: residual row on this CTA's column slice
    if (g == 0 && tid == 0) B.cR[cur] = 1;
    for (int l = tid; l < k; l += NT) row[l] = (double)__ldcg(BW + cur + (int64_t)l * ld);
    if (fuse && j_lo >= j_hi)  // an empty slice contributes zero dots
      for (int e = tid; e < NW * (k - 1); e += NT) dotw[(e / (k - 1)) * ldd + e % (k - 1)] = 0.0;
    __syncthreads();
    const int gi = B.r0 + cur;
    double xi[3] = {0.0, 0.0, 0.0};
    if (!S.dense) {
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < S.kp.dim) xi[d] = __ldg(S.pts + d * S.ld + gi);
    }
    double bv = -1.0, sv = 0.0;
    int bi = INT_MAX, cand = INT_MAX;
    if constexpr (RING)
      residual_pass_wring<NT, E, true>(L, B, BV, j_lo, j_hi, k, row, fuse, dotw, ldd, gi, xi,
                                       1.0, B.cC, bv, bi, cand, sv, nonfinite, S, ring, B.c0);
    else
      residual_pass<NT, E, true>(L, B, BV, j_lo, j_hi, k, row, fuse, dotw, ldd, gi, xi, 1.0,
                                 B.cC, bv, bi, cand, sv, nonfinite, S);
    __syncthreads();
    if (fuse)  // CTA partial dots of V, warps summed in order
      for (int l = tid; l < k - 1; l += NT) {
        double t = 0.0;
        for (int q = 0; q < NW; ++q) t += dotw[q * ldd + l];
        part_me[bk + l] = t;
      }
    block_argmax<NT>(sh, bv, bi);
    cand = block_min_int<NT>(sh, cand);
    sv = block_sum<NT>(sh, sv);
    if (tid == 0) {
      part_me[0] = bv;
      part_me[1] = (double)bi;
      part_me[2] = (bi != INT_MAX) ? (double)__ldcg(B.cC + bi) : 0.0;
      part_me[3] = (double)cand;
      part_me[bk + 2 * B.kcap + 1] = sv;
    }
    if (!group_sync(L, bar, G, gen, L.err)) { status = ACA_ERROR; break; }

    // ---------------- phase B: pivot column, residual column on the row slice
    double mv;
    int mi, mflag, mcand;
    reduce_partials(sh, part_grp, L.part_stride, G, 0, mv, mi, mflag, mcand);
    if (mv <= minPiv) {
      // zero residual row (src/lowRank.cpp:187-195).  Whether the reference
      // even reached this step depends on epsilon_{k-1}: settle it first.
      if (pending) {
        dots_only_pass<NT>(L, BW, BV, k, i_lo, i_hi, j_lo, j_hi, B.kcap, part_me + bk);
        if (!group_sync(L, bar, G, gen, L.err)) { status = ACA_ERROR; break; }
        eps = resolve_eps<NT>(sh, L, B, part_grp, G, bk, k, swp, svp, frob2);
        pending = 0;
        note_margin(k);
        if (!(eps > tol) && k >= minR) {
          --iters;
          status = ACA_POST;
          break;
        }
      }
      int f = INT_MAX;
      for (int i = tid; i < m; i += NT)
        if (__ldcg(B.cR + i) == 0) { f = i; break; }
      f = block_min_int<NT>(sh, f);
      if (f == INT_MAX) { status = ACA_POST; break; }
      cur = f;
      if (!group_sync(L, bar, G, gen, L.err)) { status = ACA_ERROR; break; }
      continue;
    }
    int cc;
    if (!mflag) {
      cc = mi;
    } else {
      // whichever way epsilon_{k-1} goes, the rank is k (src/lowRank.cpp:200-202)
      if (mcand == INT_MAX) { status = ACA_POST; break; }
      cc = mcand;
    }
    if (g == 0 && tid == 0) B.cC[cc] = 1;
    const double piv = __ddiv_rn(1.0, (double)__ldcg(BV + cc + (int64_t)k * ld));
    for (int l = tid; l < k; l += NT) row[l] = (double)__ldcg(BV + cc + (int64_t)l * ld);
    if (fuse && i_lo >= i_hi)
      for (int e = tid; e < NW * (k - 1); e += NT) dotw[(e / (k - 1)) * ldd + e % (k - 1)] = 0.0;
    __syncthreads();
    const int gj = B.c0 + cc;
    double xj[3] = {0.0, 0.0, 0.0};
    if (!S.dense) {
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < S.kp.dim) xj[d] = __ldg(S.pts + d * S.ld + gj);
    }
    bv = -1.0;
    bi = INT_MAX;
    cand = INT_MAX;
    double sw = 0.0;
    if constexpr (RING)
      residual_pass_wring<NT, E, false>(L, B, BW, i_lo, i_hi, k, row, fuse, dotw, ldd, gj, xj,
                                        piv, B.cR, bv, bi, cand, sw, nonfinite, S, ring, B.r0);
    else
      residual_pass<NT, E, false>(L, B, BW, i_lo, i_hi, k, row, fuse, dotw, ldd, gj, xj, piv,
                                  B.cR, bv, bi, cand, sw, nonfinite, S);
    __syncthreads();
    if (fuse)
      for (int l = tid; l < k - 1; l += NT) {
        double t = 0.0;
        for (int q = 0; q < NW; ++q) t += dotw[q * ldd + l];
        part_me[bk + B.kcap + l] = t;
      }
    block_argmax<NT>(sh, bv, bi);
    cand = block_min_int<NT>(sh, cand);
    sw = block_sum<NT>(sh, sw);
    if (tid == 0) {
      part_me[4] = bv;
      part_me[5] = (double)bi;
      part_me[6] = (bi != INT_MAX) ? (double)__ldcg(B.cR + bi) : 0.0;
      part_me[7] = (double)cand;
      part_me[bk + 2 * B.kcap] = sw;
    }
    if (!group_sync(L, bar, G, gen, L.err)) { status = ACA_ERROR; break; }

    // ---------------- phase C: epsilon of step k-1, then step k's next row
    if (pending) {
      eps = fuse ? resolve_eps<NT>(sh, L, B, part_grp, G, bk, k, swp, svp, frob2)
                 : [&]() {  // k == 1: no earlier columns, the dots are empty
                     frob2 += swp * svp;
                     return sqrt(swp) * sqrt(svp) / sqrt(frob2);
                   }();
      pending = 0;
      note_margin(k);
      if (!(eps > tol) && k >= minR) {  // step k is discarded: the reference stopped before it
        --iters;
        status = ACA_POST;
        break;
      }
    }
    int nflag, ncand, ni;
    double nv;
    reduce_partials(sh, part_grp, L.part_stride, G, 4, nv, ni, nflag, ncand);
    const int nr = nflag ? ncand : ni;
    if (nr == INT_MAX) {  // no admissible next row: stop before storing (src/lowRank.cpp:226-227)
      status = ACA_POST;
      break;
    }
    double swt = 0.0, svt = 0.0;
    for (int q = 0; q < G; ++q) {
      swt += __ldcg(part_grp + q * L.part_stride + bk + 2 * B.kcap);
      svt += __ldcg(part_grp + q * L.part_stride + bk + 2 * B.kcap + 1);
    }
    if (g == 0 && tid == 0) {
      B.prow[k] = cur;
      B.pcol[k] = cc;
    }
    swp = swt;
    svp = svt;
    pending = 1;
    cur = nr;
    ++k;
    if (k == maxR) {  // the rank ceiling: stop without the last epsilon (src/lowRank.cpp:244-247)
      pending = 0;
      status = ACA_POST;
      break;
    }
    // No barrier needed here: the next writes to the partials come after
    // every CTA has passed barrier 2, and W(:,k) / V(:,k) are final.
  }

  // ---------------- post-processing (src/lowRank.cpp:250-277)
  int rank = k;
  if (status == ACA_POST) {
    if (k == 0) {
      for (int i = i_lo + tid; i < i_hi; i += NT) BW[i] = (T)0;
      for (int j = j_lo + tid; j < j_hi; j += NT) BV[j] = (T)0;
      rank = 1;
      status = ACA_DONE;
    } else if (k >= ub - 1) {
      const int full = (n <= m) ? n : m;
      if (B.kcap < full) {
        status = ACA_NEED_CAP_POST;  // the full representation needs more columns
        rank = full;
      } else if (n <= m) {  // W = block (m x n), V = I_n
        for (int l = 0; l < n; ++l) {
          double xc[3] = {0.0, 0.0, 0.0};
          if (!S.dense) {
#pragma unroll
            for (int d = 0; d < 3; ++d)
              if (d < S.kp.dim) xc[d] = __ldg(S.pts + d * S.ld + B.c0 + l);
          }
          for (int i = i_lo + tid; i < i_hi; i += NT)
            BW[i + (int64_t)l * ld] = (T)src_entry_xj(S, xc, B.r0 + i, B.c0 + l);
          for (int j = j_lo + tid; j < j_hi; j += NT)
            BV[j + (int64_t)l * ld] = (T)((j == l) ? 1.0 : 0.0);
        }
        rank = n;
        status = ACA_DONE;
      } else {  // W = I_m, V = block^T (n x m)
        for (int l = 0; l < m; ++l) {
          double xr[3] = {0.0, 0.0, 0.0};
          if (!S.dense) {
#pragma unroll
            for (int d = 0; d < 3; ++d)
              if (d < S.kp.dim) xr[d] = __ldg(S.pts + d * S.ld + B.r0 + l);
          }
          for (int j = j_lo + tid; j < j_hi; j += NT)
            BV[j + (int64_t)l * ld] = (T)src_entry_xi(S, xr, B.r0 + l, B.c0 + j);
          for (int i = i_lo + tid; i < i_hi; i += NT)
            BW[i + (int64_t)l * ld] = (T)((i == l) ? 1.0 : 0.0);
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
  if (status != ACA_ERROR && !group_sync(L, bar, G, gen, L.err)) status = ACA_ERROR;
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
    st->swp = swp;
    st->svp = svp;
    st->pending = pending;
  }
  if constexpr (RING)
    if ((tid & 31) == 0) wring_drain(ring, tid >> 5);
}

}  // namespace

// Stages of the warp rings that fit beside kcap_max row coefficients (the
// ring's dots are always in global memory): 3, 2, or 0 (no ring).
int aca_ring_stages(int kcap_max) {
  for (int st = WR_SMAX; st >= 2; --st)
    if (wring_bytes(st) + sizeof(double) * (size_t)kcap_max <= 224 * 1024) return st;
  return 0;
}

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it.
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// A 2D map over an n x kcap column-major arena (leading dimension n) whose
// box is one ring tile: WR_ROWS rows by WR_BC columns.  The copy's start row
// must give a 16-byte aligned address; the kernel keeps it even.
bool panel_map(CUtensorMap* m, const double* base, int64_t n, int kcap) {
  EncodeTiledFn f = encode_tiled();
  if (!f || !base || ((uintptr_t)base & 15) || (n & 1) || n <= 0 || kcap <= 0) return false;
  const cuuint64_t dim[2] = {(cuuint64_t)n, (cuuint64_t)kcap};
  const cuuint64_t stride[1] = {(cuuint64_t)n * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)WR_ROWS, (cuuint32_t)WR_BC};
  const cuuint32_t elem[2] = {1, 1};
  return f(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dim, stride, box,
           elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// The launch's W and V maps for one tensor copy per ring tile; false (and
// the per-column copies) when either cannot be encoded.
bool aca_ring_tile_maps(AcaLaunch& L, const double* W, const double* V, int64_t n, int kcap) {
  return panel_map(&L.map_w, W, n, kcap) && panel_map(&L.map_v, V, n, kcap);
}

static size_t aca_smem(int nt, int kcap_max, bool global_dots, bool ring, bool f32) {
  (void)f32;
  return (ring ? wring_bytes(aca_ring_stages(kcap_max)) : 0) +
         sizeof(double) * (size_t)(global_dots ? 1 : 1 + nt / 32) * (size_t)kcap_max;
}

// The per-warp dot partials move to global memory once the CTA's shared
// memory would pass 100 KB (beyond that fewer than two 256-thread CTAs fit on
// an SM), and always with the warp rings (their stages fill shared memory).
bool aca_dots_global(int nt, int kcap_max, bool ring, bool f32) {
  return ring || aca_smem(nt, kcap_max, false, false, f32) > 100 * 1024;
}

size_t aca_smem_bytes(int nt, int kcap_max, bool ring, bool f32) {
  return aca_smem(nt, kcap_max, aca_dots_global(nt, kcap_max, ring, f32), ring, f32);
}

template <typename T>
static void* aca_fn_t(int nt, bool ring, bool narrow) {
  if (ring) return (void*)aca_kernel<WR_NT, WR_E, true, T>;
  if (nt == 256)
    return narrow ? (void*)aca_kernel<256, 2, false, T> : (void*)aca_kernel<256, 4, false, T>;
  return (void*)aca_kernel<128, 2, false, T>;
}

static void* aca_fn(int nt, bool ring, bool f32, bool narrow = false) {
  (void)f32;  // FP64 panels only
  return aca_fn_t<double>(nt, ring, narrow);
}

// Dynamic shared memory above 48 KB.  The ring kernels (160+ KB per CTA)
// also ask for the largest shared-memory carveout, so that the occupancy
// query sizing their cooperative launch and the launch see the same
// capacity; the others keep the default split and its larger L1 for their
// per-thread panel loads.
static int set_smem(void* fn, size_t smem, bool ring) {
  cudaError_t e = cudaSuccess;
  if (ring)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) e = smem_opt_in(fn, smem);
  if (e != cudaSuccess) cudaGetLastError();  // consume it: later launch checks stay clean
  return (int)e;
}

int aca_launch(const AcaLaunch& L, int nt, int kcap_max, bool cooperative, cudaStream_t s) {
  const bool ring = L.ring != 0, f32 = false;
  if (ring && (nt != WR_NT || (L.ld % 2) || L.ring_stages != aca_ring_stages(kcap_max) ||
               L.ring_stages < 2))
    return (int)cudaErrorInvalidValue;
  const size_t smem = aca_smem(nt, kcap_max, L.dotg != nullptr, ring, f32);
  dim3 grid(L.cta_block ? L.ncta : L.nblocks * L.G), block(nt);
  void* args[] = {(void*)&L};
  void* fn = aca_fn(nt, ring, f32, L.narrow != 0);
  if (int e = set_smem(fn, smem, ring)) return e;
  cudaError_t e = cooperative ? cudaLaunchCooperativeKernel(fn, grid, block, args, smem, s)
                              : cudaLaunchKernel(fn, grid, block, args, smem, s);
  if (e != cudaSuccess) cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

int aca_max_coresident(int nt, int kcap_max, bool ring, bool f32, int* per_sm) {
  const size_t smem = aca_smem_bytes(nt, kcap_max, ring, f32);
  void* fn = aca_fn(nt, ring, f32);
  *per_sm = 0;
  if (int e = set_smem(fn, smem, ring)) return e;
  int nb = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, nt, smem);
  if (e != cudaSuccess) cudaGetLastError();
  *per_sm = nb;
  return e == cudaSuccess ? 0 : (int)e;
}
