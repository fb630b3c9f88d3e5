// Grouped batched GEMMs on the 5th-generation tensor cores (tcgen05) for the
// mixed-precision form of the Woodbury products:
//   TN:     C (M x N)  = A^T B      A is K x M, B is K x N
//   NN-sub: C (M x N) -= A B        A is M x K, B is K x N
// (the same problems as gemm.cu, src/HODLR_Matrix.cpp:672-687, 743-750).
// Operands stay FP64 in HBM; each CTA converts its tiles to BF16 or TF32 while
// staging them into shared memory in the canonical K-major layout, one thread
// issues tcgen05.mma with the accumulator in tensor memory (FP32), and the
// epilogue reads it back with tcgen05.ld and writes / subtracts FP64.
//
// CTA tile 128 x 64, K in stages of 64 (32 for 3xTF32), two stage buffers: the MMAs of one
// stage run while the threads stage the next; an mbarrier signalled by
// tcgen05.commit tells when a buffer may be overwritten.  Every wait is
// bounded; on a timeout the kernel records DEV_ERR_TIMEOUT, waits (bounded)
// for its own MMAs, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "gemm.h"

namespace {

constexpr int UM = 128;   // tile rows (= TMEM lanes)
constexpr int UN = 64;    // tile columns (= TMEM columns, fp32)
constexpr int UNT = 128;  // 4 warps: one per TMEM lane quarter
constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ float to_tf32(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return __uint_as_float(r);
}

// Operand formats.  `parts` = 2 splits each operand into a TF32 head and a
// TF32 tail (x = hi + lo); the product is hi*hi + hi*lo + lo*hi, which keeps
// about FP32 accuracy (the error-compensated "3xTF32" scheme).
template <int PREC>
struct Fmt;
template <>
struct Fmt<HODLR_GEMM_BF16> {  // kind::f16 with BF16 operands
  using T = __nv_bfloat16;
  static constexpr int per16 = 8;  // elements per 16-byte chunk
  static constexpr int mmak = 16;  // K of one MMA
  static constexpr int uk = 64;    // K per stage
  static constexpr int parts = 1;
  static constexpr uint32_t code = 1;
  static __device__ __forceinline__ void cvt(double x, T* hi, T* lo) {
    *hi = __double2bfloat16(x);
    (void)lo;
  }
};
template <>
struct Fmt<HODLR_GEMM_TF32> {  // kind::tf32, fp32 storage rounded to tf32
  using T = float;
  static constexpr int per16 = 4;
  static constexpr int mmak = 8;
  static constexpr int uk = 64;
  static constexpr int parts = 1;
  static constexpr uint32_t code = 2;
  static __device__ __forceinline__ void cvt(double x, T* hi, T* lo) {
    *hi = to_tf32((float)x);
    (void)lo;
  }
};
template <>
struct Fmt<HODLR_GEMM_TF32X3> {
  using T = float;
  static constexpr int per16 = 4;
  static constexpr int mmak = 8;
  static constexpr int uk = 32;
  static constexpr int parts = 2;
  static constexpr uint32_t code = 2;
  static __device__ __forceinline__ void cvt(double x, T* hi, T* lo) {
    const float h = to_tf32((float)x);
    *hi = h;
    *lo = to_tf32((float)(x - (double)h));
  }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: no swizzle, K-major canonical layout
// ((8 rows, m groups), (2 chunks)) : ((16 B, SBO), LBO), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Stage rows [r0, r0+R) x k [k0, k0+uk) of an operand into a K-major tile
// (and, for split formats, its tail into tile + R * uk elements).
// KCONTIG: element (r, k) at src[k + r * ld]; else at src[r + k * ld].
template <int PREC, int R, bool KCONTIG>
__device__ __forceinline__ void stage_tile(uint8_t* tile, const double* __restrict__ src,
                                           int64_t ld, int r0, int rlim, int k0, int klim) {
  using F = Fmt<PREC>;
  using T = typename F::T;
  constexpr int UK = F::uk;
  constexpr int CPR = UK / F::per16;  // chunks per row
  constexpr int SBO = CPR * 128;
  constexpr int TASKS = R * CPR;
  constexpr int PART_BYTES = R * UK * (int)sizeof(T);
  for (int q = threadIdx.x; q < TASKS; q += UNT) {
    int r, c;
    if (KCONTIG) {  // a warp covers whole rows: contiguous k in memory
      r = q / CPR;
      c = q % CPR;
    } else {  // a warp covers consecutive rows: contiguous r in memory
      r = q % R;
      c = q / R;
    }
    const int gr = r0 + r;
    alignas(16) T v[F::per16];
    alignas(16) T w[F::per16];
#pragma unroll
    for (int e = 0; e < F::per16; ++e) {
      const int gk = k0 + c * F::per16 + e;
      double x = 0.0;
      if (gr < rlim && gk < klim) x = KCONTIG ? src[gk + (int64_t)gr * ld] : src[gr + (int64_t)gk * ld];
      F::cvt(x, &v[e], &w[e]);
    }
    uint8_t* dst = tile + (r >> 3) * SBO + c * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
    if (F::parts == 2) *reinterpret_cast<uint4*>(dst + PART_BYTES) = *reinterpret_cast<const uint4*>(w);
  }
}

template <int PREC, bool TRANS_A, int MODE>
__global__ void __launch_bounds__(UNT) umma_gemm_kernel(const GemmProblem* __restrict__ probs,
                                                         const int4* __restrict__ tiles,
                                                         double* __restrict__ ws, unsigned* err) {
  using F = Fmt<PREC>;
  constexpr int UK = F::uk;
  constexpr int CPR = UK / F::per16;
  constexpr int SBO = CPR * 128;
  constexpr int A_PART = UM * UK * (int)sizeof(typename F::T);
  constexpr int B_PART = UN * UK * (int)sizeof(typename F::T);
  constexpr int A_BYTES = A_PART * F::parts;
  constexpr int B_BYTES = B_PART * F::parts;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail;

  const int4 t = tiles[blockIdx.x];
  const GemmProblem P = probs[t.x];
  const int m0 = t.y * UM, n0 = t.z * UN;
  const int kchunk = P.kchunk > 0 ? P.kchunk : P.K;
  const int kb = t.w * kchunk, ke = min(P.K, kb + kchunk);
  const int nstages = ke > kb ? (ke - kb + UK - 1) / UK : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_slot)), "r"(UN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = (1u << 4) | (F::code << 7) | (F::code << 10) | ((uint32_t)(UN >> 3) << 17) |
                         ((uint32_t)(UM >> 4) << 24);

  int issued = 0;  // stages whose MMAs were issued (thread 0)
  for (int s = 0; s < nstages; ++s) {
    const int buf = s & 1;
    uint8_t* A_s = smem + buf * (A_BYTES + B_BYTES);
    uint8_t* B_s = A_s + A_BYTES;
    if (s >= 2) {  // the MMAs of stage s-2 must be done reading this buffer
      if (threadIdx.x == 0 && !mbar_wait(&mbar[buf], ((s - 2) >> 1) & 1)) s_fail = 1;
      __syncthreads();
      if (s_fail) break;
    }
    const int k0 = kb + s * UK;
    // A tile: rows = output rows m (A^T for TN: element (m,k) = A[k + m*lda])
    stage_tile<PREC, UM, TRANS_A>(A_s, P.A, P.lda, m0, P.M, k0, ke);
    // B tile: rows = output columns n, element (n,k) = B[k + n*ldb]
    stage_tile<PREC, UN, true>(B_s, P.B, P.ldb, n0, P.N, k0, ke);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(A_s), b0 = smem_u32(B_s);
#pragma unroll
      for (int kk = 0; kk < UK / F::mmak; ++kk) {
        // (head, head), then for split formats (head, tail), (tail, head)
#pragma unroll
        for (int pp = 0; pp < (F::parts == 2 ? 3 : 1); ++pp) {
          const uint32_t ao = (pp == 2) ? A_PART : 0u, bo = (pp == 1) ? B_PART : 0u;
          const uint64_t ad = smem_desc(a0 + ao + kk * 256, 128, SBO);
          const uint64_t bd = smem_desc(b0 + bo + kk * 256, 128, SBO);
          const uint32_t accum = (s > 0 || kk > 0 || pp > 0) ? 1u : 0u;
          if (PREC == HODLR_GEMM_BF16)
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u),
                "r"(0u));
          else
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u),
                "r"(0u));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(smem_u32(&mbar[buf])));
      ++issued;
    }
  }
  // all MMAs done (also after a timeout: never free tensor memory that MMAs
  // still write): wait, bounded, on the commit of the last stage issued
  if (threadIdx.x == 0 && issued > 0) {
    const int last = issued - 1;
    if (!mbar_wait(&mbar[last & 1], (last >> 1) & 1)) s_fail = 1;
  }
  __syncthreads();
  const bool ok = !s_fail;
  if (!ok && threadIdx.x == 0) atomicOr(err, DEV_ERR_TIMEOUT);
  asm volatile("tcgen05.fence::after_thread_sync;");
  // epilogue: thread = output row; 64 columns in four loads of 16
  const int row = warp * 32 + lane;
  const int gm = m0 + row;
  if (ok) {
#pragma unroll
    for (int c4 = 0; c4 < UN / 16; ++c4) {
      uint32_t r[16];
      if (nstages > 0) {
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c4 * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = 0u;
      }
      if (gm < P.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int gn = n0 + c4 * 16 + j;
          if (gn >= P.N) continue;
          const double v = (double)__uint_as_float(r[j]);
          if (MODE == 1) {
            double* c = P.C + (int64_t)gn * P.ldc + gm;
            *c = *c - v;
          } else if (P.splits > 1) {
            ws[P.ws_off + ((int64_t)t.w * P.N + gn) * P.M + gm] = v;
          } else {
            P.C[(int64_t)gn * P.ldc + gm] = v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UN));
}

template <int PREC, bool TRANS_A, int MODE>
int launch_umma(const GemmProblem* probs, const int4* tiles, int ntiles, double* ws, unsigned* err,
                cudaStream_t s) {
  using F = Fmt<PREC>;
  const size_t smem = 2 * (size_t)(UM + UN) * F::uk * sizeof(typename F::T) * F::parts;
  auto fn = umma_gemm_kernel<PREC, TRANS_A, MODE>;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  fn<<<ntiles, UNT, smem, s>>>(probs, tiles, ws, err);
  return (int)cudaGetLastError();
}

__global__ void umma_splitk_reduce(const GemmProblem* __restrict__ probs, const double* __restrict__ ws) {
  const GemmProblem P = probs[blockIdx.y];
  if (P.splits <= 1) return;
  const int64_t total = (int64_t)P.M * P.N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < P.splits; ++q) s += ws[P.ws_off + q * total + e];
    P.C[(int64_t)(e / P.M) * P.ldc + (e % P.M)] = s;
  }
}

}  // namespace

constexpr int UMMA_MAX_KCHUNK = 4096;

void umma_plan(std::vector<GemmProblem>& probs, std::vector<int4>& tiles, int64_t& ws_elems,
               bool allow_split, int target_ctas) {
  tiles.clear();
  ws_elems = 0;
  int64_t mn_tiles = 0;
  for (auto& p : probs) mn_tiles += (int64_t)((p.M + UM - 1) / UM) * ((p.N + UN - 1) / UN);
  for (size_t q = 0; q < probs.size(); ++q) {
    GemmProblem& p = probs[q];
    p.splits = 1;
    p.kchunk = 0;
    if (p.M <= 0 || p.N <= 0 || p.K <= 0) continue;
    const int tm = (p.M + UM - 1) / UM, tn = (p.N + UN - 1) / UN;
    int splits = 1;
    if (allow_split && mn_tiles < target_ctas) {
      int want = (int)((target_ctas + mn_tiles - 1) / std::max<int64_t>(mn_tiles, 1));
      splits = std::max(1, std::min(want, p.K / 1024));
    }
    // FP32 accumulation in TMEM over at most UMMA_MAX_KCHUNK terms; longer
    // reductions (V^T Y over the rows of a top node) are split and their
    // partial tiles summed in FP64, so the accumulation error stays at the
    // level of a few thousand FP32 additions whatever the node size
    if (allow_split) splits = std::max(splits, (p.K + UMMA_MAX_KCHUNK - 1) / UMMA_MAX_KCHUNK);
    int kchunk = (p.K + splits - 1) / splits;
    kchunk = ((kchunk + 63) / 64) * 64;
    splits = (p.K + kchunk - 1) / kchunk;
    p.splits = splits;
    p.kchunk = splits > 1 ? kchunk : 0;
    if (splits > 1) {
      p.ws_off = ws_elems;
      ws_elems += (int64_t)splits * p.M * p.N;
    }
    for (int ks = 0; ks < splits; ++ks)
      for (int j = 0; j < tn; ++j)
        for (int i = 0; i < tm; ++i) tiles.push_back(make_int4((int)q, i, j, ks));
  }
}

int umma_tn_launch(int prec, const GemmProblem* d_probs, const int4* d_tiles, int ntiles, int nprob,
                   double* d_ws, bool any_split, unsigned* err, cudaStream_t s) {
  if (ntiles == 0) return 0;
  int e = prec == HODLR_GEMM_BF16
              ? launch_umma<HODLR_GEMM_BF16, true, 0>(d_probs, d_tiles, ntiles, d_ws, err, s)
          : prec == HODLR_GEMM_TF32X3
              ? launch_umma<HODLR_GEMM_TF32X3, true, 0>(d_probs, d_tiles, ntiles, d_ws, err, s)
              : launch_umma<HODLR_GEMM_TF32, true, 0>(d_probs, d_tiles, ntiles, d_ws, err, s);
  if (e) return e;
  if (any_split) umma_splitk_reduce<<<dim3(64, nprob), 256, 0, s>>>(d_probs, d_ws);
  return (int)cudaGetLastError();
}

int umma_nn_sub_launch(int prec, const GemmProblem* d_probs, const int4* d_tiles, int ntiles,
                       unsigned* err, cudaStream_t s) {
  if (ntiles == 0) return 0;
  return prec == HODLR_GEMM_BF16
             ? launch_umma<HODLR_GEMM_BF16, false, 1>(d_probs, d_tiles, ntiles, nullptr, err, s)
         : prec == HODLR_GEMM_TF32X3
             ? launch_umma<HODLR_GEMM_TF32X3, false, 1>(d_probs, d_tiles, ntiles, nullptr, err, s)
             : launch_umma<HODLR_GEMM_TF32, false, 1>(d_probs, d_tiles, ntiles, nullptr, err, s);
}
