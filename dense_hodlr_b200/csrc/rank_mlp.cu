// Learned rank predictor: a 14-64-64-1 MLP with GELU that maps an
// off-diagonal block's geometry (both clusters' bounding-box centres and
// extents, 3D), log l and log tol to log(1 + ACA rank).  It runs in BF16 with
// FP32 accumulation: inputs, weights and hidden activations are rounded to
// BF16, every dot product accumulates BF16 x BF16 products (exact in FP32) in
// FP32.  Training keeps FP32 master weights and Adam moments.
//
// The reference has no learned part; the predictor only sizes ACA's
// workspace and balances its CTAs, while ACA's own stopping test decides
// every rank.
//
// Parameter blob (FP32): [mean(14) | inv_std(14) | W1 64x14 | b1 64 |
// W2 64x64 | b2 64 | W3 64 | b3 1], row-major W (out x in).  Inputs are
// standardised as (x - mean) * inv_std before the BF16 rounding.
//
// Training step (deterministic): mlp_sample_kernel runs forward and
// backward per sample (one thread each) and stores the activations and
// their gradients; mlp_param_kernel gives every parameter one thread that
// sums its gradient over the batch in sample order and applies Adam.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include "../../include/hodlr_b200.h"
#include "common.cuh"
#include "rank_mlp.h"

namespace {

constexpr int NI = HODLR_MLP_INPUTS, NH = HODLR_MLP_HIDDEN;
constexpr int OFF_MEAN = 0, OFF_ISTD = NI, OFF_W1 = 2 * NI, OFF_B1 = OFF_W1 + NH * NI,
              OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH, OFF_W3 = OFF_B2 + NH,
              OFF_B3 = OFF_W3 + NH, NPARAM = OFF_B3 + 1;
static_assert(NPARAM == HODLR_MLP_PARAMS, "parameter count");
constexpr int NTRAIN = NPARAM - 2 * NI;  // trained parameters (W and b)
// per-sample scratch: x (standardised, bf16-rounded), a1, h1, a2, h2, da1, da2, dy, err
constexpr int S_X = 0, S_A1 = S_X + NI, S_H1 = S_A1 + NH, S_A2 = S_H1 + NH, S_H2 = S_A2 + NH,
              S_DA1 = S_H2 + NH, S_DA2 = S_DA1 + NH, S_DY = S_DA2 + NH, S_ERR = S_DY + 1,
              SAMPLE = S_ERR + 1;

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// GELU(a) = a Phi(a); GELU'(a) = Phi(a) + a phi(a)
__device__ __forceinline__ float gelu(float a) { return 0.5f * a * (1.0f + erff(a * 0.70710678f)); }
__device__ __forceinline__ float gelu_d(float a) {
  return 0.5f * (1.0f + erff(a * 0.70710678f)) + a * 0.39894228f * expf(-0.5f * a * a);
}

// BF16 copies of the weights in shared memory (rounded once per CTA).
struct SmemW {
  float w1[NH * NI], b1[NH], w2[NH * NH], b2[NH], w3[NH], b3, mean[NI], istd[NI];
};

__device__ void load_weights(SmemW& s, const float* __restrict__ p) {
  for (int i = threadIdx.x; i < NH * NI; i += blockDim.x) s.w1[i] = bf(p[OFF_W1 + i]);
  for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) s.w2[i] = bf(p[OFF_W2 + i]);
  for (int i = threadIdx.x; i < NH; i += blockDim.x) {
    s.b1[i] = p[OFF_B1 + i];
    s.b2[i] = p[OFF_B2 + i];
    s.w3[i] = bf(p[OFF_W3 + i]);
  }
  for (int i = threadIdx.x; i < NI; i += blockDim.x) {
    s.mean[i] = p[OFF_MEAN + i];
    s.istd[i] = p[OFF_ISTD + i];
  }
  if (threadIdx.x == 0) s.b3 = p[OFF_B3];
  __syncthreads();
}

// Forward of one sample: returns y; with `sc` also stores x, a1, h1, a2, h2
// (h1/h2 BF16-rounded) in the sample's scratch.
__device__ float forward(const SmemW& s, const float* __restrict__ xin, float* sc) {
  float x[NI];
#pragma unroll
  for (int i = 0; i < NI; ++i) x[i] = bf((xin[i] - s.mean[i]) * s.istd[i]);
  float h1[NH];
#pragma unroll 4
  for (int j = 0; j < NH; ++j) {
    float a = s.b1[j];
#pragma unroll
    for (int i = 0; i < NI; ++i) a = fmaf(s.w1[j * NI + i], x[i], a);
    h1[j] = bf(gelu(a));
    if (sc) {
      sc[S_A1 + j] = a;
      sc[S_H1 + j] = h1[j];
    }
  }
  float y = s.b3;
  for (int j = 0; j < NH; ++j) {
    float a = s.b2[j];
#pragma unroll
    for (int i = 0; i < NH; ++i) a = fmaf(s.w2[j * NH + i], h1[i], a);
    const float h2 = bf(gelu(a));
    if (sc) {
      sc[S_A2 + j] = a;
      sc[S_H2 + j] = h2;
    }
    y = fmaf(s.w3[j], h2, y);
  }
  if (sc)
#pragma unroll
    for (int i = 0; i < NI; ++i) sc[S_X + i] = x[i];
  return y;
}

__global__ void mlp_forward_kernel(const float* __restrict__ p, const float* __restrict__ X, int B,
                                   float* __restrict__ y) {
  __shared__ SmemW s;
  load_weights(s, p);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B) y[b] = forward(s, X + (int64_t)b * NI, nullptr);
}

// Forward + backward of one sample per thread, loss 1/B sum (y - t)^2.
__global__ void mlp_sample_kernel(const float* __restrict__ p, const float* __restrict__ X,
                                  const float* __restrict__ T, int B, float* __restrict__ S) {
  __shared__ SmemW s;
  load_weights(s, p);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float* sc = S + (int64_t)b * SAMPLE;
  const float y = forward(s, X + (int64_t)b * NI, sc);
  const float e = y - T[b];
  const float dy = 2.0f * e / (float)B;
  sc[S_DY] = dy;
  sc[S_ERR] = e;
  float da2[NH];
#pragma unroll 4
  for (int j = 0; j < NH; ++j) da2[j] = dy * s.w3[j] * gelu_d(sc[S_A2 + j]);
  for (int i = 0; i < NH; ++i) {
    float d = 0.0f;
#pragma unroll
    for (int j = 0; j < NH; ++j) d = fmaf(s.w2[j * NH + i], da2[j], d);
    sc[S_DA1 + i] = d * gelu_d(sc[S_A1 + i]);
  }
#pragma unroll 4
  for (int j = 0; j < NH; ++j) sc[S_DA2 + j] = da2[j];
}

// One thread per trained parameter: gradient summed over the batch in
// sample order, then (when lr > 0) an Adam step.  grad_out (optional)
// receives the gradient; loss_out (optional) 1/B sum e^2.
__global__ void mlp_param_kernel(float* __restrict__ p, float* __restrict__ m1,
                                 float* __restrict__ m2, const float* __restrict__ S, int B,
                                 float lr, float beta1, float beta2, float eps, int t,
                                 float* __restrict__ grad_out, float* __restrict__ loss_out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q == 0 && loss_out) {
    float l = 0.0f;
    for (int b = 0; b < B; ++b) {
      const float e = S[(int64_t)b * SAMPLE + S_ERR];
      l = fmaf(e, e, l);
    }
    *loss_out = l / (float)B;
  }
  if (q >= NTRAIN) return;
  const int pi = q + 2 * NI;  // index into the blob
  int ga, gb = -1;            // gradient = sum_b sc[ga] * (gb < 0 ? 1 : sc[gb])
  if (pi < OFF_B1) {
    const int r = pi - OFF_W1;
    ga = S_DA1 + r / NI;
    gb = S_X + r % NI;
  } else if (pi < OFF_W2) {
    ga = S_DA1 + (pi - OFF_B1);
  } else if (pi < OFF_B2) {
    const int r = pi - OFF_W2;
    ga = S_DA2 + r / NH;
    gb = S_H1 + r % NH;
  } else if (pi < OFF_W3) {
    ga = S_DA2 + (pi - OFF_B2);
  } else if (pi < OFF_B3) {
    ga = S_DY;
    gb = S_H2 + (pi - OFF_W3);
  } else {
    ga = S_DY;
  }
  float g = 0.0f;
  for (int b = 0; b < B; ++b) {
    const float* sc = S + (int64_t)b * SAMPLE;
    g = fmaf(sc[ga], gb < 0 ? 1.0f : sc[gb], g);
  }
  if (grad_out) grad_out[q] = g;
  if (lr > 0.0f) {
    const float a = beta1 * m1[q] + (1.0f - beta1) * g;
    const float v = beta2 * m2[q] + (1.0f - beta2) * g * g;
    m1[q] = a;
    m2[q] = v;
    const float ah = a / (1.0f - powf(beta1, (float)t));
    const float vh = v / (1.0f - powf(beta2, (float)t));
    p[pi] -= lr * ah / (sqrtf(vh) + eps);
  }
}

// Features of each off-diagonal block: bounding boxes of its row cluster
// [r0, r0+m) and column cluster [c0, c0+n) of the (k-d ordered) points, as
// centre and extent per axis (axes beyond dim are 0), then log l and log tol.
__global__ void block_features_kernel(const double* __restrict__ pts, int64_t ld, int dim,
                                      const int4* __restrict__ geom, int nb, float log_l,
                                      float log_tol, float* __restrict__ F) {
  const int blk = blockIdx.x;
  if (blk >= nb) return;
  const int4 gm = geom[blk];  // r0, c0, m, n
  __shared__ double red[2][3][2][32];
  for (int side = 0; side < 2; ++side) {
    const int lo = side == 0 ? gm.x : gm.y, cnt = side == 0 ? gm.z : gm.w;
    for (int d = 0; d < 3; ++d) {
      double mn = INFINITY, mx = -INFINITY;
      if (d < dim)
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
          const double v = pts[d * ld + lo + i];
          mn = fmin(mn, v);
          mx = fmax(mx, v);
        }
      for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      }
      if ((threadIdx.x & 31) == 0) {
        red[side][d][0][threadIdx.x >> 5] = mn;
        red[side][d][1][threadIdx.x >> 5] = mx;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int side = threadIdx.x / 3, d = threadIdx.x % 3;
    double mn = INFINITY, mx = -INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      mn = fmin(mn, red[side][d][0][w]);
      mx = fmax(mx, red[side][d][1][w]);
    }
    if (d >= dim || !(mx >= mn)) mn = mx = 0.0;
    float* f = F + (int64_t)blk * NI + side * 6;
    f[d] = (float)(0.5 * (mn + mx));
    f[3 + d] = (float)(mx - mn);
  }
  if (threadIdx.x == 0) {
    F[(int64_t)blk * NI + 12] = log_l;
    F[(int64_t)blk * NI + 13] = log_tol;
  }
}

}  // namespace

int mlp_sample_floats() { return SAMPLE; }

int mlp_forward_launch(const float* p, const float* X, int B, float* y, cudaStream_t s) {
  if (B <= 0) return 0;
  mlp_forward_kernel<<<(B + 127) / 128, 128, 0, s>>>(p, X, B, y);
  return (int)cudaGetLastError();
}

int mlp_train_launch(float* p, float* m1, float* m2, const float* X, const float* T, int B,
                     float* S, float lr, int t, float* grad_out, float* loss_out,
                     cudaStream_t s) {
  if (B <= 0) return (int)cudaErrorInvalidValue;
  mlp_sample_kernel<<<(B + 127) / 128, 128, 0, s>>>(p, X, T, B, S);
  mlp_param_kernel<<<(NTRAIN + 127) / 128, 128, 0, s>>>(p, m1, m2, S, B, lr, 0.9f, 0.999f,
                                                        1e-8f, t, grad_out, loss_out);
  return (int)cudaGetLastError();
}

int block_features_launch(const double* pts, int64_t ld, int dim, const int4* geom, int nb,
                          float log_l, float log_tol, float* F, cudaStream_t s) {
  if (nb <= 0) return 0;
  block_features_kernel<<<nb, 256, 0, s>>>(pts, ld, dim, geom, nb, log_l, log_tol, F);
  return (int)cudaGetLastError();
}
