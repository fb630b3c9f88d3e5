// Fast FP64 kernel entries for the full-kernel residual r = b - K x.
//
// The residual needs FP64-accurate entries (a few ulp), not entries that are
// bit-identical to the ones ACA used, so it may contract into FMAs and use a
// cheaper exponential.  exp here follows Tang's table-driven method (P. T. P.
// Tang, "Table-driven implementation of the exponential function in IEEE
// floating-point arithmetic", ACM TOMS 15(2), 1989): x = (64k + j) ln2/64 + r,
// |r| <= ln2/128, e^x = 2^k * 2^(j/64) * e^r with e^r - 1 from its Taylor
// series to degree 5 (truncation below 4e-17) and 2^(j/64) from a 64-entry
// table (each entry correctly rounded, computed with exact arithmetic).
#pragma once

#include "kfun.h"

// 2^(j/64), j = 0..63, correctly rounded.
#define HX_TANG_TABLE_INIT { \
    0x1.0000000000000p+0, 0x1.02c9a3e778061p+0, 0x1.059b0d3158574p+0, 0x1.0874518759bc8p+0, \
    0x1.0b5586cf9890fp+0, 0x1.0e3ec32d3d1a2p+0, 0x1.11301d0125b51p+0, 0x1.1429aaea92de0p+0, \
    0x1.172b83c7d517bp+0, 0x1.1a35beb6fcb75p+0, 0x1.1d4873168b9aap+0, 0x1.2063b88628cd6p+0, \
    0x1.2387a6e756238p+0, 0x1.26b4565e27cddp+0, 0x1.29e9df51fdee1p+0, 0x1.2d285a6e4030bp+0, \
    0x1.306fe0a31b715p+0, 0x1.33c08b26416ffp+0, 0x1.371a7373aa9cbp+0, 0x1.3a7db34e59ff7p+0, \
    0x1.3dea64c123422p+0, 0x1.4160a21f72e2ap+0, 0x1.44e086061892dp+0, 0x1.486a2b5c13cd0p+0, \
    0x1.4bfdad5362a27p+0, 0x1.4f9b2769d2ca7p+0, 0x1.5342b569d4f82p+0, 0x1.56f4736b527dap+0, \
    0x1.5ab07dd485429p+0, 0x1.5e76f15ad2148p+0, 0x1.6247eb03a5585p+0, 0x1.6623882552225p+0, \
    0x1.6a09e667f3bcdp+0, 0x1.6dfb23c651a2fp+0, 0x1.71f75e8ec5f74p+0, 0x1.75feb564267c9p+0, \
    0x1.7a11473eb0187p+0, 0x1.7e2f336cf4e62p+0, 0x1.82589994cce13p+0, 0x1.868d99b4492edp+0, \
    0x1.8ace5422aa0dbp+0, 0x1.8f1ae99157736p+0, 0x1.93737b0cdc5e5p+0, 0x1.97d829fde4e50p+0, \
    0x1.9c49182a3f090p+0, 0x1.a0c667b5de565p+0, 0x1.a5503b23e255dp+0, 0x1.a9e6b5579fdbfp+0, \
    0x1.ae89f995ad3adp+0, 0x1.b33a2b84f15fbp+0, 0x1.b7f76f2fb5e47p+0, 0x1.bcc1e904bc1d2p+0, \
    0x1.c199bdd85529cp+0, 0x1.c67f12e57d14bp+0, 0x1.cb720dcef9069p+0, 0x1.d072d4a07897cp+0, \
    0x1.d5818dcfba487p+0, 0x1.da9e603db3285p+0, 0x1.dfc97337b9b5fp+0, 0x1.e502ee78b3ff6p+0, \
    0x1.ea4afa2a490dap+0, 0x1.efa1bee615a27p+0, 0x1.f50765b6e4540p+0, 0x1.fa7c1819e90d8p+0, \
}

static const double hx_tang_host[64] = HX_TANG_TABLE_INIT;

// e^x with the 2^(j/64) table at `tab` (shared or global memory).
HX_HD double hx_exp_tang(double x, const double* tab) {
  const double INV_L = 0x1.71547652b82fep+6;  // 64 / ln2
  const double L_HI = 0x1.62e42fe000000p-7;   // ln2/64, 29 significant bits
  const double L_LO = 0x1.f473de6af278fp-36;
  if (!(x > -745.2)) return x != x ? x : 0.0;
  if (x > 709.78) return HUGE_VAL;
  // round-to-nearest integer by the 1.5 * 2^52 shifter: the sum's low word
  // holds n, its difference with the shifter is n as a double
  const double SHIFTER = 0x1.8p52;
  double t0 = fma(x, INV_L, SHIFTER);
  double nd = t0 - SHIFTER;
#if defined(__CUDA_ARCH__)
  int n = __double2loint(t0);
#else
  uint64_t tb;
  memcpy(&tb, &t0, sizeof(tb));
  int n = (int)(uint32_t)(tb & 0xffffffffu);
#endif
  double r = fma(-nd, L_LO, fma(-nd, L_HI, x));
  // e^r - 1 = r + r^2 (1/2 + r (1/6 + r (1/24 + r/120)))
  double p = fma(r, 0x1.1111111111111p-7, 0x1.5555555555555p-5);
  p = fma(p, r, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p * r, r, r);
  const int j = n & 63;
  const int k = (n - j) >> 6;  // floor(n / 64)
  const double t = tab[j];
  double v = fma(t, p, t);
  if (k < -1021) return (v * hx_pow2i(k + 600)) * hx_pow2i(-600);
  if (k > 1023) return (v * 2.0) * hx_pow2i(k - 1);
  return v * hx_pow2i(k);
}

// e^x for x <= 0 without branches.  x is clamped at -707 so that 2^k stays in
// the normal range (k >= -1020) and the scale is a single integer add to the
// exponent field; for x < -707 the result is e^-707 ~ 1e-307 instead of a
// smaller or subnormal value, an absolute difference below 1e-306.
HX_HD double hx_exp_tang_neg(double x, const double* tab) {
  const double INV_L = 0x1.71547652b82fep+6;
  const double L_HI = 0x1.62e42fe000000p-7;
  const double L_LO = 0x1.f473de6af278fp-36;
  const double SHIFTER = 0x1.8p52;
  x = fmax(x, -707.0);
  double t0 = fma(x, INV_L, SHIFTER);
  double nd = t0 - SHIFTER;
#if defined(__CUDA_ARCH__)
  int n = __double2loint(t0);
#else
  uint64_t tb;
  memcpy(&tb, &t0, sizeof(tb));
  int n = (int)(uint32_t)(tb & 0xffffffffu);
#endif
  double r = fma(-nd, L_LO, fma(-nd, L_HI, x));
  double p = fma(r, 0x1.1111111111111p-7, 0x1.5555555555555p-5);
  p = fma(p, r, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p * r, r, r);
  const double t = tab[n & 63];
  const double v = fma(t, p, t);
  const int64_t k = (int64_t)((n - (n & 63)) >> 6);
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(__double_as_longlong(v) + (k << 52));
#else
  int64_t vb;
  memcpy(&vb, &v, sizeof(vb));
  vb += (int64_t)((uint64_t)k << 52);
  double out;
  memcpy(&out, &vb, sizeof(out));
  return out;
#endif
}

#if defined(__CUDACC__)
// Square roots by Newton's method from the hardware reciprocal-square-root
// approximation (rsqrt.approx.ftz.f64, relative error below 2^-20 on this
// GPU).  One Newton step y <- y + y (1 - x y^2) / 2 on 1/sqrt(x) squares the
// error (~2^-40), and hx_rsqrt_nr takes a second one.  x must be a positive
// normal number.
__device__ __forceinline__ double hx_rsqrt_seed(double x) {
  double y;
#if defined(__CUDA_ARCH__)
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#else
  y = 1.0 / sqrt(x);
#endif
  return y;
}
__device__ __forceinline__ double hx_rsqrt_step(double x, double y) {
  const double e = fma(-(x * y), y, 1.0);  // 1 - x y^2
  return fma(0.5 * y, e, y);
}
// sqrt(x) from the seed y0 ~ 1/sqrt(x) (relative error e ~ 2^-20) by one
// third-order correction: with y = x y0 and t = y y0 - 1 (~2e),
// sqrt(x) = y (1 + t)^(-1/2) = y (1 - t/2 + 3t^2/8 - ...), and the dropped
// term 5t^3/16 is below 2^-57.  The rounding of y enters as half its relative
// error, so the result is within 1 ulp of the correctly rounded square root
// (checked against libm's sqrt on 2e7 inputs with seeds perturbed by 2^-20).
__device__ __forceinline__ double hx_sqrt_nr(double x) {
  const double y0 = hx_rsqrt_seed(x);
  const double y = x * y0;
  const double t = fma(y, y0, -1.0);
  return fma(y, t * fma(t, 0.375, -0.5), y);
}
__device__ __forceinline__ double hx_rsqrt_nr(double x) {
  return hx_rsqrt_step(x, hx_rsqrt_step(x, hx_rsqrt_seed(x)));
}
#endif

// Lower bound of the scaled squared distances given to hx_kernel_unit_t: a
// sum of squares that starts here instead of at 0 keeps the reciprocal
// square-root seed finite at r2 = 0 (the diagonal) without a per-entry max,
// and changes no sum above 1e-284 (it is below their half ulp).
#define HX_R2_FLOOR 1e-300

#if defined(__CUDACC__)
// Coordinates scaled by c = hx_point_scale<KTYPE>(a) turn the kernel into a
// function of the scaled squared distance alone (hx_kernel_unit_t): one
// multiply per point instead of one per entry.  r2 >= HX_R2_FLOOR.
template <int KTYPE>
__device__ __forceinline__ double hx_point_scale(double a) {
  if (KTYPE == HX_KERNEL_GAUSSIAN) return sqrt(-a);
  if (KTYPE == HX_KERNEL_MATERN32 || KTYPE == HX_KERNEL_EXPONENTIAL) return a;
  return sqrt(a);  // inverse multiquadric, quadratic
}
template <int KTYPE>
__device__ __forceinline__ double hx_kernel_unit_t(double r2, const double* tab) {
  if (KTYPE == HX_KERNEL_GAUSSIAN) return hx_exp_tang_neg(-r2, tab);
  if (KTYPE == HX_KERNEL_MATERN32) {
    const double s = hx_sqrt_nr(r2);
    const double e = hx_exp_tang_neg(-s, tab);
    return fma(e, s, e);  // (1 + s) e^-s
  }
  if (KTYPE == HX_KERNEL_INV_MULTIQUADRIC) return hx_rsqrt_nr(1.0 + r2);
  if (KTYPE == HX_KERNEL_QUADRATIC) return 1.0 + r2;
  return hx_exp_tang_neg(-hx_sqrt_nr(r2), tab);
}
#endif

// Kernel value of r2 for a kernel family fixed at compile time (no per-entry
// dispatch in the residual kernel).
template <int KTYPE>
HX_HD double hx_kernel_r2_fast_t(double a, double r2, const double* tab) {
  if (KTYPE == HX_KERNEL_GAUSSIAN) return hx_exp_tang_neg(r2 * a, tab);
  if (KTYPE == HX_KERNEL_MATERN32) {
#if defined(__CUDA_ARCH__)
    const double s = hx_sqrt_nr(fmax(r2, 1e-300)) * a;
#else
    const double s = sqrt(r2) * a;
#endif
    const double e = hx_exp_tang_neg(-s, tab);
    return fma(e, s, e);  // (1 + s) e^-s
  }
#if defined(__CUDA_ARCH__)
  if (KTYPE == HX_KERNEL_INV_MULTIQUADRIC) return hx_rsqrt_nr(fma(r2, a, 1.0));
  if (KTYPE == HX_KERNEL_QUADRATIC) return fma(r2, a, 1.0);
  return hx_exp_tang_neg(-hx_sqrt_nr(fmax(r2, 1e-300)) * a, tab);
#else
  if (KTYPE == HX_KERNEL_INV_MULTIQUADRIC) return 1.0 / sqrt(fma(r2, a, 1.0));
  if (KTYPE == HX_KERNEL_QUADRATIC) return fma(r2, a, 1.0);
  return hx_exp_tang_neg(-sqrt(r2) * a, tab);
#endif
}
