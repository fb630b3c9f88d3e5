// Fast FP64 kernel entries for the full-kernel residual r = b - K x.
//
// The residual needs FP64-accurate entries (a few ulp), not entries that are
// bit-identical to the ones ACA used, so it may contract into FMAs and use a
// cheaper exponential.  exp here follows Tang's table-driven method (P. T. P.
// Tang, "Table-driven implementation of the exponential function in IEEE
// floating-point arithmetic", ACM TOMS 15(2), 1989): x = (256k + j) ln2/256 + r,
// |r| <= ln2/512, e^x = 2^k * 2^(j/256) * e^r with e^r - 1 from its Taylor
// series to degree 4 (truncation below 4e-17) and 2^(j/256) from a 256-entry
// table (each entry correctly rounded, computed with exact arithmetic).
#pragma once

#include "kfun.h"

// 2^(j/256), j = 0..255, correctly rounded.
#define HX_TANG_TABLE_SIZE 256
#define HX_TANG_TABLE_INIT { \
    0x1.0000000000000p+0, 0x1.00b1afa5abcbfp+0, 0x1.0163da9fb3335p+0, 0x1.02168143b0281p+0, \
    0x1.02c9a3e778061p+0, 0x1.037d42e11bbccp+0, 0x1.04315e86e7f85p+0, 0x1.04e5f72f654b1p+0, \
    0x1.059b0d3158574p+0, 0x1.0650a0e3c1f89p+0, 0x1.0706b29ddf6dep+0, 0x1.07bd42b72a836p+0, \
    0x1.0874518759bc8p+0, 0x1.092bdf66607e0p+0, 0x1.09e3ecac6f383p+0, 0x1.0a9c79b1f3919p+0, \
    0x1.0b5586cf9890fp+0, 0x1.0c0f145e46c85p+0, 0x1.0cc922b7247f7p+0, 0x1.0d83b23395decp+0, \
    0x1.0e3ec32d3d1a2p+0, 0x1.0efa55fdfa9c5p+0, 0x1.0fb66affed31bp+0, 0x1.1073028d7233ep+0, \
    0x1.11301d0125b51p+0, 0x1.11edbab5e2ab6p+0, 0x1.12abdc06c31ccp+0, 0x1.136a814f204abp+0, \
    0x1.1429aaea92de0p+0, 0x1.14e95934f312ep+0, 0x1.15a98c8a58e51p+0, 0x1.166a45471c3c2p+0, \
    0x1.172b83c7d517bp+0, 0x1.17ed48695bbc0p+0, 0x1.18af9388c8deap+0, 0x1.1972658375d2fp+0, \
    0x1.1a35beb6fcb75p+0, 0x1.1af99f8138a1cp+0, 0x1.1bbe084045cd4p+0, 0x1.1c82f95281c6bp+0, \
    0x1.1d4873168b9aap+0, 0x1.1e0e75eb44027p+0, 0x1.1ed5022fcd91dp+0, 0x1.1f9c18438ce4dp+0, \
    0x1.2063b88628cd6p+0, 0x1.212be3578a819p+0, 0x1.21f49917ddc96p+0, 0x1.22bdda27912d1p+0, \
    0x1.2387a6e756238p+0, 0x1.2451ffb82140ap+0, 0x1.251ce4fb2a63fp+0, 0x1.25e85711ece75p+0, \
    0x1.26b4565e27cddp+0, 0x1.2780e341ddf29p+0, 0x1.284dfe1f56381p+0, 0x1.291ba7591bb70p+0, \
    0x1.29e9df51fdee1p+0, 0x1.2ab8a66d10f13p+0, 0x1.2b87fd0dad990p+0, 0x1.2c57e39771b2fp+0, \
    0x1.2d285a6e4030bp+0, 0x1.2df961f641589p+0, 0x1.2ecafa93e2f56p+0, 0x1.2f9d24abd886bp+0, \
    0x1.306fe0a31b715p+0, 0x1.31432edeeb2fdp+0, 0x1.32170fc4cd831p+0, 0x1.32eb83ba8ea32p+0, \
    0x1.33c08b26416ffp+0, 0x1.3496266e3fa2dp+0, 0x1.356c55f929ff1p+0, 0x1.36431a2de883bp+0, \
    0x1.371a7373aa9cbp+0, 0x1.37f26231e754ap+0, 0x1.38cae6d05d866p+0, 0x1.39a401b7140efp+0, \
    0x1.3a7db34e59ff7p+0, 0x1.3b57fbfec6cf4p+0, 0x1.3c32dc313a8e5p+0, 0x1.3d0e544ede173p+0, \
    0x1.3dea64c123422p+0, 0x1.3ec70df1c5175p+0, 0x1.3fa4504ac801cp+0, 0x1.40822c367a024p+0, \
    0x1.4160a21f72e2ap+0, 0x1.423fb2709468ap+0, 0x1.431f5d950a897p+0, 0x1.43ffa3f84b9d4p+0, \
    0x1.44e086061892dp+0, 0x1.45c2042a7d232p+0, 0x1.46a41ed1d0057p+0, 0x1.4786d668b3237p+0, \
    0x1.486a2b5c13cd0p+0, 0x1.494e1e192aed2p+0, 0x1.4a32af0d7d3dep+0, 0x1.4b17dea6db7d7p+0, \
    0x1.4bfdad5362a27p+0, 0x1.4ce41b817c114p+0, 0x1.4dcb299fddd0dp+0, 0x1.4eb2d81d8abffp+0, \
    0x1.4f9b2769d2ca7p+0, 0x1.508417f4531eep+0, 0x1.516daa2cf6642p+0, 0x1.5257de83f4eefp+0, \
    0x1.5342b569d4f82p+0, 0x1.542e2f4f6ad27p+0, 0x1.551a4ca5d920fp+0, 0x1.56070dde910d2p+0, \
    0x1.56f4736b527dap+0, 0x1.57e27dbe2c4cfp+0, 0x1.58d12d497c7fdp+0, 0x1.59c0827ff07ccp+0, \
    0x1.5ab07dd485429p+0, 0x1.5ba11fba87a03p+0, 0x1.5c9268a5946b7p+0, 0x1.5d84590998b93p+0, \
    0x1.5e76f15ad2148p+0, 0x1.5f6a320dceb71p+0, 0x1.605e1b976dc09p+0, 0x1.6152ae6cdf6f4p+0, \
    0x1.6247eb03a5585p+0, 0x1.633dd1d1929fdp+0, 0x1.6434634ccc320p+0, 0x1.652b9febc8fb7p+0, \
    0x1.6623882552225p+0, 0x1.671c1c70833f6p+0, 0x1.68155d44ca973p+0, 0x1.690f4b19e9538p+0, \
    0x1.6a09e667f3bcdp+0, 0x1.6b052fa75173ep+0, 0x1.6c012750bdabfp+0, 0x1.6cfdcddd47645p+0, \
    0x1.6dfb23c651a2fp+0, 0x1.6ef9298593ae5p+0, 0x1.6ff7df9519484p+0, 0x1.70f7466f42e87p+0, \
    0x1.71f75e8ec5f74p+0, 0x1.72f8286ead08ap+0, 0x1.73f9a48a58174p+0, 0x1.74fbd35d7cbfdp+0, \
    0x1.75feb564267c9p+0, 0x1.77024b1ab6e09p+0, 0x1.780694fde5d3fp+0, 0x1.790b938ac1cf6p+0, \
    0x1.7a11473eb0187p+0, 0x1.7b17b0976cfdbp+0, 0x1.7c1ed0130c132p+0, 0x1.7d26a62ff86f0p+0, \
    0x1.7e2f336cf4e62p+0, 0x1.7f3878491c491p+0, 0x1.80427543e1a12p+0, 0x1.814d2add106d9p+0, \
    0x1.82589994cce13p+0, 0x1.8364c1eb941f7p+0, 0x1.8471a4623c7adp+0, 0x1.857f4179f5b21p+0, \
    0x1.868d99b4492edp+0, 0x1.879cad931a436p+0, 0x1.88ac7d98a6699p+0, 0x1.89bd0a478580fp+0, \
    0x1.8ace5422aa0dbp+0, 0x1.8be05bad61778p+0, 0x1.8cf3216b5448cp+0, 0x1.8e06a5e0866d9p+0, \
    0x1.8f1ae99157736p+0, 0x1.902fed0282c8ap+0, 0x1.9145b0b91ffc6p+0, 0x1.925c353aa2fe2p+0, \
    0x1.93737b0cdc5e5p+0, 0x1.948b82b5f98e5p+0, 0x1.95a44cbc8520fp+0, 0x1.96bdd9a7670b3p+0, \
    0x1.97d829fde4e50p+0, 0x1.98f33e47a22a2p+0, 0x1.9a0f170ca07bap+0, 0x1.9b2bb4d53fe0dp+0, \
    0x1.9c49182a3f090p+0, 0x1.9d674194bb8d5p+0, 0x1.9e86319e32323p+0, 0x1.9fa5e8d07f29ep+0, \
    0x1.a0c667b5de565p+0, 0x1.a1e7aed8eb8bbp+0, 0x1.a309bec4a2d33p+0, 0x1.a42c980460ad8p+0, \
    0x1.a5503b23e255dp+0, 0x1.a674a8af46052p+0, 0x1.a799e1330b358p+0, 0x1.a8bfe53c12e59p+0, \
    0x1.a9e6b5579fdbfp+0, 0x1.ab0e521356ebap+0, 0x1.ac36bbfd3f37ap+0, 0x1.ad5ff3a3c2774p+0, \
    0x1.ae89f995ad3adp+0, 0x1.afb4ce622f2ffp+0, 0x1.b0e07298db666p+0, 0x1.b20ce6c9a8952p+0, \
    0x1.b33a2b84f15fbp+0, 0x1.b468415b749b1p+0, 0x1.b59728de5593ap+0, 0x1.b6c6e29f1c52ap+0, \
    0x1.b7f76f2fb5e47p+0, 0x1.b928cf22749e4p+0, 0x1.ba5b030a1064ap+0, 0x1.bb8e0b79a6f1fp+0, \
    0x1.bcc1e904bc1d2p+0, 0x1.bdf69c3f3a207p+0, 0x1.bf2c25bd71e09p+0, 0x1.c06286141b33dp+0, \
    0x1.c199bdd85529cp+0, 0x1.c2d1cd9fa652cp+0, 0x1.c40ab5fffd07ap+0, 0x1.c544778fafb22p+0, \
    0x1.c67f12e57d14bp+0, 0x1.c7ba88988c933p+0, 0x1.c8f6d9406e7b5p+0, 0x1.ca3405751c4dbp+0, \
    0x1.cb720dcef9069p+0, 0x1.ccb0f2e6d1675p+0, 0x1.cdf0b555dc3fap+0, 0x1.cf3155b5bab74p+0, \
    0x1.d072d4a07897cp+0, 0x1.d1b532b08c968p+0, 0x1.d2f87080d89f2p+0, 0x1.d43c8eacaa1d6p+0, \
    0x1.d5818dcfba487p+0, 0x1.d6c76e862e6d3p+0, 0x1.d80e316c98398p+0, 0x1.d955d71ff6075p+0, \
    0x1.da9e603db3285p+0, 0x1.dbe7cd63a8315p+0, 0x1.dd321f301b460p+0, 0x1.de7d5641c0658p+0, \
    0x1.dfc97337b9b5fp+0, 0x1.e11676b197d17p+0, 0x1.e264614f5a129p+0, 0x1.e3b333b16ee12p+0, \
    0x1.e502ee78b3ff6p+0, 0x1.e653924676d76p+0, 0x1.e7a51fbc74c83p+0, 0x1.e8f7977cdb740p+0, \
    0x1.ea4afa2a490dap+0, 0x1.eb9f4867cca6ep+0, 0x1.ecf482d8e67f1p+0, 0x1.ee4aaa2188510p+0, \
    0x1.efa1bee615a27p+0, 0x1.f0f9c1cb6412ap+0, 0x1.f252b376bba97p+0, 0x1.f3ac948dd7274p+0, \
    0x1.f50765b6e4540p+0, 0x1.f6632798844f8p+0, 0x1.f7bfdad9cbe14p+0, 0x1.f91d802243c89p+0, \
    0x1.fa7c1819e90d8p+0, 0x1.fbdba3692d514p+0, 0x1.fd3c22b8f71f1p+0, 0x1.fe9d96b2a23d9p+0, \
}

static const double hx_tang_host[HX_TANG_TABLE_SIZE] = HX_TANG_TABLE_INIT;

// e^x with the 2^(j/256) table at `tab` (shared or global memory).
HX_HD double hx_exp_tang(double x, const double* tab) {
  const double INV_L = 0x1.71547652b82fep+8;  // 256 / ln2
  const double L_HI = 0x1.62e42fe000000p-9;   // ln2/256, 29 significant bits
  const double L_LO = 0x1.f473de6af278fp-38;
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
  // e^r - 1 = r + r^2 (1/2 + r (1/6 + r/24))
  double p = fma(r, 0x1.5555555555555p-5, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p * r, r, r);
  const int j = n & 255;
  const int k = (n - j) >> 8;  // floor(n / 256)
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
  const double INV_L = 0x1.71547652b82fep+8;
  const double L_HI = 0x1.62e42fe000000p-9;
  const double L_LO = 0x1.f473de6af278fp-38;
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
  double p = fma(r, 0x1.5555555555555p-5, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p * r, r, r);
  const double t = tab[n & 255];
  const double v = fma(t, p, t);
  const int64_t k = (int64_t)((n - (n & 255)) >> 8);
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
