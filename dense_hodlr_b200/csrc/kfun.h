// Kernel-entry formulas shared by the device kernels and the CPU oracle.
//
// The reference evaluates a matrix entry through a user index functor
// `double (*)(int i, int j, void*)` (include/kernel.hpp:6-33,
// src/kernel.cpp:37-39).  A host function pointer cannot run on the GPU, so
// the entry is instead computed from point coordinates by one of the closed
// forms below.  Every operation is written unfused and correctly rounded
// (explicit _rn intrinsics on the device, -ffp-contract=off on the host) so
// that the same inputs give the same bits on the CPU and on the GPU; that is
// what lets ACA pivot sequences be compared bit for bit.
//
// hx_exp is written from the mathematics (Cody & Waite argument reduction,
// "Software Manual for the Elementary Functions", 1980, followed by the
// Taylor series of e^r on |r| <= ln2/2 evaluated by Horner's rule); it does
// not follow any vendor implementation.  Its accuracy against libm is tested
// (tests/test_oracle.py).
#pragma once

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define HX_HD __host__ __device__ __forceinline__
#else
#define HX_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define HX_MUL(a, b) __dmul_rn((a), (b))
#define HX_ADD(a, b) __dadd_rn((a), (b))
#define HX_SUB(a, b) __dsub_rn((a), (b))
#define HX_DIV(a, b) __ddiv_rn((a), (b))
#define HX_SQRT(a) __dsqrt_rn((a))
#else
#define HX_MUL(a, b) ((a) * (b))
#define HX_ADD(a, b) ((a) + (b))
#define HX_SUB(a, b) ((a) - (b))
#define HX_DIV(a, b) ((a) / (b))
#define HX_SQRT(a) sqrt((a))
#endif

// Kernel families.  Values are part of the C ABI (include/hodlr_b200.h).
enum {
  HX_KERNEL_GAUSSIAN = 0,          // exp(-r^2 / l^2)
  HX_KERNEL_MATERN32 = 1,          // (1 + sqrt(3) r / l) exp(-sqrt(3) r / l)
  HX_KERNEL_INV_MULTIQUADRIC = 2,  // 1 / sqrt(1 + r^2 / l^2)
  HX_KERNEL_QUADRATIC = 3,         // 1 + r^2 / l^2
  HX_KERNEL_EXPONENTIAL = 4,       // exp(-r / l)
};

// Parameters of one kernel, derived once on the host from the length scale
// so that both sides use the identical constant `a`.
struct hx_kparams {
  int type;
  int dim;
  double a;            // type-dependent scale, see hx_make_kparams
  double shift;        // added to the diagonal (diag_replace == 0)
  double diag_value;   // replaces the diagonal (diag_replace == 1)
  int diag_replace;
};

static inline hx_kparams hx_make_kparams(int type, int dim, double length_scale,
                                         double shift, int diag_replace,
                                         double diag_value) {
  hx_kparams p;
  p.type = type;
  p.dim = dim;
  p.shift = shift;
  p.diag_value = diag_value;
  p.diag_replace = diag_replace;
  double l = length_scale;
  switch (type) {
    case HX_KERNEL_GAUSSIAN: p.a = -1.0 / (l * l); break;
    case HX_KERNEL_MATERN32: p.a = sqrt(3.0) / l; break;
    case HX_KERNEL_EXPONENTIAL: p.a = 1.0 / l; break;
    default: p.a = 1.0 / (l * l); break;  // INV_MULTIQUADRIC, QUADRATIC
  }
  return p;
}

// 2^k for -1022 <= k <= 1023, built from its bit pattern.
HX_HD double hx_pow2i(int k) {
  uint64_t bits = (uint64_t)(int64_t)(k + 1023) << 52;
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)bits);
#else
  double d;
  memcpy(&d, &bits, sizeof(d));
  return d;
#endif
}

// e^x.  x = k ln2 + r with ln2 split into a 32-bit head (exact products for
// |k| < 2^21) and a tail; e^r from its Taylor series to degree 13, whose
// truncation error on |r| <= 0.347 is below 5e-18 relative.
HX_HD double hx_exp(double x) {
  const double LOG2E = 0x1.71547652b82fep+0;
  const double LN2_HI = 0x1.62e42fee00000p-1;
  const double LN2_LO = 0x1.a39ef35793c76p-33;
  if (x != x) return x;
  if (x > 709.782712893384) return HUGE_VAL;
  if (x < -745.2) return 0.0;
  double kd = rint(HX_MUL(x, LOG2E));
  double r = HX_SUB(HX_SUB(x, HX_MUL(kd, LN2_HI)), HX_MUL(kd, LN2_LO));
  // 1/i! for i = 13 .. 1, each correctly rounded.
  double p = 0x1.6124613a86d09p-33;
  p = HX_ADD(HX_MUL(p, r), 0x1.1eed8eff8d898p-29);
  p = HX_ADD(HX_MUL(p, r), 0x1.ae64567f544e4p-26);
  p = HX_ADD(HX_MUL(p, r), 0x1.27e4fb7789f5cp-22);
  p = HX_ADD(HX_MUL(p, r), 0x1.71de3a556c734p-19);
  p = HX_ADD(HX_MUL(p, r), 0x1.a01a01a01a01ap-16);
  p = HX_ADD(HX_MUL(p, r), 0x1.a01a01a01a01ap-13);
  p = HX_ADD(HX_MUL(p, r), 0x1.6c16c16c16c17p-10);
  p = HX_ADD(HX_MUL(p, r), 0x1.1111111111111p-7);
  p = HX_ADD(HX_MUL(p, r), 0x1.5555555555555p-5);
  p = HX_ADD(HX_MUL(p, r), 0x1.5555555555555p-3);
  p = HX_ADD(HX_MUL(p, r), 0.5);
  p = HX_ADD(HX_MUL(p, r), 1.0);
  p = HX_ADD(HX_MUL(p, r), 1.0);
  int k = (int)kd;
  if (k > 1023) return HX_MUL(HX_MUL(p, 2.0), hx_pow2i(k - 1));
  if (k < -1022) return HX_MUL(HX_MUL(p, hx_pow2i(k + 600)), hx_pow2i(-600));
  return HX_MUL(p, hx_pow2i(k));
}

// Kernel value as a function of the squared distance r2 (off-diagonal form).
HX_HD double hx_kernel_r2(const hx_kparams& p, double r2) {
  switch (p.type) {
    case HX_KERNEL_GAUSSIAN:
      return hx_exp(HX_MUL(r2, p.a));
    case HX_KERNEL_MATERN32: {
      double s = HX_MUL(HX_SQRT(r2), p.a);
      return HX_MUL(HX_ADD(1.0, s), hx_exp(-s));
    }
    case HX_KERNEL_INV_MULTIQUADRIC:
      return HX_DIV(1.0, HX_SQRT(HX_ADD(1.0, HX_MUL(r2, p.a))));
    case HX_KERNEL_QUADRATIC:
      return HX_ADD(HX_MUL(r2, p.a), 1.0);
    case HX_KERNEL_EXPONENTIAL:
      return hx_exp(-HX_MUL(HX_SQRT(r2), p.a));
    default:
      return 0.0;
  }
}

// Squared distance between point i and point j; coordinates are stored
// dimension-major (SoA): pts[d * ld + i].  Summed in dimension order.
HX_HD double hx_dist2(const double* pts, int64_t ld, int dim, int i, int j) {
  double r2 = 0.0;
  for (int d = 0; d < dim; ++d) {
    double t = HX_SUB(pts[d * ld + i], pts[d * ld + j]);
    r2 = HX_ADD(r2, HX_MUL(t, t));
  }
  return r2;
}

// Entry K(i, j): kernel of the distance, with the diagonal either shifted
// (K_ii = f(0) + shift) or replaced (K_ii = diag_value).
HX_HD double hx_entry(const hx_kparams& p, const double* pts, int64_t ld, int i,
                      int j) {
  if (i == j && p.diag_replace) return p.diag_value;
  double v = hx_kernel_r2(p, hx_dist2(pts, ld, p.dim, i, j));
  if (i == j) v = HX_ADD(v, p.shift);
  return v;
}
