// C++ test of the device-functor constructor of include/HODLR_Matrix.hpp
// (the GPU form of HODLR_Matrix(int, int, double (*)(int,int,void*), void*,
// int), reference include/HODLR_Matrix.hpp:162), compiled with nvcc against
// libhodlr_b200.so; returns non-zero on failure.
//  1. A functor returning the library's own closed-form Gaussian entries
//     (kfun.h hx_entry) gives the same block ranks and the same solution as
//     the closed-form kernel constructor on the same points.
//  2. A kernel with no closed form in the library (Cauchy, 1 / (1 + r^2/l^2),
//     plus 2 on the diagonal) solves to a small residual, checked on the host.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "HODLR_Matrix.hpp"
#include "kfun.h"

using hodlr_b200::Matrix;

struct LibraryEntry {
  const double* x;
  hx_kparams kp;
  int n;
  __device__ double operator()(int i, int j) const { return hx_entry(kp, x, n, i, j); }
};

struct Cauchy {
  const double* x;
  double inv_l2;
  __host__ __device__ double operator()(int i, int j) const {
    const double d = x[i] - x[j];
    return 1.0 / (1.0 + d * d * inv_l2) + (i == j ? 2.0 : 0.0);
  }
};

int main() {
  int fails = 0;
  const int n = 6000;
  std::mt19937_64 rng(17);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  std::normal_distribution<double> G;
  std::vector<double> x(n);
  for (double& v : x) v = U(rng);
  std::sort(x.begin(), x.end());
  double* dx = nullptr;
  if (cudaMalloc(&dx, sizeof(double) * n) != cudaSuccess ||
      cudaMemcpy(dx, x.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
    std::printf("FAIL: device points\n");
    return 1;
  }
  Matrix b(n, 2);
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < n; ++i) b(i, j) = G(rng);

  {  // 1. functor vs closed form
    const hodlr_kernel_desc k{HODLR_KERNEL_GAUSSIAN, 0.1, 1.0, 0, 0.0};
    const hx_kparams kp = hx_make_kparams(k.type, 1, k.length_scale, k.diag_shift, 0, 0.0);
    HODLR_Matrix F(n, n, LibraryEntry{dx, kp, n}, 64);
    HODLR_Matrix C(n, n, k, x.data(), 1, 64);
    F.set_LRTolerance(1e-10);
    C.set_LRTolerance(1e-10);
    Matrix xf = F.recLU_Solve(b), xc = C.recLU_Solve(b);
    int nb_f = 0, nb_c = 0;
    hodlr_get_num_blocks(F.handle(), &nb_f);
    hodlr_get_num_blocks(C.handle(), &nb_c);
    std::vector<int> rf(nb_f), rc(nb_c);
    hodlr_get_ranks(F.handle(), rf.data());
    hodlr_get_ranks(C.handle(), rc.data());
    const bool same_ranks = nb_f == nb_c && rf == rc;
    double dmax = 0, xmax = 0;
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < n; ++i) {
        dmax = std::max(dmax, std::fabs(xf(i, j) - xc(i, j)));
        xmax = std::max(xmax, std::fabs(xc(i, j)));
      }
    std::printf("functor vs closed form: %d blocks, ranks %s, max |dx| / max |x| = %.3e\n", nb_f,
                same_ranks ? "identical" : "DIFFER", dmax / xmax);
    if (!same_ranks || dmax > 1e-14 * xmax) ++fails;
  }

  {  // 2. a kernel the library has no closed form for
    const double l = 0.05;
    HODLR_Matrix F(n, n, Cauchy{dx, 1.0 / (l * l)}, 64);
    F.set_LRTolerance(1e-10);
    Matrix xs = F.recLU_Solve(b);
    const Cauchy h{x.data(), 1.0 / (l * l)};
    double num = 0, den = 0;
    for (int c = 0; c < 2; ++c)
      for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int j = 0; j < n; ++j) s += h(i, j) * xs(j, c);
        num += (s - b(i, c)) * (s - b(i, c));
        den += b(i, c) * b(i, c);
      }
    const double rel = std::sqrt(num / den);
    std::printf("Cauchy functor: relative residual %.3e\n", rel);
    if (!(rel < 1e-8)) ++fails;
  }

  {  // a non-square functor matrix is refused
    bool threw = false;
    try {
      HODLR_Matrix F(n, n - 1, Cauchy{dx, 1.0}, 64);
    } catch (const hodlr_b200::Error& e) {
      threw = e.status() == HODLR_ERR_ARG;
    }
    std::printf("non-square functor refused: %s\n", threw ? "yes" : "NO");
    if (!threw) ++fails;
  }
  cudaFree(dx);
  std::printf(fails ? "FAILED (%d)\n" : "all passed\n", fails);
  return fails ? 1 : 0;
}
