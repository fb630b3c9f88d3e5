// C++ host test of include/HODLR_Matrix.hpp: the reference's test shapes
// through the drop-in class (test/test.cpp:57-69 exact-rank HODLR, the kernel
// path of test/test.cpp:565-576), returning non-zero on failure.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>

#include "HODLR_Matrix.hpp"

using hodlr_b200::Matrix;

static double rel_err(const Matrix& a, const Matrix& b) {
  double num = 0, den = 0;
  for (int j = 0; j < a.cols(); ++j)
    for (int i = 0; i < a.rows(); ++i) {
      double d = a(i, j) - b(i, j);
      num += d * d;
      den += b(i, j) * b(i, j);
    }
  return std::sqrt(num / den);
}

int main() {
  int fails = 0;
  // kernel path: K_ij = (x_i - x_j)^2 + 1, K_ii = 0 on LinSpaced(-2, 2)
  {
    const int n = 10000;
    Matrix X = Matrix::LinSpaced(n, -2, 2);
    hodlr_kernel_desc k{HODLR_KERNEL_QUADRATIC, 1.0, 0.0, 1, 0.0};
    HODLR_Matrix K(n, n, k, X.data(), 1, 30);
    Matrix b(n, 1);
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int j = 0; j < n; ++j)
        if (i != j) s += ((X(i, 0) - X(j, 0)) * (X(i, 0) - X(j, 0)) + 1.0) * X(j, 0);
      b(i, 0) = s;
    }
    K.printResultInfo = true;
    Matrix x = K.recLU_Solve(b);
    double e = rel_err(x, X);
    std::printf("kernel path rel. error %g\n", e);
    fails += !(e < 1e-6);
  }
  // dense path: exact rank-10 HODLR blocks are not needed for the facade;
  // a diagonally dominant Gaussian kernel matrix, solved directly and by GMRES
  {
    const int n = 4096;
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1, 1);
    std::vector<double> p(n);
    for (auto& v : p) v = U(rng);
    std::sort(p.begin(), p.end());
    Matrix A(n, n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        A(i, j) = std::exp(-(p[i] - p[j]) * (p[i] - p[j]) / 0.01) + (i == j ? 1.0 : 0.0);
    HODLR_Matrix H(A, 64);
    H.set_LRTolerance(1e-10);
    Matrix xe = Matrix::LinSpaced(n, -2, 2), b(n, 1);
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int j = 0; j < n; ++j) s += A(i, j) * xe(j, 0);
      b(i, 0) = s;
    }
    Matrix x = H.recLU_Solve(b);
    double e = rel_err(x, xe);
    std::printf("dense path rel. error %g (total %g s)\n", e, H.get_recLU_TotalTime());
    fails += !(e < 1e-8);
    Matrix x2 = H.iterative_Solve(b, 100, 1e-12, 1e-6, "partialPiv_ACA");
    double e2 = rel_err(x2, xe);
    std::printf("iterative_Solve rel. error %g after %d iterations\n", e2, H.last_iterations());
    fails += !(e2 < 1e-9);
  }
  // user_IndexTree (reference :184) and logAbsDeterminant (:249): a root split
  // off-centre with default subtrees; the solution and the determinant agree
  // with the default tree's
  {
    const int n = 3000;
    Matrix X = Matrix::LinSpaced(n, -1, 1);
    hodlr_kernel_desc k{HODLR_KERNEL_GAUSSIAN, 0.1, 1.0, 0, 0.0};
    user_IndexTree t;
    t.rootNode = new user_IndexTree::node();
    t.rootNode->splitIndex = 999;
    HODLR_Matrix Ku(n, n, k, X.data(), 1, 64, t);
    HODLR_Matrix Kd(n, n, k, X.data(), 1, 64);
    Ku.set_LRTolerance(1e-12);
    Kd.set_LRTolerance(1e-12);
    Matrix b(n, 1);
    for (int i = 0; i < n; ++i) b(i, 0) = std::sin(3.0 * i);
    double e = rel_err(Ku.recLU_Solve(b), Kd.recLU_Solve(b));
    double du = Ku.logAbsDeterminant(), dd = Kd.logAbsDeterminant();
    std::printf("user tree: solution diff %g, log|det| %.12g vs %.12g\n", e, du, dd);
    fails += !(e < 1e-9) + !(std::fabs(du - dd) < 1e-8 * std::fabs(dd));
    // rank bounds of a user node reach the GPU ACA: the root's top block
    // stops at rank 5 (src/lowRank.cpp:244-247)
    user_IndexTree bounded;
    bounded.rootNode = new user_IndexTree::node();
    bounded.rootNode->splitIndex = 999;
    bounded.rootNode->topOffDiag_maxRank = 5;
    HODLR_Matrix Kb(n, n, k, X.data(), 1, 64, bounded);
    Kb.set_LRTolerance(1e-12);
    Kb.storeLRinTree();
    int rk[2] = {0, 0};
    hodlr_b200::check(Kb.handle(), hodlr_get_ranks(Kb.handle(), rk), "ranks");
    std::printf("bounded user tree: root ranks %d %d\n", rk[0], rk[1]);
    fails += !(rk[0] == 5 && rk[1] > 5);
    // recSM_Solve (reference :215): the perturbI factorization solves the
    // same system
    Matrix xs = Kd.recSM_Solve(b), xl = Kd.recLU_Solve(b);
    double es = rel_err(xs, xl);
    std::printf("recSM vs recLU: %g\n", es);
    fails += !(es < 1e-10);
  }
  try {
    HODLR_Matrix bad(10, 10, [](int, int, void*) { return 0.0; }, nullptr, 30);
    fails += 1;
  } catch (const hodlr_b200::Error& e) {
    fails += (e.status() != HODLR_ERR_UNSUPPORTED);
  }
  std::printf("%s\n", fails ? "FAILED" : "OK");
  return fails;
}
