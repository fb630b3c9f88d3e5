// HODLR_Matrix.hpp -- C++ drop-in for the recLU path of amiraa127/Dense_HODLR,
// header-only, over the C ABI of libhodlr_b200.so (hodlr_b200.h).
//
// Same class name, constructors, setters, solver entries and getters as the
// reference's include/HODLR_Matrix.hpp (:76, :162, :211-241) for this path;
// everything runs on the GPU.  Differences a caller sees:
//  * errors throw hodlr_b200::Error (with the C status) where the reference
//    prints and calls exit(EXIT_FAILURE);
//  * a host function-pointer kernel cannot run on the GPU: that constructor
//    throws HODLR_ERR_UNSUPPORTED; pass a closed-form kernel of points instead
//    (hodlr_kernel_desc + coordinates), a dense matrix, or (compiled with
//    nvcc) a functor with a __device__ operator()(int i, int j), evaluated on
//    the GPU into a stored n x n matrix;
//  * only the "partialPiv_ACA" low-rank method exists; recLU_Solve and
//    recSM_Solve share one factorization at a time (switching refactors).
// Without Eigen the matrices are hodlr_b200::Matrix (column-major); with
// Eigen on the include path the Eigen::MatrixXd overloads are added.
#ifndef HODLR_B200_HODLR_MATRIX_HPP
#define HODLR_B200_HODLR_MATRIX_HPP

#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "hodlr_b200.h"

#if defined(__CUDACC__)
#include <cuda_runtime.h>

#include <type_traits>
#endif

#if defined(__has_include)
#if __has_include(<Eigen/Dense>)
#include <Eigen/Dense>
#define HODLR_B200_HAVE_EIGEN 1
#endif
#endif

namespace hodlr_b200 {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what)
      : std::runtime_error(std::string(hodlr_status_string(status)) + ": " + what),
        status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

// Column-major dense matrix (the Eigen::MatrixXd stand-in).
class Matrix {
 public:
  Matrix() : r_(0), c_(0) {}
  Matrix(int rows, int cols, double fill = 0.0) : r_(rows), c_(cols), a_((size_t)rows * cols, fill) {}
  int rows() const { return r_; }
  int cols() const { return c_; }
  double& operator()(int i, int j) { return a_[(size_t)j * r_ + i]; }
  double operator()(int i, int j) const { return a_[(size_t)j * r_ + i]; }
  double* data() { return a_.data(); }
  const double* data() const { return a_.data(); }
  static Matrix LinSpaced(int n, double lo, double hi) {
    Matrix m(n, 1);
    for (int i = 0; i < n; ++i) m(i, 0) = n > 1 ? lo + (hi - lo) * i / (n - 1) : lo;
    return m;
  }

 private:
  int r_, c_;
  std::vector<double> a_;
};

inline void check(hodlr_t h, int status, const char* where) {
  if (status != HODLR_OK)
    throw Error(status, std::string(where) + (h ? std::string(" (") + hodlr_last_error(h) + ")" : ""));
}

}  // namespace hodlr_b200

// user_IndexTree (reference include/user_IndexTree.hpp:7-38): a user-defined
// splitting scheme.  splitIndex is the last row of a node's top half (-1:
// none); children may be left NULL for default subtrees below.  The rank
// bounds and per-node low-rank method must keep their defaults (-1, and the
// empty string or "partialPiv_ACA"): the GPU path runs partial-pivot ACA with
// the matrix's tolerance on every block.
class user_IndexTree {
 public:
  struct node {
    node* left = nullptr;
    node* right = nullptr;
    int splitIndex = -1;
    int topOffDiag_minRank = -1;
    int bottOffDiag_minRank = -1;
    int topOffDiag_maxRank = -1;
    int bottOffDiag_maxRank = -1;
    std::string LR_Method;
  };
  node* rootNode = nullptr;

  user_IndexTree() = default;
  user_IndexTree(const user_IndexTree&) = delete;
  user_IndexTree& operator=(const user_IndexTree&) = delete;
  ~user_IndexTree() { freeTree(rootNode); }
  void setChildren_NULL(node* parent) {
    parent->left = nullptr;
    parent->right = nullptr;
  }
  void printTree() const { printTree(rootNode, 0); }

  // pre-order arrays for hodlr_set_index_tree_bounds: split and children, and
  // the four rank bounds of every node (bounds[0..3] = top min, bottom min,
  // top max, bottom max; -1: none)
  void flatten(std::vector<int>& split, std::vector<int>& left, std::vector<int>& right,
               std::vector<int> (&bounds)[4]) const {
    split.clear();
    left.clear();
    right.clear();
    for (auto& b : bounds) b.clear();
    if (rootNode) add(rootNode, split, left, right, bounds);
  }

 private:
  static int add(const node* nd, std::vector<int>& split, std::vector<int>& left,
                 std::vector<int>& right, std::vector<int> (&bounds)[4]) {
    if (!(nd->LR_Method.empty() || nd->LR_Method == "partialPiv_ACA"))
      throw hodlr_b200::Error(HODLR_ERR_UNSUPPORTED,
                              "only partial-pivot ACA is on the GPU path");
    const int id = (int)split.size();
    split.push_back(nd->splitIndex);
    left.push_back(-1);
    right.push_back(-1);
    bounds[0].push_back(nd->topOffDiag_minRank);
    bounds[1].push_back(nd->bottOffDiag_minRank);
    bounds[2].push_back(nd->topOffDiag_maxRank);
    bounds[3].push_back(nd->bottOffDiag_maxRank);
    if (nd->left) left[id] = add(nd->left, split, left, right, bounds);
    if (nd->right) right[id] = add(nd->right, split, left, right, bounds);
    return id;
  }
  static void freeTree(node* nd) {
    if (!nd) return;
    freeTree(nd->left);
    freeTree(nd->right);
    delete nd;
  }
  static void printTree(const node* nd, int depth) {
    if (!nd) return;
    std::printf("%*ssplit %d\n", 2 * depth, "", nd->splitIndex);
    printTree(nd->left, depth + 1);
    printTree(nd->right, depth + 1);
  }
};

#if defined(__CUDACC__)
namespace detail {
// A[i + j ld] = f(i, j): one thread per row, coalesced in i; grid.y strides
// over the columns.
template <class F>
__global__ void fill_from_functor(F f, double* A, int64_t ld, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y) A[(int64_t)j * ld + i] = f(i, j);
}
}  // namespace detail
#endif

class HODLR_Matrix {
 public:
  bool printResultInfo = false;

  // HODLR_Matrix(Eigen::MatrixXd&, int, std::string)  (reference :76)
  explicit HODLR_Matrix(const hodlr_b200::Matrix& A, int inputSizeThreshold = 30,
                        std::string LR_Method = "partialPiv_ACA") {
    if (A.rows() != A.cols()) throw hodlr_b200::Error(HODLR_ERR_ARG, "matrix must be square");
    hodlr_b200::check(nullptr, hodlr_create_dense(&h_, A.rows(), A.data(), A.rows(), inputSizeThreshold),
                      "HODLR_Matrix(dense)");
    n_ = A.rows();
    set_LRMethod(LR_Method);
  }

#ifdef HODLR_B200_HAVE_EIGEN
  explicit HODLR_Matrix(Eigen::MatrixXd& A, int inputSizeThreshold = 30,
                        std::string LR_Method = "partialPiv_ACA") {
    if (A.rows() != A.cols()) throw hodlr_b200::Error(HODLR_ERR_ARG, "matrix must be square");
    hodlr_b200::check(nullptr,
                      hodlr_create_dense(&h_, (int)A.rows(), A.data(), (int)A.rows(), inputSizeThreshold),
                      "HODLR_Matrix(dense)");
    n_ = (int)A.rows();
    set_LRMethod(LR_Method);
  }
#endif

  // HODLR_Matrix(int, int, double (*)(int,int,void*), void*, int)  (reference :162):
  // a host function cannot be evaluated by the GPU kernels.
  HODLR_Matrix(int numRows, int numCols, double (*inputKernel)(int, int, void*),
               void* inputKernelData, int inputSizeThreshold = 30) {
    hodlr_b200::check(nullptr,
                      hodlr_create_fnptr(&h_, numRows, numCols, inputKernel, inputKernelData,
                                         inputSizeThreshold),
                      "HODLR_Matrix(kernel function)");
  }

#if defined(__CUDACC__)
  // HODLR_Matrix(int, int, double (*)(int,int,void*), void*, int)  (reference :162)
  // as a device functor: kernel(i, j) is a __device__ (or __host__ __device__)
  // call operator over data the functor reaches on the device.  It is
  // evaluated once per entry by a kernel compiled in the caller's translation
  // unit into an n x n matrix the handle owns (n^2 doubles of HBM); from
  // there compression, factorization and solves are those of the dense
  // constructor, and the entries are exactly what the functor returns.
  template <class KernelFunctor,
            class = typename std::enable_if<std::is_class<KernelFunctor>::value>::type>
  HODLR_Matrix(int numRows, int numCols, KernelFunctor kernel, int inputSizeThreshold = 30) {
    if (numRows != numCols)
      throw hodlr_b200::Error(HODLR_ERR_ARG, "only square kernel matrices form a HODLR tree");
    double* dA = nullptr;
    int64_t ld = 0;
    hodlr_b200::check(nullptr,
                      hodlr_create_dense_device(&h_, numRows, inputSizeThreshold, &dA, &ld),
                      "HODLR_Matrix(kernel functor)");
    n_ = numRows;
    const unsigned gy = numRows < 65535 ? (unsigned)numRows : 65535u;
    detail::fill_from_functor<<<dim3((unsigned)((numRows + 255) / 256), gy), 256>>>(kernel, dA, ld,
                                                                                     numRows);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
      hodlr_destroy(h_);
      h_ = nullptr;
      throw hodlr_b200::Error(HODLR_ERR_CUDA, std::string("kernel functor fill: ") +
                                                  cudaGetErrorString(e));
    }
  }
#endif

  // The GPU form of the kernel constructor: K_ij = f(|x_i - x_j|) for points
  // pts (dim x numRows, SoA, host memory; copied).
  HODLR_Matrix(int numRows, int numCols, const hodlr_kernel_desc& kernel, const double* pts,
               int dim, int inputSizeThreshold = 30) {
    if (numRows != numCols)
      throw hodlr_b200::Error(HODLR_ERR_ARG, "only square kernel matrices form a HODLR tree");
    hodlr_b200::check(nullptr,
                      hodlr_create_kernel(&h_, numRows, dim, pts, &kernel, inputSizeThreshold),
                      "HODLR_Matrix(kernel)");
    n_ = numRows;
  }

  // With a user_IndexTree (reference :85 dense, :184 kernel)
  HODLR_Matrix(const hodlr_b200::Matrix& A, int inputSizeThreshold, user_IndexTree& input_IndexTree)
      : HODLR_Matrix(A, inputSizeThreshold) {
    set_tree(input_IndexTree);
  }
#ifdef HODLR_B200_HAVE_EIGEN
  HODLR_Matrix(Eigen::MatrixXd& A, int inputSizeThreshold, user_IndexTree& input_IndexTree)
      : HODLR_Matrix(A, inputSizeThreshold) {
    set_tree(input_IndexTree);
  }
#endif
  HODLR_Matrix(int numRows, int numCols, const hodlr_kernel_desc& kernel, const double* pts,
               int dim, int inputSizeThreshold, user_IndexTree& input_IndexTree)
      : HODLR_Matrix(numRows, numCols, kernel, pts, dim, inputSizeThreshold) {
    set_tree(input_IndexTree);
  }

  HODLR_Matrix(const HODLR_Matrix&) = delete;
  HODLR_Matrix& operator=(const HODLR_Matrix&) = delete;
  HODLR_Matrix(HODLR_Matrix&& o) noexcept : h_(o.h_), n_(o.n_) { o.h_ = nullptr; }
  ~HODLR_Matrix() { hodlr_destroy(h_); }

  // ---------------------------------------------------- attribute setters
  void set_LRTolerance(double tolerance) {
    hodlr_b200::check(h_, hodlr_set_lr_tolerance(h_, tolerance), "set_LRTolerance");
  }
  void set_minPivot(double minPivot) {
    hodlr_b200::check(h_, hodlr_set_min_pivot(h_, minPivot), "set_minPivot");
  }
  void set_LRMethod(const std::string& method) {
    hodlr_b200::check(h_, hodlr_set_lr_method(h_, method.c_str()), "set_LRMethod");
  }

  // ------------------------------------------------------------- solvers
  void storeLRinTree() { hodlr_b200::check(h_, hodlr_compress(h_), "storeLRinTree"); }
  void recLU_Compute() {
    form(HODLR_FORM_RECLU);
    hodlr_b200::check(h_, hodlr_factorize(h_), "recLU_Compute");
  }

  hodlr_b200::Matrix recLU_Solve(const hodlr_b200::Matrix& input_RHS) {
    form(HODLR_FORM_RECLU);
    hodlr_b200::Matrix x(input_RHS.rows(), input_RHS.cols());
    solve_raw(input_RHS.rows(), input_RHS.cols(), input_RHS.data(), x.data());
    if (printResultInfo) print_result(input_RHS.cols(), input_RHS.data(), x.data());
    return x;
  }

  hodlr_b200::Matrix iterative_Solve(const hodlr_b200::Matrix& input_RHS, int maxIterations,
                                     double stop_tolerance, double init_LRTolerance,
                                     const std::string& input_LR_Method,
                                     const std::string& directSolve_Method = "recLU") {
    if (directSolve_Method != "recLU")
      throw hodlr_b200::Error(HODLR_ERR_UNSUPPORTED, "only the recLU direct solver is on the GPU path");
    set_LRTolerance(init_LRTolerance);
    set_LRMethod(input_LR_Method);
    hodlr_b200::Matrix x(input_RHS.rows(), input_RHS.cols());
    std::vector<double> rel(input_RHS.cols());
    int iters = 0;
    hodlr_b200::check(h_,
                      hodlr_iterative_solve(h_, input_RHS.cols(), input_RHS.data(), input_RHS.rows(),
                                            x.data(), input_RHS.rows(), stop_tolerance,
                                            maxIterations, 32, &iters, rel.data()),
                      "iterative_Solve");
    last_iterations_ = iters;
    return x;
  }

  // recSM_Solve (reference :215, src/HODLR_Matrix.cpp:805-841): the recursive
  // Sherman-Morrison (perturbI) factorization and its solve
  hodlr_b200::Matrix recSM_Solve(const hodlr_b200::Matrix& input_RHS) {
    form(HODLR_FORM_RECSM);
    hodlr_b200::Matrix x(input_RHS.rows(), input_RHS.cols());
    solve_raw(input_RHS.rows(), input_RHS.cols(), input_RHS.data(), x.data());
    if (printResultInfo) print_result(input_RHS.cols(), input_RHS.data(), x.data());
    return x;
  }

#ifdef HODLR_B200_HAVE_EIGEN
  Eigen::MatrixXd recSM_Solve(const Eigen::MatrixXd& input_RHS) {
    form(HODLR_FORM_RECSM);
    Eigen::MatrixXd b = input_RHS;
    Eigen::MatrixXd x(b.rows(), b.cols());
    solve_raw((int)b.rows(), (int)b.cols(), b.data(), x.data());
    if (printResultInfo) print_result((int)b.cols(), b.data(), x.data());
    return x;
  }

  Eigen::MatrixXd recLU_Solve(const Eigen::MatrixXd& input_RHS) {
    form(HODLR_FORM_RECLU);
    Eigen::MatrixXd b = input_RHS;  // contiguous, column-major
    Eigen::MatrixXd x(b.rows(), b.cols());
    solve_raw((int)b.rows(), (int)b.cols(), b.data(), x.data());
    if (printResultInfo) print_result((int)b.cols(), b.data(), x.data());
    return x;
  }
#endif

  // determinant() / logAbsDeterminant()  (reference :248-249)
  double logAbsDeterminant() {
    double v = 0;
    int sign = 1;
    hodlr_b200::check(h_, hodlr_logdet(h_, &v, &sign), "logAbsDeterminant");
    return v;
  }
  double determinant() {
    double v = 0;
    int sign = 1;
    hodlr_b200::check(h_, hodlr_logdet(h_, &v, &sign), "determinant");
    return sign * std::exp(v);
  }

  // ------------------------------------------------------------- getters
  double get_LR_ComputationTime() const { return times()[0]; }
  double get_recLU_FactorizationTime() const { return times()[1]; }
  double get_recLU_SolveTime() const { return times()[2]; }
  double get_recLU_TotalTime() const { return times()[3]; }
  double get_MatrixSize() const { return n_; }
  int rows() const { return n_; }
  int cols() const { return n_; }
  int last_iterations() const { return last_iterations_; }
  hodlr_t handle() const { return h_; }

 private:
  hodlr_t h_ = nullptr;
  int n_ = 0;
  int last_iterations_ = 0;

  void set_tree(const user_IndexTree& t) {
    std::vector<int> split, left, right, b[4];
    t.flatten(split, left, right, b);
    hodlr_b200::check(h_,
                      hodlr_set_index_tree_bounds(h_, (int)split.size(), split.data(),
                                                  left.data(), right.data(), b[0].data(),
                                                  b[1].data(), b[2].data(), b[3].data()),
                      "user_IndexTree");
  }

  void form(int f) { hodlr_b200::check(h_, hodlr_set_solver_form(h_, f), "solver form"); }

  void solve_raw(int rows, int nrhs, const double* b, double* x) {
    if (rows != n_) throw hodlr_b200::Error(HODLR_ERR_ARG, "right-hand side has the wrong number of rows");
    hodlr_b200::check(h_, hodlr_solve(h_, nrhs, b, rows, x, rows), "recLU_Solve");
  }

  std::vector<double> times() const {
    std::vector<double> t(4, 0.0);
    hodlr_get_times(h_, &t[0], &t[1], &t[2], &t[3]);
    return t;
  }

  // The printResultInfo report of recLU_Solve (src/HODLR_Matrix.cpp:776-788).
  void print_result(int nrhs, const double* b, const double* x) {
    std::vector<double> rel(nrhs);
    hodlr_b200::check(h_, hodlr_residual(h_, nrhs, b, n_, x, n_, rel.data()), "residual");
    double worst = 0;
    for (double r : rel) worst = r > worst ? r : worst;
    std::vector<double> t = times();
    std::printf("**************************************************\n");
    std::printf("Solver Type                      = recLU\n");
    std::printf("Low-Rank Computation Time        = %g seconds\n", t[0]);
    std::printf("Factorization Time               = %g seconds\n", t[1]);
    std::printf("Solve Time                       = %g seconds\n", t[2]);
    std::printf("Total Solve Time                 = %g seconds\n", t[3]);
    std::printf("Residual l2 Relative Error       = %g\n", worst);
  }
};

#endif  // HODLR_B200_HODLR_MATRIX_HPP
