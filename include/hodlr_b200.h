/*
 * hodlr_b200.h -- C ABI of the B200 HODLR direct solver.
 *
 * Drop-in boundary for the recLU hot path of amiraa127/Dense_HODLR: kernel
 * matrix assembly, partial-pivot ACA compression of every off-diagonal
 * block, recursive LU / Sherman-Morrison-Woodbury factorization and solve.
 * Every entry point names the reference interface it replaces
 * (include/HODLR_Matrix.hpp unless stated).  Plain pointers and sizes only;
 * matrices are column-major FP64.  Every call returns an int status
 * (HODLR_OK == 0).  A handle is used by one host thread at a time; all its
 * GPU work runs on one CUDA stream.  There is no CPU fallback: without a
 * usable GPU, hodlr_create_* returns HODLR_ERR_CUDA.
 */
#ifndef HODLR_B200_H
#define HODLR_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hodlr_handle_s* hodlr_t;

/* status codes */
#define HODLR_OK 0
#define HODLR_ERR_ARG 1         /* invalid argument */
#define HODLR_ERR_CUDA 2        /* CUDA runtime error / no device */
#define HODLR_ERR_ALLOC 3       /* device memory exhausted */
#define HODLR_ERR_UNSUPPORTED 4 /* feature not available on the GPU path */
#define HODLR_ERR_SINGULAR 5    /* exact-zero pivot in a leaf or capacitance LU */
#define HODLR_ERR_STATE 6       /* call out of order */
#define HODLR_ERR_NONFINITE 7   /* a NaN/Inf matrix entry or residual */
#define HODLR_ERR_TIMEOUT 8     /* a bounded device wait gave up */
#define HODLR_ERR_IO 9          /* a file could not be opened, read or written */
#define HODLR_ERR_CHECK 10      /* checked mode: an extent or index outside its buffer */

/* kernel families: K_ij = f(r_ij) (+ shift on the diagonal) */
#define HODLR_KERNEL_GAUSSIAN 0          /* exp(-r^2/l^2) */
#define HODLR_KERNEL_MATERN32 1          /* (1+sqrt(3)r/l) exp(-sqrt(3)r/l) */
#define HODLR_KERNEL_INV_MULTIQUADRIC 2  /* 1/sqrt(1+r^2/l^2) */
#define HODLR_KERNEL_QUADRATIC 3         /* 1 + r^2/l^2 */
#define HODLR_KERNEL_EXPONENTIAL 4       /* exp(-r/l) */

typedef struct {
  int type;            /* HODLR_KERNEL_* */
  double length_scale; /* l */
  double diag_shift;   /* K_ii = f(0) + diag_shift   (diag_replace == 0) */
  int diag_replace;    /* 1: K_ii = diag_value instead */
  double diag_value;
} hodlr_kernel_desc;

/* Low-rank methods (set_LRMethod strings of the reference). */
#define HODLR_LR_PARTIAL_PIV_ACA 0 /* "partialPiv_ACA", the only GPU method */

/* HODLR_Matrix(int numRows, int numCols, double (*kernel)(int,int,void*),
 *              void* data, int leaf = 30)                         (:162)
 * The entry functor becomes a closed-form kernel of points: pts holds dim
 * rows of n coordinates (SoA, pts[d*n + i]), host memory, copied.  dim <= 3. */
int hodlr_create_kernel(hodlr_t* out, int n, int dim, const double* pts,
                        const hodlr_kernel_desc* kernel, int leaf_size);

/* HODLR_Matrix(Eigen::MatrixXd& A, int leaf = 30,
 *              std::string LR_Method = "partialPiv_ACA")           (:76)
 * A is n x n column-major host memory with leading dimension lda, copied. */
int hodlr_create_dense(hodlr_t* out, int n, const double* A, int lda, int leaf_size);

/* HODLR_Matrix(int, int, double (*)(int,int,void*), void*, int)     (:162)
 * in its device-functor form: a dense handle whose n x n column-major FP64
 * matrix lives in device memory owned by the handle, left uninitialised.
 * *dA receives its address and *ld its leading dimension (n).  The caller
 * writes every entry K(i, j) = dA[i + j * ld] on the device (the C++ facade
 * launches a kernel evaluating a __device__ functor, compiled in the caller's
 * translation unit) and completes that work before the next call on the
 * handle; from then on the handle behaves as hodlr_create_dense's.  Memory
 * is n^2 doubles: entries are stored, not regenerated. */
int hodlr_create_dense_device(hodlr_t* out, int n, int leaf_size, double** dA, int64_t* ld);

/* HODLR_Matrix(int, int, double (*)(int,int,void*), void*, int)     (:162)
 * with an arbitrary host function: returns HODLR_ERR_UNSUPPORTED, because a
 * host function pointer cannot be evaluated by GPU kernels.  Use
 * hodlr_create_kernel (closed-form kernels) or hodlr_create_dense. */
int hodlr_create_fnptr(hodlr_t* out, int rows, int cols,
                       double (*kernel)(int, int, void*), void* data, int leaf_size);

void hodlr_destroy(hodlr_t h);

/* reset_attributes() (src/HODLR_Matrix.cpp:1232-1246): discard the
 * compression and the factorization so the next call recomputes them. */
int hodlr_reset(hodlr_t h);

/* Run all GPU work of the handle on `stream` (a cudaStream_t); NULL restores
 * the handle's own stream.  The caller keeps ownership of the stream. */
int hodlr_set_stream(hodlr_t h, void* stream);

/* set_LRTolerance(double) (:222); default 1e-6.  A changed value discards the
 * compression and the factorization (reset_attributes,
 * src/HODLR_Matrix.cpp:1232-1257). */
int hodlr_set_lr_tolerance(hodlr_t h, double tol);
/* set_minPivot(double) (:223); truncated to int as the reference does when it
 * passes it to ACA (include/lowRank.hpp:25). */
int hodlr_set_min_pivot(hodlr_t h, double min_pivot);
/* set_LRMethod(std::string) (:225): "partialPiv_ACA" only, else
 * HODLR_ERR_UNSUPPORTED. */
int hodlr_set_lr_method(hodlr_t h, const char* method);

/* storeLRinTree() (:211): ACA of every off-diagonal block. */
int hodlr_compress(hodlr_t h);
/* recLU_Compute() (:217): compression (if needed) + recLU_Factorize. */
int hodlr_factorize(hodlr_t h);
/* recLU_Solve(const Eigen::MatrixXd&) (:214): compresses and factors on
 * first use, then solves.  b and x are host memory, n x nrhs. */
int hodlr_solve(hodlr_t h, int nrhs, const double* b, int ldb, double* x, int ldx);
/* Same with device pointers (no host copies). */
int hodlr_solve_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                       int ldx);

/* Iterative refinement to a residual target: the direct recLU solve, then
 * x += recLU_Solve(b - K x) with the full FP64 kernel residual
 * (kernelMatrix::operator*, src/kernel.cpp:27-35) until
 * max_c ||b_c - K x_c|| / ||b_c|| <= tol or max_iter corrections.  The
 * reference offers refinement only for dense input (iterative_Solve,
 * src/HODLR_Matrix.cpp:1138-1213, GMRES with the HODLR preconditioner);
 * this is its kernel-matrix form.  *iters = corrections applied; relres[c]
 * the final relative residual of column c.  Device pointers. */
int hodlr_solve_refined_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                               int ldx, double tol, int max_iter, int* iters, double* relres);
/* Same with host buffers. */
int hodlr_solve_refined(hodlr_t h, int nrhs, const double* b, int ldb, double* x, int ldx,
                        double tol, int max_iter, int* iters, double* relres);

/* iterative_Solve(rhs, maxIterations, stop_tolerance, ...) (:219,
 * src/HODLR_Matrix.cpp:1138-1213): GMRES(restart) preconditioned by the HODLR
 * factor, starting from the recLU solution.  The reference runs IML GMRES
 * with left preconditioning on dense input only; here the preconditioner is
 * applied on the right so that the stopping test is the relative residual
 * max_c ||b_c - K x_c|| / ||b_c|| <= tol of the iterate itself: the residual
 * of the initial guess comes from one full-kernel product, and each cycle's
 * update x += Z y is matched by r -= (K Z) y with the products the iterations
 * computed (no further product for the test).  The full-kernel product is
 * FP64 with entries generated on the fly, and all right-hand sides iterate
 * together.  *iters = GMRES iterations (full-kernel products after the
 * first residual).  Device pointers; the second form takes host buffers. */
int hodlr_iterative_solve_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                                 int ldx, double tol, int max_iter, int restart, int* iters,
                                 double* relres);
int hodlr_iterative_solve(hodlr_t h, int nrhs, const double* b, int ldb, double* x, int ldx,
                          double tol, int max_iter, int restart, int* iters, double* relres);

/* kernelMatrix::operator* (src/kernel.cpp:27-35): d_y = K d_x, FP64, entries
 * generated on the fly (device pointers). */
int hodlr_kernel_matvec_device(hodlr_t h, int nrhs, const double* d_x, int ldx,
                               double* d_y, int ldy);
/* The printResultInfo residual (src/HODLR_Matrix.cpp:785-787) per column:
 * relres[c] = ||K x_c - b_c||_2 / ||b_c||_2, full kernel in FP64.  Host
 * buffers. */
int hodlr_residual(hodlr_t h, int nrhs, const double* b, int ldb, const double* x,
                   int ldx, double* relres);

/* get_LR_ComputationTime / get_recLU_FactorizationTime / get_recLU_SolveTime /
 * get_recLU_TotalTime (:234-241), seconds of device time (CUDA events). */
int hodlr_get_times(hodlr_t h, double* lr, double* factor, double* solve, double* total);

/* Tree and block introspection.  Blocks are numbered 2p (top off-diagonal)
 * and 2p+1 (bottom off-diagonal) for inner node p in level order, the order
 * of HODLR_Tree::nodeLevelVec (include/HODLR_Tree.hpp:86). */
int hodlr_get_num_levels(hodlr_t h, int* levels); /* inner levels */
int hodlr_get_num_blocks(hodlr_t h, int* blocks);
int hodlr_get_block_info(hodlr_t h, int block, int* level, int* row0, int* col0, int* m,
                         int* n, int* rank, int* iters);
int hodlr_get_ranks(hodlr_t h, int* ranks);
/* ACA pivot (row, column) of each stored step, block-local indices. */
int hodlr_get_pivots(hodlr_t h, int block, int* rows, int* cols, int* count);
/* Low-rank factors of a block: W (m x rank) and V (n x rank), host memory. */
int hodlr_get_lowrank(hodlr_t h, int block, double* W, double* V);
/* Smallest |eps - tol| / tol met by the block's stopping tests, and how many
 * of them were within 1e-10 (ranks can differ from a CPU run only there). */
int hodlr_get_block_margin(hodlr_t h, int block, double* margin, int* near);

/* ACA kernel statistics of the last compression: launches, summed device
 * time (seconds) and algorithmic bytes: per block and step t, one read of
 * the W and V panels (8 t (m+n) bytes; the norm-update dots ride along), the
 * two new columns (8 (m+n)) and the coordinates of the entries evaluated
 * (8 dim (m+n)). */
int hodlr_get_aca_stats(hodlr_t h, int* launches, double* seconds, double* bytes);

/* Initial number of low-rank columns to allocate per inner level (caps[l],
 * 0 = default).  ACA grows a level that needs more and resumes its blocks
 * where they stopped, so a hint changes memory traffic, never results.  The
 * reference grows W and V by doubling inside partialPivACA_LowRankApprox
 * (src/lowRank.cpp:151-157). */
int hodlr_set_capacity_hint(hodlr_t h, const int* caps, int nlevels);

/* Device memory of all handles on the current device comes from one
 * stream-ordered pool owned by the library; memory that hodlr_destroy frees
 * stays reserved there for the next handle.  This returns it to the driver
 * (after a device synchronise).  No reference counterpart: the reference
 * allocates host memory per object. */
int hodlr_trim_device_memory(void);

/* ------------------------------------------------------------------------
 * Forests of independent systems.  No reference counterpart: the reference
 * solves one HODLR_Matrix per object.  nsys systems with sizes[q] points
 * each, concatenated in pts (dim x sum(sizes), SoA, each system's points
 * contiguous and ordered as the caller wants its tree), kernels[q] the
 * kernel of system q (point dimensions below `dim` are padded with zeros by
 * the caller).  Every system gets the tree the reference would build for it
 * alone; all systems' roots sit at level 0, so each level's ACA launch,
 * batched leaf LUs, GEMMs and capacitance LUs span all systems, and the
 * full-kernel product is block diagonal.  Every entry point above works on a
 * forest (global point and row indices; the matrix is block diagonal).
 * ------------------------------------------------------------------------ */
int hodlr_create_forest(hodlr_t* out, int nsys, const int* sizes, int dim, const double* pts,
                        const hodlr_kernel_desc* kernels, int leaf_size);
int hodlr_get_num_systems(hodlr_t h, int* nsys);

/* log|det K| and the sign of det K from the factorization (factors first if
 * needed): the product of the leaf determinants and of every node's
 * capacitance determinant.  Replaces logAbsDeterminant() / determinant()
 * (include/HODLR_Matrix.hpp:248-249; src/HODLR_Matrix.cpp:1661-1697, which
 * reach the same determinant through recSM_Factorize and perturbI nodes; its
 * signed value omits the row permutations, this one does not). */
int hodlr_logdet(hodlr_t h, double* log_abs_det, int* sign);

/* Factorization form.  HODLR_FORM_RECLU (default): recLU_Factorize /
 * recLU_Solve (src/HODLR_Matrix.cpp:612-755), each node's Schur system with
 * the bottom block's rank first.  HODLR_FORM_RECSM: recSM_Factorize /
 * recSM_Solve (src/HODLR_Matrix.cpp:520-610,805-841), each node a perturbed
 * identity I + U V^T (src/perturbI.cpp:15-59) whose K^-1 U panels come from
 * the descendants' inverses applied level by level and whose capacitance
 * system I + V^T U has the top block's rank first.  Both run the same
 * level-batched kernels; the form decides the capacitance systems (and so
 * their pivots and the rounding of the solution, not its value).  Changing
 * the form drops the factorization (the compression is kept); every solve,
 * refinement and log-determinant entry point then uses the new form. */
#define HODLR_FORM_RECLU 0
#define HODLR_FORM_RECSM 1
int hodlr_set_solver_form(hodlr_t h, int form);
int hodlr_get_solver_form(hodlr_t h, int* form);

/* User index tree, replacing the constructors that take a user_IndexTree
 * (include/HODLR_Matrix.hpp:85,184; built by userTree_To_HODLRTree,
 * src/HODLR_Tree.cpp:207-327).  Nodes in pre-order, node 0 the root covering
 * all rows: split[i] is the last row of node i's top half (-1: none; a node
 * no larger than the leaf size with no split is a leaf), left[i] and
 * right[i] its child nodes (both -1: default subtrees below, the right one
 * with floor(s/2) rows on top as in the reference).  The low-rank method of
 * user_IndexTree::node is not taken: partial-pivot ACA with the handle's
 * tolerance on every block.  Discards any compression; one-system handles
 * only.  Invalid trees return HODLR_ERR_ARG and leave the default tree. */
int hodlr_set_index_tree(hodlr_t h, int nnodes, const int* split, const int* left,
                         const int* right);
/* The same with user_IndexTree::node's rank bounds (include/user_IndexTree.hpp:
 * topOffDiag_minRank, bottOffDiag_minRank, topOffDiag_maxRank,
 * bottOffDiag_maxRank; src/HODLR_Tree.cpp:241-244), one value per user node,
 * -1 for none: ACA continues while the rank is below the minimum (even past
 * the tolerance) and stops at the maximum (src/lowRank.cpp:149,244-247).
 * Nodes of the default subtrees below a user leaf take no bounds.  All four
 * arrays or none. */
int hodlr_set_index_tree_bounds(hodlr_t h, int nnodes, const int* split, const int* left,
                                const int* right, const int* top_min, const int* bott_min,
                                const int* top_max, const int* bott_max);
/* Factor (if needed), direct solve, then iterative refinement with the FP64
 * residual until every system q has max_c ||b_c - K x_c|| / ||b_c|| <= tol
 * over its own rows (or max_iter corrections).  relres: nsys x nrhs,
 * system-major; a converged system's x is left unchanged afterwards, and its
 * rows leave the full-kernel product.  hodlr_iterative_solve(_device) on a
 * forest runs GMRES per system instead: every (system, column) pair has its
 * own inner products, Hessenberg matrix and stopping test on the system's
 * rows; relres[c] is then the worst system's residual of column c. */
int hodlr_forest_refine_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                               int ldx, double tol, int max_iter, int* iters, double* relres);

/* ------------------------------------------------------------------------
 * Learned rank predictor.  No reference counterpart: the reference learns
 * nothing and grows W and V by doubling as ACA runs
 * (src/lowRank.cpp:151-157).  A 14-64-64-1 MLP with GELU, BF16 with FP32
 * accumulation, maps a block's features -- the bounding-box centre (3) and
 * extent (3) of its row cluster, then of its column cluster (axes beyond
 * the points' dimension are 0), log l and log tol -- to log(1 + ACA rank).
 * Parameters are one FP32 blob of HODLR_MLP_PARAMS floats:
 * [mean(14) | inv_std(14) | W1 64x14 | b1(64) | W2 64x64 | b2(64) | W3(64) | b3],
 * row-major weights; inputs are standardised as (x - mean) * inv_std.
 * With a model set, hodlr_compress predicts every block's rank first, sizes
 * each level's W/V capacity from the predictions and starts the largest
 * predicted work first; ACA's own stopping test still decides every rank.
 * ------------------------------------------------------------------------ */
#define HODLR_MLP_INPUTS 14
#define HODLR_MLP_HIDDEN 64
#define HODLR_MLP_PARAMS 5213

/* Model for this handle (host blob; NULL removes it) and the kernel length
 * scale its log l feature uses.  Point-coordinate handles only. */
int hodlr_set_rank_model(hodlr_t h, const float* params, double length_scale);
/* Predicted rank of every block, in hodlr_get_block_info order. */
int hodlr_get_predicted_ranks(hodlr_t h, int* ranks);
/* Features of every block (num_blocks x 14, row-major, host) for training. */
int hodlr_block_features(hodlr_t h, double length_scale, float* features);

/* Device-side MLP: forward y[b] = MLP(X[b, :]) for X row-major batch x 14;
 * one training step (forward, backward, gradient summed over the batch in
 * sample order; Adam with beta 0.9/0.999, eps 1e-8 when lr > 0, step >= 1)
 * on loss 1/batch sum (y_b - T_b)^2, optional d_grad (trained parameters,
 * HODLR_MLP_PARAMS - 28 floats, blob order after the standardisation) and
 * d_loss (one float).  d_scratch holds hodlr_mlp_scratch_floats(batch)
 * floats; d_m1 and d_m2 are the Adam moments of the trained parameters.
 * The train step is asynchronous on `stream`. */
int hodlr_mlp_scratch_floats(int batch, long long* floats);
int hodlr_mlp_forward(const float* d_params, const float* d_X, int batch, float* d_y,
                      void* stream);
int hodlr_mlp_train_step(float* d_params, float* d_m1, float* d_m2, const float* d_X,
                         const float* d_T, int batch, float* d_scratch, float lr, int step,
                         float* d_grad, float* d_loss, void* stream);

/* Arithmetic of the Woodbury products (V^T K^-1 U, V^T X and the updates)
 * in the factorization and the solve.  FP64 (default) reproduces the
 * reference; TF32 and BF16 run them on the tcgen05 tensor cores with FP32
 * accumulation (the mixed-precision form) while leaf and capacitance LUs,
 * their pivoting and the full-kernel residual stay FP64; GMRES
 * (hodlr_iterative_solve) recovers full accuracy when cond(K) * u is well
 * below 1 (u = 4.9e-4 for TF32, 3.9e-3 for BF16).  TF32X3 splits each
 * operand into TF32 head and tail and sums three tensor-core products
 * (about FP32 accuracy, u ~ 1e-7) for ill-conditioned systems.  Changing it
 * discards the factorization, not the compression. */
#define HODLR_PRECISION_FP64 0
#define HODLR_PRECISION_TF32 1
#define HODLR_PRECISION_BF16 2
#define HODLR_PRECISION_TF32X3 3
int hodlr_set_precision(hodlr_t h, int precision);

/* One product in the given arithmetic, device pointers, column-major:
 * mode 0: C (m x n) = A^T B, A is k x m;  mode 1: C (m x n) -= A B, A is m x k;
 * B is k x n.  The Woodbury GEMM kernels as a utility (and their test hook). */
int hodlr_gemm_device(int precision, int mode, int m, int n, int k, const double* A, int lda,
                      const double* B, int ldb, double* C, int ldc, void* stream);

/* Memory of the factorization (no counterpart in the reference, which keeps
 * U and K^-1 U side by side in each node, include/HODLR_Tree.hpp:41-58).
 * K^-1 U of a level needs N x kmax doubles.  mode 1: it overwrites the
 * level's U panel (W) in place; mode 0: it always gets its own memory
 * (HODLR_ERR_ALLOC if there is none); mode -1 (default): its own memory when
 * that can be allocated, else in place.  Results are the same.  Once a level
 * is factored in place its W is gone: hodlr_get_lowrank returns
 * HODLR_ERR_STATE for its blocks, and a refactorization (another precision)
 * compresses again.  hodlr_get_factor_in_place reports how many levels the
 * last factorization overwrote. */
int hodlr_set_factor_in_place(hodlr_t h, int mode);

/* How the ACA of the few-block top levels reads its W/V panel slices (no
 * counterpart in the reference): on = 2 (default) streams them through
 * per-warp shared-memory rings (used when N is even), each ring tile of 128
 * rows x 4 columns filled by one 2D tensor copy; 1 fills the tiles with one
 * bulk copy per panel column; 0 loads the panels per thread.  Measured ACA
 * time at N = 262144, modes 2 / 1 / 0: 0.188 / 0.218 / 0.260 s (2D Matern
 * cloud, tol 1e-8), 9.0 / 10.3 / 12.3 s (sphere, tol 1e-10).  Pivots, ranks
 * and W/V are the same in every mode; the setting applies from the next
 * compression.  HODLR_ACA_STREAMING=0, 1 or 2 in the environment sets the
 * mode of every new handle. */
int hodlr_set_aca_streaming(hodlr_t h, int on);

/* Bounded device waits (no counterpart in the reference).  The CTAs of one
 * ACA block group meet at a barrier in global memory; a barrier that is not
 * complete after `polls` polls (0: the default, 2^26) gives up, the launch
 * ends and the call returns HODLR_ERR_TIMEOUT, leaving the handle usable.
 * unreachable = 1 makes every such barrier wait for one arrival more than
 * its group has -- a wait nothing completes -- so that this path can be
 * tested; set it back to 0 for normal work. */
int hodlr_set_wait_limit(hodlr_t h, unsigned polls, int unreachable);

/* Checked mode (no counterpart in the reference; a debugging aid).  on = 1:
 * before every grouped GEMM, capacitance and leaf launch the host verifies
 * that each operand's extent lies inside a live allocation of the handle,
 * the direct solve runs without its CUDA graph, and the stream is
 * synchronised after every launch group so that a device error names the
 * group that raised it.  A violation returns HODLR_ERR_CHECK without
 * launching.  The environment variable HODLR_CHECKED=1 turns it on for
 * every handle at creation.  Results are the same as unchecked; only
 * slower.  (Pivot and permutation indices are range-checked on the device
 * in every mode: an index outside its range skips the access and the call
 * returns HODLR_ERR_CHECK.) */
int hodlr_set_checked(hodlr_t h, int on);
int hodlr_get_factor_in_place(hodlr_t h, int* levels);

/* Number of kernels this handle has launched since it was created. */
int hodlr_get_launch_count(hodlr_t h, long long* count);

/* Dense-matrix files of the reference's binary format (include/matrixIO.hpp:38-53,
 * saveMatrixXdToBinary / readBinaryIntoMatrixXd, src/matrixIO.cpp:159-202):
 * two native int32 (rows, cols), then rows x cols FP64 values row by row.
 * Matrices here are column-major with leading dimension lda.  Host-only: no
 * GPU is needed.  HODLR_ERR_IO: the file cannot be opened, is short, or its
 * header holds negative sizes; HODLR_ERR_ARG: null pointers, lda < rows, or
 * (read) sizes other than the file's. */
int hodlr_matrix_file_dims(const char* path, int* rows, int* cols);
int hodlr_read_matrix_file(const char* path, int rows, int cols, double* A, int lda);
int hodlr_write_matrix_file(const char* path, int rows, int cols, const double* A, int lda);

/* Full-kernel FP64 product d_y = K d_x that allocates no device memory.  It
 * has no counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc when they need K x: applications whose memory manager has
 * already reserved the device memory (a new allocation would fail or break
 * their budget), plugins that must not allocate behind their host
 * framework's allocator, and latency-bound code that avoids cudaMalloc
 * because it can synchronise the device.  Such callers cannot create a
 * handle (handles allocate), so this call takes the points (d_pts, dim x n,
 * SoA, device memory), X and Y as caller-owned device buffers, runs on
 * `stream` (NULL: the default stream) and returns after synchronising that
 * stream.  Its scratch is a file-scope device array of
 * HODLR_NOALLOC_SPLITS * HODLR_NOALLOC_MAX_ELEMS doubles (16 MiB) that every
 * GPU loading the library holds until exit; hence the limit
 * n * nrhs <= HODLR_NOALLOC_MAX_ELEMS, beyond which the call returns
 * HODLR_ERR_ARG without launching.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress, with that device current):
 * make that first call before any stream capture begins.  All calls share
 * the array and it keeps the last call's contents (nothing in it needs to
 * start at zero); calls whose kernels overlap on the GPU race on it, so
 * issue them on one stream or serialise them.  A CUDA error already pending
 * from the caller's earlier work is left pending and the call returns
 * HODLR_ERR_STATE without launching. */
#define HODLR_NOALLOC_SPLITS 4
#define HODLR_NOALLOC_MAX_ELEMS 524288
int hodlr_kernel_matvec_noalloc(int n, int dim, const double* d_pts,
                                const hodlr_kernel_desc* kernel, int nrhs, const double* d_x,
                                int ldx, double* d_y, int ldy, void* stream);

const char* hodlr_status_string(int status);
const char* hodlr_last_error(hodlr_t h);

#ifdef __cplusplus
}
#endif

#endif /* HODLR_B200_H */
