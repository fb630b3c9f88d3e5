// Internal interface of the host orchestration units: the handle, its
// per-level device data, and the helpers the units share.
//
// Replaces, for the recLU path, HODLR_Matrix (include/HODLR_Matrix.hpp:38-413,
// src/HODLR_Matrix.cpp) and HODLR_Tree::createDefaultTree
// (src/HODLR_Tree.cpp:33-132).  The pointer tree of the reference becomes
// level arrays; the recursions of recLU_Factorize / recLU_Solve
// (src/HODLR_Matrix.cpp:612-755) become bottom-up sweeps over levels in which
// every node of a level is processed by one batched launch.
//
//   tree.cu      createDefaultTree / userTree_To_HODLRTree as level arrays
//   compress.cu  storeLRinTree: the ACA launches, level by level
//   factor.cu    recLU_Factorize: leaves, K^-1 U panels, capacitance LUs
//   solve.cu     recLU_Solve, refinement, GMRES, the full-kernel product
//   handle.cu    device memory, copies, error words, handle set-up
//   hodlr_capi.cu  the C ABI (include/hodlr_b200.h)
//
// HBM layout (N = matrix size, column-major, leading dimension N):
//   pts        dim x N coordinates (SoA)            or A  N x N dense input
//   W_l, V_l   N x kcap_l per inner level l: the blocks of a level tile the
//              rows (W) and the columns (V) of the matrix exactly once
//   Y_l        N x kmax_l per level (its own allocation, or the first kmax_l
//              columns of W_l, overwritten): K^-1 U of the level's nodes
//              (topDiagSoln_LR / bottDiagSoln_LR) after the factorization
//   leaf LU    sum over leaves of s^2, plus a row permutation (N ints)
//   S_l        per node (k_b + k_t)^2 capacitance LU + pivots
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/hodlr_b200.h"
#include "common.cuh"
#include "gemm.h"
#include "kmatvec.h"
#include "lu.h"
#include "rank_mlp.h"

int aca_launch(const AcaLaunch& L, int nt, int kcap_max, bool cooperative, cudaStream_t s);
int aca_max_coresident(int nt, int kcap_max, bool ring, bool f32, int* per_sm);
bool aca_dots_global(int nt, int kcap_max, bool ring, bool f32);
size_t aca_smem_bytes(int nt, int kcap_max, bool ring, bool f32);
int aca_ring_stages(int kcap_max);
bool aca_ring_tile_maps(AcaLaunch& L, const double* W, const double* V, int64_t n, int kcap);

namespace hodlr_impl {

struct DevPlan {  // a grouped GEMM uploaded to the device
  GemmProblem* probs = nullptr;
  int4* tiles = nullptr;
  int nprob = 0, ntiles = 0;
  int64_t ws_elems = 0;
  bool any_split = false;
};

struct Level {
  std::vector<int> nmin, nsplit, nmax;  // inner nodes of this level
  // per node: rank bounds of its top and bottom blocks (-1: none; set by a
  // user index tree, user_IndexTree::node, include/user_IndexTree.hpp)
  std::vector<int> tmin, bmin, tmax, bmax;
  int nblocks() const { return 2 * (int)nmin.size(); }
  int ub_max = 0;  // largest min(m, n) of the level's blocks
  int kcap = 0;
  double* W = nullptr;
  double* V = nullptr;
  unsigned char* cR = nullptr;
  unsigned char* cC = nullptr;
  int* prow = nullptr;
  int* pcol = nullptr;
  AcaState* d_st = nullptr;
  std::vector<AcaState> st;
  int G = 1;
  int kmax = 0, coff = 0;
  // K^-1 U of the level's blocks (N x kmax, ld N): its own allocation, or
  // (y_alias) the first kmax columns of W, overwritten in place
  double* Yl = nullptr;
  bool y_alias = false;
  // factorization
  double* S = nullptr;
  int* piv = nullptr;
  SchurNode* d_nodes = nullptr;
  std::vector<SchurNode> nodes;
  int max_sd = 0;
  DevPlan tn, nn;          // factor GEMMs
  int solve_nrhs = -1;     // nrhs the solve plans were built for
  DevPlan stn, snn;        // solve GEMMs
  SchurNode* d_snodes = nullptr;  // solve: r_off into the solve buffer
  int64_t zs_elems = 0;
};

inline void block_geom(const Level& L, int q, int& r0, int& c0, int& m, int& n) {
  int p = q >> 1;
  if ((q & 1) == 0) {  // top off-diagonal: rows [min, split], cols [split+1, max]
    r0 = L.nmin[p];
    c0 = L.nsplit[p] + 1;
    m = L.nsplit[p] - L.nmin[p] + 1;
    n = L.nmax[p] - L.nsplit[p];
  } else {  // bottom off-diagonal: rows [split+1, max], cols [min, split]
    r0 = L.nsplit[p] + 1;
    c0 = L.nmin[p];
    m = L.nmax[p] - L.nsplit[p];
    n = L.nsplit[p] - L.nmin[p] + 1;
  }
}


cudaMemPool_t device_pool();

// Device memory cache of one handle.  Freed blocks go to `pending` and become
// reusable only after the handle's stream has been synchronised, so a reused
// block is never still read by an earlier kernel or host copy.
// Per-handle cache on top of the device pool: buffers freed by the handle are
// reused by its next allocations of a similar size once its stream has
// drained (pending -> free).
struct DevPool {
  cudaMemPool_t mp = nullptr;
  std::multimap<size_t, void*> freeb, pending;
  std::unordered_map<void*, size_t> size;
  cudaError_t raw_alloc(void** p, size_t bytes, cudaStream_t s) {
    if (!mp) mp = device_pool();
    if (!mp) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(p, bytes, mp, s);
  }
  cudaError_t alloc(void** p, size_t bytes, cudaStream_t s) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (int pass = 0; pass < 2; ++pass) {
      auto it = freeb.lower_bound(bytes);
      if (it != freeb.end() && it->first <= bytes + bytes / 4 + (1u << 20)) {
        *p = it->second;
        freeb.erase(it);
        return cudaSuccess;
      }
      if (pass == 0 && !pending.empty()) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return e;
        freeb.insert(pending.begin(), pending.end());
        pending.clear();
      }
    }
    cudaError_t e = raw_alloc(p, bytes, s);
    if (e == cudaErrorMemoryAllocation) {  // give back every cache, retry once
      cudaGetLastError();
      release_free(s);
      for (auto& f : pending) {
        cudaFreeAsync(f.second, s);
        size.erase(f.second);
      }
      pending.clear();
      cudaStreamSynchronize(s);
      cudaMemPoolTrimTo(mp, 0);
      e = raw_alloc(p, bytes, s);
    }
    if (e == cudaSuccess) size[*p] = bytes;
    return e;
  }
  // the live allocation that holds [p, p + bytes), if any (checked mode)
  bool holds(const void* p, size_t bytes) const {
    const char* c = (const char*)p;
    for (auto& a : size) {
      const char* b = (const char*)a.first;
      if (c >= b && c + bytes <= b + a.second) return true;
    }
    return false;
  }
  void free(void* p) {
    auto it = size.find(p);
    if (it == size.end()) return;
    pending.insert({it->second, p});
  }
  void release_free(cudaStream_t s) {
    for (auto& f : freeb) {
      cudaFreeAsync(f.second, s);
      size.erase(f.second);
    }
    freeb.clear();
  }
  void release_all(cudaStream_t s) {
    for (auto& f : size) cudaFreeAsync(f.first, s);
    size.clear();
    freeb.clear();
    pending.clear();
    cudaStreamSynchronize(s);
  }
};

}  // namespace hodlr_impl

struct hodlr_handle_s {
  hodlr_impl::DevPool pool;
  // the direct solve as a CUDA graph, replayed while its key is unchanged
  cudaGraphExec_t sg_exec = nullptr;
  int sg_nrhs = -1;
  cudaStream_t sg_stream = nullptr;
  const void* sg_key[4] = {nullptr, nullptr, nullptr, nullptr};
  long sg_gen = -1;
  long long sg_launches = 0;
  bool sg_off = false;  // capture refused once: direct launches from then on
  long factor_gen = 0;
  // forest of independent systems (hodlr_create_forest); nsys == 0: one system
  int nsys = 0;
  std::vector<int> sys_off;  // nsys + 1 point offsets
  std::vector<hx_kparams> sys_kp;
  hx_kparams* d_kps = nullptr;
  int* d_psys = nullptr;
  int* d_sysoff = nullptr;  // nsys + 1 row offsets on the device (GMRES segments)
  int4* d_fitems = nullptr;  // full-kernel product work items, by kernel family
  int ftype_off[HX_FOREST_TYPES + 1] = {0};
  double* d_fnorm = nullptr;  // per-system residual and right-hand-side norms
  int* d_cta = nullptr;  // CTA -> block table of uneven ACA groups
  int cta_cap = 0;
  double* dotg = nullptr;  // ACA dot partials in global memory (large ranks)
  int64_t dotg_cap = 0;
  // rank predictor (rank_mlp.cu): FP32 parameter blob on the device, the
  // length scale its features use, and the last predictions (block order)
  float* d_model = nullptr;
  double model_l = 0.0;
  std::vector<int> pred;
  int n = 0, leaf = 30, dim = 0;
  bool dense = false;
  hx_kparams kp{};
  double* d_pts = nullptr;
  double* d_A = nullptr;
  double tol = 1e-6;
  int minPivot = 0;
  std::vector<hodlr_impl::Level> lv;
  std::vector<int> cap_hint;  // initial W/V columns per level (0 = default)
  int gemm_prec = HODLR_GEMM_FP64;  // arithmetic of the Woodbury products
  // group-level ACA panels through the warps' rings (per-thread loads: 3.59
  // TB/s on the sphere shape at N = 262144, 2.38 on the 2D cloud) ...
  bool aca_ring = true;
  // ... each ring tile one 2D tensor copy (4.87 and 3.30 TB/s) rather than
  // one bulk copy per column (4.28 and 2.85 TB/s); the same bits every way
  bool aca_ring_tile = true;
  // factorization form (hodlr_set_solver_form): false recLU's Schur systems
  // [bottom; top], true recSM's perturbI systems [top; bottom]
  bool sm_form = false;
  // checked mode (hodlr_set_checked): operand extents verified on the host
  // before launches, no solve graph, a sync + error check after each group
  bool checked = false;
  unsigned spin_limit = 0;       // polls of an ACA group barrier (0: HODLR_SPIN_LIMIT)
  bool bar_unreachable = false;  // ACA group barriers wait for one arrival too many
  std::vector<int> leaf_min, leaf_size;
  int* d_leaf_min = nullptr;
  int* d_leaf_size = nullptr;
  // user index tree (hodlr_set_index_tree): pre-order nodes, split index and
  // child indices (-1: none)
  std::vector<int> ut_split, ut_left, ut_right;
  std::vector<int> ut_tmin, ut_bmin, ut_tmax, ut_bmax;  // per user node, or empty
  int64_t* d_lu_off = nullptr;
  double* d_lu = nullptr;
  int* d_perm = nullptr;
  int smax = 0;
  int64_t C = 0;  // sum over levels of kmax: the columns of all K^-1 U panels
  // factor in place: -1 only when a separate K^-1 U panel cannot be
  // allocated, 0 never, 1 always (hodlr_set_factor_in_place)
  int in_place = -1;
  bool w_consumed = false;  // some level's W holds K^-1 U: recompress before refactoring
  // pinned host staging of uploads that do not wait for the stream (h2d_async)
  char* pin = nullptr;
  size_t pin_cap = 0, pin_used = 0;
  double* ws = nullptr;  // GEMM split-K / kmatvec workspace
  int64_t ws_cap = 0;
  double* Z = nullptr;  // per-level Schur right-hand sides (factor)
  int64_t z_cap = 0;
  double* X = nullptr;  // solve panel N x nrhs
  int x_cols = 0;
  double* ir_b = nullptr;  // refinement: right-hand sides, iterate, K x, partial norms
  double* ir_x = nullptr;
  double* ir_y = nullptr;
  double* ir_part = nullptr;
  int ir_cols = 0;
  double* gm_V = nullptr;  // GMRES bases: (m+1) and m panels of N x nrhs
  double* gm_Z = nullptr;
  double* gm_W = nullptr;  // the products K Z_j (m panels): the residual's update
  double* gm_h = nullptr;  // small device buffers of coefficients / partials
  double* gm_part = nullptr;
  int gm_m = 0, gm_cols = 0;
  double* zs = nullptr;  // solve Schur right-hand sides
  int64_t zs_cap = 0;
  double* part = nullptr;
  int64_t part_cap = 0;
  unsigned* bar = nullptr;
  int bar_cap = 0;
  AcaBlock* d_blocks = nullptr;
  int blocks_cap = 0;
  unsigned* d_err = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  long long nlaunch = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int num_sms = 0;
  bool compressed = false, factored = false;
  double t_lr = 0, t_fact = 0, t_solve = 0, t_total = 0;
  int aca_launches = 0;
  double aca_seconds = 0, aca_bytes = 0;
  std::string err;
};

namespace hodlr_impl {

// Internal status (never returned by the C ABI): a cooperative launch was
// refused as too large and may be retried with fewer CTAs.
constexpr int HODLR_ERR_RETRY_SMALLER = 1000;

#define CK(call)                                               \
  do {                                                         \
    cudaError_t e__ = (call);                                  \
    if (e__ != cudaSuccess) return cuda_fail(h, e__, #call);   \
  } while (0)

template <class T>
cudaError_t dalloc(hodlr_t h, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return h->pool.alloc((void**)p, sizeof(T) * count, h->stream);
}

template <class T>
void dfree(hodlr_t h, T*& p) {
  if (p) h->pool.free((void*)p);
  p = nullptr;
}

int fail(hodlr_t h, int code, const std::string& msg);
int cuda_fail(hodlr_t h, cudaError_t e, const char* where);
void free_plan(hodlr_t h, DevPlan& p);
void drop_solve_graph(hodlr_t h);
void free_factor(hodlr_t h);
void free_compress(hodlr_t h);
void push_inner_node(hodlr_t h, int level, int mn, int split, int mx, int u = -1);
void build_subtree(hodlr_t h, int o, int N);
void grow_default(hodlr_t h, int level, int mn, int split, int mx);
bool user_subtree(hodlr_t h, int level, int mn, int mx, int u, std::vector<char>& seen);
void build_tree(hodlr_t h);
int ensure_ws(hodlr_t h, int64_t elems);
cudaError_t h2d(hodlr_t h, void* dst, const void* src, size_t bytes);
// Upload without waiting: src is copied into the handle's pinned staging
// memory at once (src may be reused on return) and the copy is queued.
cudaError_t h2d_async(hodlr_t h, void* dst, const void* src, size_t bytes);
cudaError_t d2h(hodlr_t h, void* dst, const void* src, size_t bytes);
cudaError_t copy2d(hodlr_t h, void* dst, size_t dpitch, const void* src, size_t spitch,
                   size_t width, size_t rows, cudaMemcpyKind kind);
int check_dev_err(hodlr_t h, const char* where);
// Checked mode: synchronise and check the error word after a launch group.
int check_phase(hodlr_t h, const char* where);
// Checked mode: [p, p + bytes) lies inside a live allocation of the handle.
int check_extent(hodlr_t h, const void* p, size_t bytes, const char* what, const char* where);
// Checked mode: every operand of a grouped GEMM (tn: C = A^T B, else C (-)= A B)
// and its split-K slice of the workspace.
int check_gemm(hodlr_t h, const std::vector<GemmProblem>& probs, bool tn, const char* where);
EntrySrc make_src(hodlr_t h);
int grow_level(hodlr_t h, Level& L, int cap);
void fill_block(hodlr_t h, Level& L, int q, AcaBlock& B);
bool level_done(const Level& L);
int run_aca(hodlr_t h, std::vector<AcaBlock>& blocks, int G, int nt, int kcap_max,
            bool ring = false, const std::vector<int>* groups = nullptr,
            const Level* arena = nullptr);
int init_level(hodlr_t h, Level& L, int cap);
int sync_level(hodlr_t h, Level& L, bool* done);
int level_kmax(const Level& L);
std::vector<int4> block_geoms(hodlr_t h);
int block_features_dev(hodlr_t h, const std::vector<int4>& geom, double l, float* d_F);
int predict_ranks(hodlr_t h);
int do_compress(hodlr_t h);
int upload_plan(hodlr_t h, std::vector<GemmProblem>& probs, bool split, DevPlan& out,
                const char* what = "grouped GEMM");
int level_rank(const Level& L, int q);
int run_tn(hodlr_t h, const DevPlan& P);
int run_nn(hodlr_t h, const DevPlan& P);
int do_factorize(hodlr_t h);
int do_logdet(hodlr_t h, double* log_abs_det, int* sign);
int build_solve_plans(hodlr_t h, int nrhs);
int solve_in_place(hodlr_t h, int nrhs);
int solve_fast(hodlr_t h, int nrhs);
int do_solve_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                    bool host_io);
// skip (forest only, device): per-system flags of systems whose rows are left out
int kmatvec_dev(hodlr_t h, int nrhs, const double* d_x, int ldx, double* d_y, int ldy,
                const unsigned char* skip = nullptr);
int refine_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                  double tol, int max_iter, int* iters, double* relres);
int forest_refine_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                         double tol, int max_iter, int* iters, double* relres);
int gm_dots(hodlr_t h, const double* V, int nv, const double* W, int nrhs, std::vector<double>& out);
int gm_sub(hodlr_t h, const double* V, int nv, const std::vector<double>& coef, double* W, int nrhs);
int gm_scale(hodlr_t h, const double* X, const std::vector<double>& sc, double* Y, int nrhs);
int gmres_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                 double tol, int max_iter, int m, int* iters, double* relres);
int init_common(hodlr_t h);

}  // namespace hodlr_impl
