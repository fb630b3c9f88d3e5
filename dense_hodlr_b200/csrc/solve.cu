// recLU_Solve (src/HODLR_Matrix.cpp:694-755), captured as a CUDA graph;
// iterative refinement and HODLR-preconditioned GMRES (iterative_Solve,
// src/HODLR_Matrix.cpp:1138-1213) on the full-kernel FP64 residual.
#include "handle.h"

namespace hodlr_impl {

int build_solve_plans(hodlr_t h, int nrhs) {
  const int64_t N = h->n;
  int64_t zs_tot = 0;
  for (auto& L : h->lv) {
    int64_t t = 0;
    for (auto& sn : L.nodes) t += (int64_t)(sn.kb + sn.kt) * nrhs;
    zs_tot = std::max(zs_tot, t);
  }
  if (zs_tot > h->zs_cap) {
    dfree(h, h->zs);
    CK(dalloc(h, &h->zs, (size_t)zs_tot));
    h->zs_cap = zs_tot;
  }
  if (nrhs > h->x_cols) {
    dfree(h, h->X);
    CK(dalloc(h, &h->X, (size_t)(N * nrhs)));
    h->x_cols = nrhs;
  }
  for (auto& L : h->lv) {
    if (L.solve_nrhs == nrhs) continue;
    const int nn = (int)L.nmin.size();
    std::vector<SchurNode> sn = L.nodes;
    int64_t off = 0;
    for (auto& s : sn) {
      s.r_off = off;
      off += (int64_t)(s.kb + s.kt) * nrhs;
    }
    dfree(h, L.d_snodes);
    CK(dalloc(h, &L.d_snodes, (size_t)nn));
    CK(h2d_async(h, L.d_snodes, sn.data(), sizeof(SchurNode) * nn));
    std::vector<GemmProblem> tn, up;
    for (int p = 0; p < nn; ++p) {
      const int sd = sn[p].kb + sn[p].kt;
      const int mn = L.nmin[p], sp = L.nsplit[p], mx = L.nmax[p];
      GemmProblem a{};
      a.A = L.V + mn;
      a.M = sn[p].kb;
      a.K = sp - mn + 1;
      a.lda = (int)N;
      a.B = h->X + mn;
      a.N = nrhs;
      a.ldb = (int)N;
      a.C = h->zs + sn[p].r_off + (h->sm_form ? sn[p].kt : 0);
      a.ldc = sd;
      tn.push_back(a);
      GemmProblem b{};
      b.A = L.V + sp + 1;
      b.M = sn[p].kt;
      b.K = mx - sp;
      b.lda = (int)N;
      b.B = h->X + sp + 1;
      b.N = nrhs;
      b.ldb = (int)N;
      b.C = h->zs + sn[p].r_off + (h->sm_form ? 0 : sn[p].kb);
      b.ldc = sd;
      tn.push_back(b);
      GemmProblem c{};
      c.C = h->X + mn;
      c.ldc = (int)N;
      c.A = L.Yl + mn;
      c.lda = (int)N;
      c.M = sp - mn + 1;
      c.K = sn[p].kt;
      c.B = h->zs + sn[p].r_off + (h->sm_form ? 0 : sn[p].kb);
      c.ldb = sd;
      c.N = nrhs;
      up.push_back(c);
      GemmProblem d{};
      d.C = h->X + sp + 1;
      d.ldc = (int)N;
      d.A = L.Yl + sp + 1;
      d.lda = (int)N;
      d.M = mx - sp;
      d.K = sn[p].kb;
      d.B = h->zs + sn[p].r_off + (h->sm_form ? sn[p].kt : 0);
      d.ldb = sd;
      d.N = nrhs;
      up.push_back(d);
    }
    int rc = upload_plan(h, tn, true, L.stn, "solve: V^T X products");
    if (rc) return rc;
    rc = upload_plan(h, up, false, L.snn, "solve: X updates");
    if (rc) return rc;
    L.solve_nrhs = nrhs;
  }
  return HODLR_OK;
}

// x <- K_HODLR^-1 b, with b already in h->X (N x nrhs, ld N).
int solve_in_place(hodlr_t h, int nrhs) {
  const int64_t N = h->n;
  LeafSolveLaunch S;
  S.leaf_min = h->d_leaf_min;
  S.leaf_size = h->d_leaf_size;
  S.lu_off = h->d_lu_off;
  S.lu = h->d_lu;
  S.perm = h->d_perm;
  S.X = h->X;
  S.ldx = N;
  S.ncols = nrhs;
  S.err = h->d_err;
  int e = leaf_solve_launch(S, (int)h->leaf_min.size(), h->smax, h->stream);
  if (e) return cuda_fail(h, (cudaError_t)e, "leaf_solve");
  h->nlaunch += 1;
  int rc = check_phase(h, "solve: leaves");
  if (rc) return rc;
  for (int l = (int)h->lv.size() - 1; l >= 0; --l) {
    Level& L = h->lv[l];
    const int nn = (int)L.nmin.size();
    e = run_tn(h, L.stn);
    if (e) return cuda_fail(h, (cudaError_t)e, "solve gemm_tn");
    rc = check_phase(h, "solve: V^T X products");
    if (!rc && h->checked)
      for (const auto& sn : L.nodes) {
        const int64_t sd = sn.kb + sn.kt;
        rc = check_extent(h, L.S + sn.s_off, sizeof(double) * sd * sd, "capacitance LU", "solve");
        if (!rc) rc = check_extent(h, L.piv + sn.p_off, sizeof(int) * sd, "pivots", "solve");
        if (rc) break;
      }
    if (rc) return rc;
    SchurLaunch SL;
    SL.nodes = L.d_snodes;
    SL.S = L.S;
    SL.Z = nullptr;
    SL.R = h->zs;
    SL.piv = L.piv;
    SL.err = h->d_err;
    e = schur_solve_launch(SL, nn, nrhs, nrhs, L.max_sd, h->stream);
    if (e) return cuda_fail(h, (cudaError_t)e, "solve schur");
    h->nlaunch += 1;
    rc = check_phase(h, "solve: capacitance");
    if (rc) return rc;
    e = run_nn(h, L.snn);
    if (e) return cuda_fail(h, (cudaError_t)e, "solve gemm_nn");
    rc = check_phase(h, "solve: X updates");
    if (rc) return rc;
  }
  return HODLR_OK;
}

// solve_in_place through a CUDA graph: captured on first use, replayed while
// the right-hand-side count, stream, buffers, precision and factorization
// are the same (one launch instead of ~4 per level).
int solve_fast(hodlr_t h, int nrhs) {
  if (h->sg_off || h->checked) return solve_in_place(h, nrhs);
  const void* key[4] = {h->X, h->zs, h->ws, (const void*)(intptr_t)(h->gemm_prec + 1)};
  bool same = h->sg_exec && h->sg_nrhs == nrhs && h->sg_stream == h->stream &&
              h->sg_gen == h->factor_gen;
  for (int i = 0; i < 4 && same; ++i) same = key[i] == h->sg_key[i];
  if (!same) {
    drop_solve_graph(h);
    const long long before = h->nlaunch;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      h->sg_off = true;
      return solve_in_place(h, nrhs);
    }
    int rc = solve_in_place(h, nrhs);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    cudaGraphExec_t ex = nullptr;
    if (!rc && e == cudaSuccess && g) e = cudaGraphInstantiate(&ex, g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc || e != cudaSuccess || !ex) {  // not capturable here: launch directly
      cudaGetLastError();
      h->sg_off = true;
      h->nlaunch = before;
      h->err.clear();
      return solve_in_place(h, nrhs);
    }
    h->sg_exec = ex;
    h->sg_nrhs = nrhs;
    h->sg_stream = h->stream;
    h->sg_gen = h->factor_gen;
    for (int i = 0; i < 4; ++i) h->sg_key[i] = key[i];
    h->sg_launches = h->nlaunch - before;
    h->nlaunch = before;
  }
  CK(cudaGraphLaunch(h->sg_exec, h->stream));
  h->nlaunch += h->sg_launches;
  return HODLR_OK;
}

int do_solve_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                    bool host_io) {
  int rc = do_factorize(h);
  if (rc) return rc;
  rc = build_solve_plans(h, nrhs);
  if (rc) return rc;
  const int64_t N = h->n;
  cudaMemcpyKind kin = host_io ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  cudaMemcpyKind kout = host_io ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  CK(cudaEventRecord(h->ev0, h->stream));
  CK(cudaMemcpy2DAsync(h->X, sizeof(double) * N, d_b, sizeof(double) * ldb, sizeof(double) * N,
                       nrhs, kin, h->stream));
  rc = solve_fast(h, nrhs);
  if (rc) return rc;
  CK(cudaMemcpy2DAsync(d_x, sizeof(double) * ldx, h->X, sizeof(double) * N, sizeof(double) * N,
                       nrhs, kout, h->stream));
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->t_solve = ms * 1e-3;
  h->t_total = h->t_lr + h->t_fact + h->t_solve;
  return check_dev_err(h, "solve");
}

constexpr int IR_BLOCKS = 256;

// R = B - Y (stored in Y) and per-block partial sums of |R_c|^2 and |B_c|^2.
__global__ void ir_residual_kernel(const double* B, double* Y, int64_t n, int nrhs,
                                   double* part) {
  __shared__ double red[2][8];
  for (int c = 0; c < nrhs; ++c) {
    double rr = 0.0, bb = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
      double b = B[c * n + i];
      double r = b - Y[c * n + i];
      Y[c * n + i] = r;
      rr = fma(r, r, rr);
      bb = fma(b, b, bb);
    }
    rr = warp_sum(rr);
    bb = warp_sum(bb);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      red[0][w] = rr;
      red[1][w] = bb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, d = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
        a += red[0][q];
        d += red[1][q];
      }
      part[(int64_t)(2 * c) * gridDim.x + blockIdx.x] = a;
      part[(int64_t)(2 * c + 1) * gridDim.x + blockIdx.x] = d;
    }
    __syncthreads();
  }
}

// Forest refinement: per system s (one CTA) and column c, r = b - y over
// the system's rows, out = (|r|^2, |b|^2); Y becomes r, or 0 for a system
// already converged (its x is left as it is).
__global__ void forest_residual_kernel(const double* B, double* Y, int64_t n, int nrhs,
                                       const int* off, const unsigned char* done, double* out) {
  __shared__ double red[2][8];
  const int s = blockIdx.x;
  const int r0 = off[s], r1 = off[s + 1];
  for (int c = 0; c < nrhs; ++c) {
    double rr = 0.0, bb = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const double b = B[c * n + i];
      const double r = b - Y[c * n + i];
      Y[c * n + i] = done[s] ? 0.0 : r;
      rr = fma(r, r, rr);
      bb = fma(b, b, bb);
    }
    rr = warp_sum(rr);
    bb = warp_sum(bb);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      red[0][w] = rr;
      red[1][w] = bb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, d = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
        a += red[0][q];
        d += red[1][q];
      }
      out[2 * ((int64_t)s * nrhs + c)] = a;
      out[2 * ((int64_t)s * nrhs + c) + 1] = d;
    }
    __syncthreads();
  }
}

__global__ void axpy_cols_kernel(double* X, const double* D, int64_t total) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x)
    X[e] += D[e];
}

int kmatvec_dev(hodlr_t h, int nrhs, const double* d_x, int ldx, double* d_y, int ldy,
                const unsigned char* skip) {
  if (h->nsys) {  // forest: block-diagonal product
    KmatvecLaunch L;
    L.skip = skip;
    L.src = make_src(h);
    L.X = d_x;
    L.ldx = ldx;
    L.Y = d_y;
    L.ldy = ldy;
    L.ws = nullptr;
    L.n = h->n;
    L.nrhs = nrhs;
    int e = kmatvec_forest_launch(L, h->d_fitems, h->ftype_off, h->stream);
    if (e) return cuda_fail(h, (cudaError_t)e, "forest kmatvec");
    for (int t = 0; t < HX_FOREST_TYPES; ++t) h->nlaunch += h->ftype_off[t + 1] > h->ftype_off[t];
    return HODLR_OK;
  }
  if (nrhs > 8 && kmatvec_sym_slices(h->n, 8, h->dense)) {
    // the symmetric form serves up to 8 columns: two or more of its products
    // beat one row-by-row product of all columns (measured with 16 columns at
    // N = 262144: 157 vs 172 ms, 3D Gaussian; 174 vs 205 ms, 2D Matern-3/2)
    for (int c0 = 0; c0 < nrhs; c0 += 8) {
      const int nc = std::min(8, nrhs - c0);
      int rc = kmatvec_dev(h, nc, d_x + (int64_t)c0 * ldx, ldx, d_y + (int64_t)c0 * ldy, ldy);
      if (rc) return rc;
    }
    return HODLR_OK;
  }
  const int sym = kmatvec_sym_slices(h->n, nrhs, h->dense);
  const int sp = sym ? sym : kmatvec_splits(h->n, h->num_sms);
  if (sym || sp > 1) {
    int rc = ensure_ws(h, (int64_t)sp * nrhs * h->n);
    if (rc) return rc;
  }
  KmatvecLaunch L;
  L.src = make_src(h);
  L.X = d_x;
  L.ldx = ldx;
  L.Y = d_y;
  L.ldy = ldy;
  L.ws = h->ws;
  L.n = h->n;
  L.nrhs = nrhs;
  int e = sym ? kmatvec_sym_launch(L, sym, h->stream) : kmatvec_launch(L, sp, h->stream);
  if (e) return cuda_fail(h, (cudaError_t)e, "kmatvec");
  h->nlaunch += 1 + (sym || sp > 1);
  return check_phase(h, "full-kernel product");
}


// Iterative refinement: x0 = M^-1 b, then x += M^-1 (b - K x) until
// max_c ||b_c - K x_c|| / ||b_c|| <= tol or max_iter corrections.  b and x
// are device pointers (ld n).  *iters = corrections applied.
int refine_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                  double tol, int max_iter, int* iters, double* relres) {
  const int64_t N = h->n;
  int rc = build_solve_plans(h, nrhs);
  if (rc) return rc;
  if (nrhs > h->ir_cols) {
    dfree(h, h->ir_b);
    dfree(h, h->ir_x);
    dfree(h, h->ir_y);
    dfree(h, h->ir_part);
    CK(dalloc(h, &h->ir_b, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_x, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_y, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_part, (size_t)(2 * nrhs * IR_BLOCKS)));
    h->ir_cols = nrhs;
  }
  CK(cudaMemcpy2DAsync(h->ir_b, sizeof(double) * N, d_b, sizeof(double) * ldb,
                       sizeof(double) * N, nrhs, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->X, h->ir_b, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice,
                     h->stream));
  rc = solve_fast(h, nrhs);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->ir_x, h->X, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice,
                     h->stream));
  std::vector<double> part((size_t)2 * nrhs * IR_BLOCKS);
  double worst = HUGE_VAL;
  int it = 0;
  for (;; ++it) {
    for (int c0 = 0; c0 < nrhs; c0 += 16) {
      int nc = std::min(16, nrhs - c0);
      rc = kmatvec_dev(h, nc, h->ir_x + c0 * N, (int)N, h->ir_y + c0 * N, (int)N);
      if (rc) return rc;
    }
    ir_residual_kernel<<<IR_BLOCKS, 256, 0, h->stream>>>(h->ir_b, h->ir_y, N, nrhs, h->ir_part);
    CK(cudaGetLastError());
    h->nlaunch += 1;
    CK(cudaMemcpyAsync(part.data(), h->ir_part, sizeof(double) * part.size(),
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    worst = 0.0;
    for (int c = 0; c < nrhs; ++c) {
      double a = 0.0, d = 0.0;
      for (int q = 0; q < IR_BLOCKS; ++q) {
        a += part[(size_t)(2 * c) * IR_BLOCKS + q];
        d += part[(size_t)(2 * c + 1) * IR_BLOCKS + q];
      }
      double r = d > 0 ? std::sqrt(a / d) : std::sqrt(a);
      if (relres) relres[c] = r;
      worst = std::max(worst, r);
    }
    if (worst <= tol || it >= max_iter) break;
    CK(cudaMemcpyAsync(h->X, h->ir_y, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice,
                       h->stream));
    rc = solve_fast(h, nrhs);
    if (rc) return rc;
    axpy_cols_kernel<<<1024, 256, 0, h->stream>>>(h->ir_x, h->X, N * nrhs);
    CK(cudaGetLastError());
    h->nlaunch += 1;
  }
  if (iters) *iters = it;
  CK(cudaMemcpy2DAsync(d_x, sizeof(double) * ldx, h->ir_x, sizeof(double) * N,
                       sizeof(double) * N, nrhs, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_dev_err(h, "refine");
}

// Iterative refinement of a forest with a stopping test per system:
// x0 = M^-1 b, then x += M^-1 (b - K x) on the systems whose
// max_c ||b_c - K x_c|| / ||b_c|| (over the system's rows) is still above
// tol.  relres: nsys x nrhs, system-major.
int forest_refine_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                         double tol, int max_iter, int* iters, double* relres) {
  const int64_t N = h->n;
  const int S = h->nsys;
  int rc = build_solve_plans(h, nrhs);
  if (rc) return rc;
  if (nrhs > h->ir_cols) {
    dfree(h, h->ir_b);
    dfree(h, h->ir_x);
    dfree(h, h->ir_y);
    dfree(h, h->ir_part);
    CK(dalloc(h, &h->ir_b, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_x, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_y, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_part, (size_t)(2 * nrhs * IR_BLOCKS)));
    h->ir_cols = nrhs;
  }
  double* d_out = nullptr;
  unsigned char* d_done = nullptr;
  int* d_off = nullptr;
  CK(dalloc(h, &d_out, (size_t)2 * S * nrhs));
  CK(dalloc(h, &d_done, (size_t)S));
  CK(dalloc(h, &d_off, (size_t)S + 1));
  CK(cudaMemcpyAsync(d_off, h->sys_off.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemsetAsync(d_done, 0, (size_t)S, h->stream));
  CK(cudaMemcpy2DAsync(h->ir_b, sizeof(double) * N, d_b, sizeof(double) * ldb,
                       sizeof(double) * N, nrhs, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->X, h->ir_b, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice,
                     h->stream));
  rc = solve_fast(h, nrhs);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->ir_x, h->X, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice,
                     h->stream));
  std::vector<double> out((size_t)2 * S * nrhs);
  std::vector<unsigned char> done((size_t)S, 0);
  int it = 0;
  for (;; ++it) {
    // systems frozen by an earlier pass are left out of the product (their
    // rows of Y are not read for a correction: the residual kernel zeroes them)
    for (int c0 = 0; c0 < nrhs; c0 += 16) {
      int nc = std::min(16, nrhs - c0);
      rc = kmatvec_dev(h, nc, h->ir_x + c0 * N, (int)N, h->ir_y + c0 * N, (int)N, d_done);
      if (rc) return rc;
    }
    forest_residual_kernel<<<S, 256, 0, h->stream>>>(h->ir_b, h->ir_y, N, nrhs, d_off, d_done,
                                                     d_out);
    CK(cudaGetLastError());
    h->nlaunch += 1;
    CK(d2h(h, out.data(), d_out, sizeof(double) * out.size()));
    bool all = true;
    for (int q = 0; q < S; ++q) {
      double worst = 0.0;
      for (int c = 0; c < nrhs; ++c) {
        const double a = out[2 * ((size_t)q * nrhs + c)], d = out[2 * ((size_t)q * nrhs + c) + 1];
        const double r = d > 0 ? std::sqrt(a / d) : std::sqrt(a);
        if (!done[q] && relres) relres[(size_t)q * nrhs + c] = r;
        worst = std::max(worst, r);
      }
      if (!done[q] && !(worst > tol)) done[q] = 1;
      all &= done[q] != 0;
    }
    if (all || it >= max_iter) break;
    // systems that converged in this pass still take this correction (their
    // residual rows were written); from the next pass on they are frozen
    CK(cudaMemcpyAsync(h->X, h->ir_y, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice,
                       h->stream));
    rc = solve_fast(h, nrhs);
    if (rc) return rc;
    axpy_cols_kernel<<<1024, 256, 0, h->stream>>>(h->ir_x, h->X, N * nrhs);
    CK(cudaGetLastError());
    h->nlaunch += 1;
    CK(cudaMemcpyAsync(d_done, done.data(), (size_t)S, cudaMemcpyHostToDevice, h->stream));
  }
  if (iters) *iters = it;
  CK(cudaMemcpy2DAsync(d_x, sizeof(double) * ldx, h->ir_x, sizeof(double) * N,
                       sizeof(double) * N, nrhs, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  dfree(h, d_out);
  dfree(h, d_done);
  dfree(h, d_off);
  return check_dev_err(h, "forest refine");
}

// ------------------------------------------------------------- GMRES
constexpr int GM_BLOCKS = 256;

// part[(i * nrhs + c) * GM_BLOCKS + blk] = sum over this block's rows of
// V_i[:, c] . W[:, c] for i < nv (V_i = V + i * n * nrhs).
__global__ void gm_dots_kernel(const double* V, int nv, const double* W, int64_t n, int nrhs,
                               double* part) {
  __shared__ double red[8];
  const int i = blockIdx.y;
  const double* Vi = V + (int64_t)i * n * nrhs;
  for (int c = 0; c < nrhs; ++c) {
    double a = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x)
      a = fma(Vi[c * n + r], W[c * n + r], a);
    a = warp_sum(a);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
      part[((int64_t)i * nrhs + c) * gridDim.x + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

// out[k] = sum of the GM_BLOCKS partials of k (fixed order).
__global__ void gm_sum_kernel(const double* part, int count, double* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int q = 0; q < GM_BLOCKS; ++q) t += part[(int64_t)k * GM_BLOCKS + q];
    out[k] = t;
  }
}

// Segments: in a forest every system is its own GMRES problem, so inner
// products and coefficients are per (system, column) -- "virtual column"
// v = s * nrhs + c of Vc = S * nrhs, S = 1 outside a forest.  Coefficient
// arrays are indexed [i][v]; psys (null when S == 1) maps a row to its system.

// part[(i * S + s) * nrhs + c] = V_i[rows of s, c] . W[rows of s, c]: one CTA
// per (system, i), rows in order of a fixed tree (forests only).
__global__ void gm_seg_dots_kernel(const double* V, int nv, const double* W, int64_t n, int nrhs,
                                   const int* off, int S, double* out) {
  __shared__ double red[8];
  const int sys = blockIdx.x, i = blockIdx.y;
  const double* Vi = V + (int64_t)i * n * nrhs;
  const int r0 = off[sys], r1 = off[sys + 1];
  for (int c = 0; c < nrhs; ++c) {
    double a = 0.0;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x)
      a = fma(Vi[c * n + r], W[c * n + r], a);
    a = warp_sum(a);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
      out[((int64_t)i * S + sys) * nrhs + c] = t;
    }
    __syncthreads();
  }
}

// W[:, c] -= sum_{i < nv} coef[(i * S + s) * nrhs + c] * V_i[:, c], s the row's system
__global__ void gm_sub_kernel(const double* V, int nv, const double* coef, double* W, int64_t n,
                              int nrhs, const int* psys, int S) {
  const int64_t total = n * nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / n);
    const int sys = psys ? psys[e - (int64_t)c * n] : 0;
    double w = W[e];
    for (int i = 0; i < nv; ++i)
      w = fma(-coef[((int64_t)i * S + sys) * nrhs + c], V[(int64_t)i * total + e], w);
    W[e] = w;
  }
}

// Y[:, c] = X[:, c] * scale[s * nrhs + c] (scale 0 gives an exact zero)
__global__ void gm_scale_kernel(const double* X, const double* scale, double* Y, int64_t n,
                                int nrhs, const int* psys) {
  const int64_t total = n * nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / n);
    const int sys = psys ? psys[e - (int64_t)c * n] : 0;
    const double sc = scale[(int64_t)sys * nrhs + c];
    Y[e] = sc == 0.0 ? 0.0 : X[e] * sc;
  }
}

static int gm_segments(hodlr_t h) { return h->nsys ? h->nsys : 1; }

// Host-side launch helpers bound to the handle's stream.  out / coef / sc
// hold nv * S * nrhs (dots, combinations) or S * nrhs (scaling) values.
int gm_dots(hodlr_t h, const double* V, int nv, const double* W, int nrhs, std::vector<double>& out) {
  const int64_t N = h->n;
  const int S = gm_segments(h);
  if (S == 1) {
    gm_dots_kernel<<<dim3(GM_BLOCKS, nv), 256, 0, h->stream>>>(V, nv, W, N, nrhs, h->gm_part);
    gm_sum_kernel<<<(nv * nrhs + 255) / 256, 256, 0, h->stream>>>(h->gm_part, nv * nrhs, h->gm_h);
    h->nlaunch += 2;
  } else {
    gm_seg_dots_kernel<<<dim3(S, nv), 256, 0, h->stream>>>(V, nv, W, N, nrhs, h->d_sysoff, S,
                                                            h->gm_h);
    h->nlaunch += 1;
  }
  CK(cudaGetLastError());
  const size_t cnt = (size_t)nv * S * nrhs;
  out.resize(cnt);
  CK(cudaMemcpyAsync(out.data(), h->gm_h, sizeof(double) * cnt, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return HODLR_OK;
}

int gm_sub(hodlr_t h, const double* V, int nv, const std::vector<double>& coef, double* W, int nrhs) {
  const int64_t N = h->n;
  const int S = gm_segments(h);
  CK(cudaMemcpyAsync(h->gm_h, coef.data(), sizeof(double) * nv * S * nrhs,
                     cudaMemcpyHostToDevice, h->stream));
  gm_sub_kernel<<<1024, 256, 0, h->stream>>>(V, nv, h->gm_h, W, N, nrhs,
                                             S > 1 ? h->d_psys : nullptr, S);
  CK(cudaGetLastError());
  h->nlaunch += 1;
  return check_phase(h, "gmres: basis combination");
}

int gm_scale(hodlr_t h, const double* X, const std::vector<double>& sc, double* Y, int nrhs) {
  const int64_t N = h->n;
  const int S = gm_segments(h);
  CK(cudaMemcpyAsync(h->gm_h, sc.data(), sizeof(double) * S * nrhs, cudaMemcpyHostToDevice,
                     h->stream));
  gm_scale_kernel<<<1024, 256, 0, h->stream>>>(X, h->gm_h, Y, N, nrhs,
                                               S > 1 ? h->d_psys : nullptr);
  CK(cudaGetLastError());
  h->nlaunch += 1;
  return check_phase(h, "gmres: column scaling");
}

// Restarted GMRES(m) on K x = b with the HODLR factor as a right
// preconditioner (K M^-1 u = b, x = M^-1 u), all columns in lockstep so every
// iteration costs one full-kernel product and one HODLR solve for all of
// them.  Starts from the direct solve (the initial guess of iterative_Solve,
// src/HODLR_Matrix.cpp:1169-1177) and stops when the relative residual
// max_c ||b_c - K x_c|| / ||b_c|| <= tol.  Classical Gram-Schmidt with one
// re-orthogonalisation; Givens rotations as in IML's GMRES
// (IML/include/gmres.h:83-153).  On a forest every (system, column) pair is
// its own GMRES problem -- its own inner products, Hessenberg matrix and
// stopping test on the system's rows -- and the systems whose columns have
// all converged are left out of the block-diagonal product.
//
// The residual b - K x is formed with a full-kernel product once, for the
// initial guess.  Each cycle's update x += Z y is matched by r -= W y with
// W_j = K Z_j, the products the iterations already computed (kept before
// their orthogonalisation), so r stays b - K x up to the rounding of that
// combination -- no further full-kernel product per cycle.
int gmres_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx,
                 double tol, int max_iter, int m, int* iters, double* relres) {
  const int64_t N = h->n;
  const int S = gm_segments(h);
  const int VC = S * nrhs;  // virtual columns
  int rc = build_solve_plans(h, nrhs);
  if (rc) return rc;
  if (nrhs > h->ir_cols) {
    dfree(h, h->ir_b);
    dfree(h, h->ir_x);
    dfree(h, h->ir_y);
    dfree(h, h->ir_part);
    CK(dalloc(h, &h->ir_b, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_x, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_y, (size_t)(N * nrhs)));
    CK(dalloc(h, &h->ir_part, (size_t)(2 * nrhs * IR_BLOCKS)));
    h->ir_cols = nrhs;
  }
  if (m > h->gm_m || nrhs > h->gm_cols) {
    dfree(h, h->gm_V);
    dfree(h, h->gm_Z);
    dfree(h, h->gm_W);
    dfree(h, h->gm_h);
    dfree(h, h->gm_part);
    CK(dalloc(h, &h->gm_V, (size_t)((m + 1) * N * nrhs)));
    CK(dalloc(h, &h->gm_Z, (size_t)(m * N * nrhs)));
    CK(dalloc(h, &h->gm_W, (size_t)(m * N * nrhs)));
    CK(dalloc(h, &h->gm_h, (size_t)((m + 2) * (int64_t)S * nrhs)));
    CK(dalloc(h, &h->gm_part, (size_t)((m + 2) * nrhs * GM_BLOCKS)));
    h->gm_m = m;
    h->gm_cols = nrhs;
  }
  unsigned char* d_skip = nullptr;
  if (S > 1) {
    if (!h->d_sysoff) {
      CK(dalloc(h, &h->d_sysoff, (size_t)S + 1));
      CK(h2d(h, h->d_sysoff, h->sys_off.data(), sizeof(int) * (S + 1)));
    }
    CK(dalloc(h, &d_skip, (size_t)S));
    CK(cudaMemsetAsync(d_skip, 0, (size_t)S, h->stream));
  }
  const int64_t P = N * nrhs;
  CK(cudaMemcpy2DAsync(h->ir_b, sizeof(double) * N, d_b, sizeof(double) * ldb,
                       sizeof(double) * N, nrhs, cudaMemcpyDeviceToDevice, h->stream));
  // x0 = M^-1 b
  CK(cudaMemcpyAsync(h->X, h->ir_b, sizeof(double) * P, cudaMemcpyDeviceToDevice, h->stream));
  rc = solve_fast(h, nrhs);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->ir_x, h->X, sizeof(double) * P, cudaMemcpyDeviceToDevice, h->stream));
  std::vector<double> bnorm, tmp, hcol, coef;
  rc = gm_dots(h, h->ir_b, 1, h->ir_b, nrhs, bnorm);
  if (rc) return rc;
  for (auto& v : bnorm) v = v > 0 ? std::sqrt(v) : 1.0;
  int total_it = 0;
  std::vector<double> worst_res(VC, HUGE_VAL);
  // r = b - K x0 -> ir_y (the one full-kernel product for the residual)
  for (int c0 = 0; c0 < nrhs; c0 += 16) {
    int nc = std::min(16, nrhs - c0);
    rc = kmatvec_dev(h, nc, h->ir_x + c0 * N, (int)N, h->ir_y + c0 * N, (int)N);
    if (rc) return rc;
  }
  ir_residual_kernel<<<IR_BLOCKS, 256, 0, h->stream>>>(h->ir_b, h->ir_y, N, nrhs, h->ir_part);
  CK(cudaGetLastError());
  h->nlaunch += 1;
  std::vector<unsigned char> skip(S, 0);
  for (int cycle = 0;; ++cycle) {
    // ir_y = r = b - K x ; beta = ||r|| per virtual column
    rc = gm_dots(h, h->ir_y, 1, h->ir_y, nrhs, tmp);
    if (rc) return rc;
    std::vector<double> beta(VC);
    double worst = 0.0;
    for (int v = 0; v < VC; ++v) {
      beta[v] = std::sqrt(std::max(tmp[v], 0.0));
      worst_res[v] = beta[v] / bnorm[v];
      worst = std::max(worst, worst_res[v]);
    }
    if (worst <= tol || total_it >= max_iter) break;
    // V0 = r / beta
    std::vector<double> sc(VC);
    for (int v = 0; v < VC; ++v) sc[v] = beta[v] > 0 ? 1.0 / beta[v] : 0.0;
    rc = gm_scale(h, h->ir_y, sc, h->gm_V, nrhs);
    if (rc) return rc;
    // per virtual column Hessenberg (column-major (m+1) x m), rotations, rhs g
    std::vector<double> H((size_t)(m + 1) * m * VC, 0.0), cs((size_t)m * VC),
        sn((size_t)m * VC), g((size_t)(m + 1) * VC, 0.0);
    for (int v = 0; v < VC; ++v) g[v] = beta[v];
    std::vector<int> done(VC, 0), used(VC, 0);
    for (int v = 0; v < VC; ++v)
      if (worst_res[v] <= tol) done[v] = 1;
    int j = 0;
    for (; j < m && total_it < max_iter; ++j, ++total_it) {
      double* Vj = h->gm_V + (int64_t)j * P;
      double* Zj = h->gm_Z + (int64_t)j * P;
      if (S > 1) {  // systems with every column converged leave the product
        for (int q = 0; q < S; ++q) {
          bool all = true;
          for (int c = 0; c < nrhs; ++c) all &= done[(size_t)q * nrhs + c] != 0;
          skip[q] = all;
        }
        CK(cudaMemcpyAsync(d_skip, skip.data(), (size_t)S, cudaMemcpyHostToDevice, h->stream));
      }
      // Z_j = M^-1 V_j ; W = K Z_j
      CK(cudaMemcpyAsync(h->X, Vj, sizeof(double) * P, cudaMemcpyDeviceToDevice, h->stream));
      rc = solve_fast(h, nrhs);
      if (rc) return rc;
      CK(cudaMemcpyAsync(Zj, h->X, sizeof(double) * P, cudaMemcpyDeviceToDevice, h->stream));
      for (int c0 = 0; c0 < nrhs; c0 += 16) {
        int nc = std::min(16, nrhs - c0);
        rc = kmatvec_dev(h, nc, Zj + c0 * N, (int)N, h->ir_y + c0 * N, (int)N, d_skip);
        if (rc) return rc;
      }
      CK(cudaMemcpyAsync(h->gm_W + (int64_t)j * P, h->ir_y, sizeof(double) * P,
                         cudaMemcpyDeviceToDevice, h->stream));
      // classical Gram-Schmidt, twice
      std::vector<double> hsum((size_t)(j + 1) * VC, 0.0);
      for (int pass = 0; pass < 2; ++pass) {
        rc = gm_dots(h, h->gm_V, j + 1, h->ir_y, nrhs, hcol);
        if (rc) return rc;
        for (int v = 0; v < VC; ++v)
          if (done[v])
            for (int i = 0; i <= j; ++i) hcol[(size_t)i * VC + v] = 0.0;
        rc = gm_sub(h, h->gm_V, j + 1, hcol, h->ir_y, nrhs);
        if (rc) return rc;
        for (size_t q = 0; q < hsum.size(); ++q) hsum[q] += hcol[q];
      }
      rc = gm_dots(h, h->ir_y, 1, h->ir_y, nrhs, tmp);
      if (rc) return rc;
      std::vector<double> inv(VC, 0.0);
      bool all_done = true;
      for (int v = 0; v < VC; ++v) {
        if (done[v]) continue;
        double* Hc = &H[(size_t)v * (m + 1) * m];
        for (int i = 0; i <= j; ++i) Hc[(size_t)j * (m + 1) + i] = hsum[(size_t)i * VC + v];
        double hn = std::sqrt(std::max(tmp[v], 0.0));
        Hc[(size_t)j * (m + 1) + j + 1] = hn;
        inv[v] = hn > 0 ? 1.0 / hn : 0.0;
        // apply previous rotations, then a new one
        for (int i = 0; i < j; ++i) {
          double a = Hc[(size_t)j * (m + 1) + i], b2 = Hc[(size_t)j * (m + 1) + i + 1];
          double ci = cs[(size_t)v * m + i], si = sn[(size_t)v * m + i];
          Hc[(size_t)j * (m + 1) + i] = ci * a + si * b2;
          Hc[(size_t)j * (m + 1) + i + 1] = -si * a + ci * b2;
        }
        double a = Hc[(size_t)j * (m + 1) + j], b2 = Hc[(size_t)j * (m + 1) + j + 1];
        double r = std::hypot(a, b2);
        double ci = r > 0 ? a / r : 1.0, si = r > 0 ? b2 / r : 0.0;
        cs[(size_t)v * m + j] = ci;
        sn[(size_t)v * m + j] = si;
        Hc[(size_t)j * (m + 1) + j] = r;
        Hc[(size_t)j * (m + 1) + j + 1] = 0.0;
        double gj = g[(size_t)j * VC + v];
        g[(size_t)j * VC + v] = ci * gj;
        g[(size_t)(j + 1) * VC + v] = -si * gj;
        used[v] = j + 1;
        // stop this column a little below tol; the residual update decides
        if (std::fabs(g[(size_t)(j + 1) * VC + v]) <= 0.5 * tol * bnorm[v] || hn == 0.0)
          done[v] = 1;
        if (!done[v]) all_done = false;
      }
      rc = gm_scale(h, h->ir_y, inv, h->gm_V + (int64_t)(j + 1) * P, nrhs);
      if (rc) return rc;
      if (all_done) {
        ++j;
        ++total_it;
        break;
      }
    }
    // x += Z y, y from the triangular systems (per virtual column)
    std::vector<double> ycoef((size_t)m * VC, 0.0);
    int nv = 0;
    for (int v = 0; v < VC; ++v) {
      const int k = used[v];
      nv = std::max(nv, k);
      const double* Hc = &H[(size_t)v * (m + 1) * m];
      for (int i = k - 1; i >= 0; --i) {
        double t = g[(size_t)i * VC + v];
        for (int q = i + 1; q < k; ++q) t -= Hc[(size_t)q * (m + 1) + i] * ycoef[(size_t)q * VC + v];
        ycoef[(size_t)i * VC + v] = Hc[(size_t)i * (m + 1) + i] != 0 ? t / Hc[(size_t)i * (m + 1) + i] : 0.0;
      }
    }
    // r <- beta V_0 - W y (= r - K Z y), then x <- x + Z y
    rc = gm_scale(h, h->gm_V, beta, h->ir_y, nrhs);
    if (rc) return rc;
    if (nv > 0) {
      rc = gm_sub(h, h->gm_W, nv, ycoef, h->ir_y, nrhs);
      if (rc) return rc;
      for (auto& v : ycoef) v = -v;  // gm_sub subtracts
      rc = gm_sub(h, h->gm_Z, nv, ycoef, h->ir_x, nrhs);
      if (rc) return rc;
    }
    (void)j;
  }
  if (iters) *iters = total_it;
  if (relres)  // per column, the worst system
    for (int c = 0; c < nrhs; ++c) {
      double w = 0.0;
      for (int q = 0; q < S; ++q) w = std::max(w, worst_res[(size_t)q * nrhs + c]);
      relres[c] = w;
    }
  CK(cudaMemcpy2DAsync(d_x, sizeof(double) * ldx, h->ir_x, sizeof(double) * N,
                       sizeof(double) * N, nrhs, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  dfree(h, d_skip);
  return check_dev_err(h, "gmres");
}

}  // namespace hodlr_impl
