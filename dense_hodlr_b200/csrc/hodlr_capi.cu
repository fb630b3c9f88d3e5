// C ABI of the B200 HODLR solver (include/hodlr_b200.h).  Entry points check
// their arguments and forward to the host orchestration units (handle.h).
#include "handle.h"

using namespace hodlr_impl;

// ---------------------------------------------------------------- C ABI
extern "C" {

int hodlr_create_kernel(hodlr_t* out, int n, int dim, const double* pts,
                        const hodlr_kernel_desc* k, int leaf_size) {
  if (!out || n <= 0 || dim < 1 || dim > 3 || !pts || !k || leaf_size < 1)
    return HODLR_ERR_ARG;
  if (k->type < 0 || k->type > 4 || !(k->length_scale > 0)) return HODLR_ERR_ARG;
  *out = nullptr;
  hodlr_t h = new hodlr_handle_s();
  h->n = n;
  h->dim = dim;
  h->leaf = leaf_size;
  h->kp = hx_make_kparams(k->type, dim, k->length_scale, k->diag_shift, k->diag_replace,
                          k->diag_value);
  int rc = init_common(h);
  if (!rc) {
    cudaError_t e = dalloc(h, &h->d_pts, (size_t)n * dim);
    if (e == cudaSuccess)
      e = h2d(h, h->d_pts, pts, sizeof(double) * (size_t)n * dim);
    if (e != cudaSuccess) rc = cuda_fail(h, e, "points upload");
  }
  if (rc) {
    hodlr_destroy(h);
    return rc;
  }
  *out = h;
  return HODLR_OK;
}

int hodlr_create_dense(hodlr_t* out, int n, const double* A, int lda, int leaf_size) {
  if (!out || n <= 0 || !A || lda < n || leaf_size < 1) return HODLR_ERR_ARG;
  *out = nullptr;
  hodlr_t h = new hodlr_handle_s();
  h->n = n;
  h->dim = 0;
  h->leaf = leaf_size;
  h->dense = true;
  int rc = init_common(h);
  if (!rc) {
    cudaError_t e = dalloc(h, &h->d_A, (size_t)n * n);
    if (e == cudaSuccess)
      e = copy2d(h, h->d_A, sizeof(double) * n, A, sizeof(double) * lda, sizeof(double) * n, n,
                 cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cuda_fail(h, e, "matrix upload");
  }
  if (rc) {
    hodlr_destroy(h);
    return rc;
  }
  *out = h;
  return HODLR_OK;
}

int hodlr_create_dense_device(hodlr_t* out, int n, int leaf_size, double** dA, int64_t* ld) {
  if (!out || n <= 0 || leaf_size < 1 || !dA || !ld) return HODLR_ERR_ARG;
  *out = nullptr;
  *dA = nullptr;
  *ld = 0;
  hodlr_t h = new hodlr_handle_s();
  h->n = n;
  h->dim = 0;
  h->leaf = leaf_size;
  h->dense = true;
  int rc = init_common(h);
  if (!rc) {
    cudaError_t e = dalloc(h, &h->d_A, (size_t)n * n);
    // the stream-ordered allocation is complete before the caller's fill,
    // which may run on any stream
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = cuda_fail(h, e, "matrix allocation");
  }
  if (rc) {
    hodlr_destroy(h);
    return rc;
  }
  *dA = h->d_A;
  *ld = n;
  *out = h;
  return HODLR_OK;
}

int hodlr_create_forest(hodlr_t* out, int nsys, const int* sizes, int dim, const double* pts,
                        const hodlr_kernel_desc* kernels, int leaf_size) {
  if (!out || nsys < 1 || !sizes || dim < 1 || dim > 3 || !pts || !kernels || leaf_size < 1)
    return HODLR_ERR_ARG;
  int64_t total = 0;
  for (int q = 0; q < nsys; ++q) {
    if (sizes[q] < 1) return HODLR_ERR_ARG;
    const hodlr_kernel_desc& k = kernels[q];
    if (k.type < 0 || k.type > 4 || !(k.length_scale > 0)) return HODLR_ERR_ARG;
    total += sizes[q];
  }
  if (total > INT32_MAX / 2) return HODLR_ERR_ARG;
  *out = nullptr;
  hodlr_t h = new hodlr_handle_s();
  h->n = (int)total;
  h->dim = dim;
  h->leaf = leaf_size;
  h->nsys = nsys;
  h->sys_off.assign((size_t)nsys + 1, 0);
  for (int q = 0; q < nsys; ++q) {
    h->sys_off[q + 1] = h->sys_off[q] + sizes[q];
    const hodlr_kernel_desc& k = kernels[q];
    h->sys_kp.push_back(hx_make_kparams(k.type, dim, k.length_scale, k.diag_shift,
                                        k.diag_replace, k.diag_value));
  }
  h->kp = h->sys_kp[0];
  int rc = init_common(h);
  if (!rc) {
    // point -> system, and the product's work items: 256-row tiles grouped by
    // kernel family, largest systems first
    std::vector<int> psys((size_t)total);
    std::vector<std::vector<std::pair<int, int4>>> byt(HX_FOREST_TYPES);
    for (int q = 0; q < nsys; ++q) {
      const int o = h->sys_off[q], e = h->sys_off[q + 1];
      for (int i = o; i < e; ++i) psys[(size_t)i] = q;
      for (int r = o; r < e; r += HX_FOREST_TILE)
        byt[kernels[q].type].push_back({e - o, make_int4(r, o, e, q)});
    }
    std::vector<int4> items;
    for (int t = 0; t < HX_FOREST_TYPES; ++t) {
      std::stable_sort(byt[t].begin(), byt[t].end(),
                       [](const std::pair<int, int4>& a, const std::pair<int, int4>& b) {
                         return a.first > b.first;
                       });
      h->ftype_off[t] = (int)items.size();
      for (auto& pi : byt[t]) items.push_back(pi.second);
    }
    h->ftype_off[HX_FOREST_TYPES] = (int)items.size();
    cudaError_t e = dalloc(h, &h->d_pts, (size_t)total * dim);
    if (e == cudaSuccess) e = h2d(h, h->d_pts, pts, sizeof(double) * (size_t)total * dim);
    if (e == cudaSuccess) e = dalloc(h, &h->d_kps, (size_t)nsys);
    if (e == cudaSuccess) e = h2d(h, h->d_kps, h->sys_kp.data(), sizeof(hx_kparams) * nsys);
    if (e == cudaSuccess) e = dalloc(h, &h->d_psys, (size_t)total);
    if (e == cudaSuccess) e = h2d(h, h->d_psys, psys.data(), sizeof(int) * (size_t)total);
    if (e == cudaSuccess) e = dalloc(h, &h->d_fitems, items.size());
    if (e == cudaSuccess) e = h2d(h, h->d_fitems, items.data(), sizeof(int4) * items.size());
    if (e != cudaSuccess) rc = cuda_fail(h, e, "forest upload");
  }
  if (rc) {
    hodlr_destroy(h);
    return rc;
  }
  *out = h;
  return HODLR_OK;
}

int hodlr_set_index_tree(hodlr_t h, int nnodes, const int* split, const int* left,
                         const int* right) {
  return hodlr_set_index_tree_bounds(h, nnodes, split, left, right, nullptr, nullptr, nullptr,
                                     nullptr);
}

int hodlr_set_index_tree_bounds(hodlr_t h, int nnodes, const int* split, const int* left,
                                const int* right, const int* top_min, const int* bott_min,
                                const int* top_max, const int* bott_max) {
  if (!h || nnodes < 0 || (nnodes > 0 && (!split || !left || !right))) return HODLR_ERR_ARG;
  const bool bounds = top_min || bott_min || top_max || bott_max;
  if (bounds && !(top_min && bott_min && top_max && bott_max)) return HODLR_ERR_ARG;
  if (h->nsys) return fail(h, HODLR_ERR_UNSUPPORTED, "user index trees are for one system");
  CK(cudaStreamSynchronize(h->stream));
  free_compress(h);
  h->compressed = false;
  h->ut_split.assign(split, split + nnodes);
  h->ut_left.assign(left, left + nnodes);
  h->ut_right.assign(right, right + nnodes);
  if (bounds) {
    h->ut_tmin.assign(top_min, top_min + nnodes);
    h->ut_bmin.assign(bott_min, bott_min + nnodes);
    h->ut_tmax.assign(top_max, top_max + nnodes);
    h->ut_bmax.assign(bott_max, bott_max + nnodes);
  } else {
    h->ut_tmin.clear();
    h->ut_bmin.clear();
    h->ut_tmax.clear();
    h->ut_bmax.clear();
  }
  build_tree(h);
  int rc = HODLR_OK;
  if (h->leaf_min.empty() || h->smax > 160) {
    rc = fail(h, h->leaf_min.empty() ? HODLR_ERR_ARG : HODLR_ERR_UNSUPPORTED,
              h->leaf_min.empty() ? "invalid user index tree" : "leaf size above 160");
    h->ut_split.clear();
    h->ut_left.clear();
    h->ut_right.clear();
    h->ut_tmin.clear();
    h->ut_bmin.clear();
    h->ut_tmax.clear();
    h->ut_bmax.clear();
    build_tree(h);  // back to the default tree
  }
  const int nl = (int)h->leaf_min.size();
  dfree(h, h->d_leaf_min);
  dfree(h, h->d_leaf_size);
  CK(dalloc(h, &h->d_leaf_min, (size_t)nl));
  CK(dalloc(h, &h->d_leaf_size, (size_t)nl));
  CK(h2d(h, h->d_leaf_min, h->leaf_min.data(), 4 * nl));
  CK(h2d(h, h->d_leaf_size, h->leaf_size.data(), 4 * nl));
  return rc;
}

int hodlr_logdet(hodlr_t h, double* log_abs_det, int* sign) {
  if (!h || !log_abs_det) return HODLR_ERR_ARG;
  return do_logdet(h, log_abs_det, sign);
}

int hodlr_get_num_systems(hodlr_t h, int* nsys) {
  if (!h || !nsys) return HODLR_ERR_ARG;
  *nsys = h->nsys ? h->nsys : 1;
  return HODLR_OK;
}

int hodlr_forest_refine_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                               int ldx, double tol, int max_iter, int* iters, double* relres) {
  if (!h || nrhs < 1 || !d_b || !d_x || ldb < h->n || ldx < h->n || !(tol >= 0) || max_iter < 0)
    return HODLR_ERR_ARG;
  if (!h->nsys) return fail(h, HODLR_ERR_STATE, "not a forest (hodlr_create_forest)");
  int rc = hodlr_factorize(h);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev0, h->stream));
  rc = forest_refine_device(h, nrhs, d_b, ldb, d_x, ldx, tol, max_iter, iters, relres);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->t_solve = ms * 1e-3;
  return HODLR_OK;
}

int hodlr_create_fnptr(hodlr_t* out, int rows, int cols, double (*kernel)(int, int, void*),
                       void* data, int leaf_size) {
  (void)rows;
  (void)cols;
  (void)kernel;
  (void)data;
  (void)leaf_size;
  if (out) *out = nullptr;
  return HODLR_ERR_UNSUPPORTED;
}

void hodlr_destroy(hodlr_t h) {
  if (!h) return;
  free_compress(h);
  dfree(h, h->d_pts);
  dfree(h, h->d_A);
  dfree(h, h->d_leaf_min);
  dfree(h, h->d_leaf_size);
  dfree(h, h->ws);
  dfree(h, h->Z);
  dfree(h, h->X);
  dfree(h, h->zs);
  dfree(h, h->ir_b);
  dfree(h, h->ir_x);
  dfree(h, h->ir_y);
  dfree(h, h->ir_part);
  dfree(h, h->gm_V);
  dfree(h, h->gm_Z);
  dfree(h, h->gm_W);
  dfree(h, h->gm_h);
  dfree(h, h->gm_part);
  dfree(h, h->part);
  dfree(h, h->bar);
  dfree(h, h->d_blocks);
  dfree(h, h->d_cta);
  dfree(h, h->dotg);
  dfree(h, h->d_kps);
  dfree(h, h->d_psys);
  dfree(h, h->d_sysoff);
  dfree(h, h->d_fitems);
  dfree(h, h->d_fnorm);
  dfree(h, h->d_model);
  dfree(h, h->d_err);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->pin) cudaFreeHost(h->pin);
  h->pool.release_all(h->stream);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

int hodlr_reset(hodlr_t h) {
  if (!h) return HODLR_ERR_ARG;
  free_compress(h);
  h->t_lr = h->t_fact = h->t_solve = 0;
  return HODLR_OK;
}

int hodlr_set_stream(hodlr_t h, void* stream) {
  if (!h) return HODLR_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  drop_solve_graph(h);
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return HODLR_OK;
}

int hodlr_set_precision(hodlr_t h, int precision) {
  if (!h || precision < HODLR_PRECISION_FP64 || precision > HODLR_PRECISION_TF32X3)
    return HODLR_ERR_ARG;
  if (precision != h->gemm_prec) {
    h->gemm_prec = precision;  // enum values coincide with HODLR_GEMM_*
    free_factor(h);  // the compression is kept, unless the factorization overwrote W
  }
  return HODLR_OK;
}

int hodlr_gemm_device(int precision, int mode, int m, int n, int k, const double* A, int lda,
                      const double* B, int ldb, double* C, int ldc, void* stream) {
  if (precision < HODLR_PRECISION_FP64 || precision > HODLR_PRECISION_TF32X3 || mode < 0 ||
      mode > 1 || m < 0 || n < 0 || k < 0 || !A || !B || !C || ldc < m ||
      lda < (mode == 0 ? k : m) || ldb < k)
    return HODLR_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<GemmProblem> probs(1);
  GemmProblem& p = probs[0];
  p = GemmProblem{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.M = m;
  p.N = n;
  p.K = k;
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  std::vector<int4> tiles;
  int64_t ws = 0;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (precision == HODLR_PRECISION_FP64)
    gemm_plan(probs, tiles, ws, mode == 0, 8 * sms);
  else
    umma_plan(probs, tiles, ws, mode == 0, 8 * sms);
  GemmProblem* dp = nullptr;
  int4* dt = nullptr;
  double* dws = nullptr;
  unsigned* derr = nullptr;
  int rc = HODLR_OK;
  if (cudaMalloc(&dp, sizeof(GemmProblem)) != cudaSuccess ||
      (tiles.size() && cudaMalloc(&dt, sizeof(int4) * tiles.size()) != cudaSuccess) ||
      (ws && cudaMalloc(&dws, sizeof(double) * ws) != cudaSuccess) ||
      cudaMalloc(&derr, sizeof(unsigned)) != cudaSuccess)
    rc = HODLR_ERR_ALLOC;
  if (!rc) {
    cudaMemcpyAsync(dp, probs.data(), sizeof(GemmProblem), cudaMemcpyHostToDevice, s);
    if (tiles.size())
      cudaMemcpyAsync(dt, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(derr, 0, sizeof(unsigned), s);
    const bool split = probs[0].splits > 1;
    int e;
    if (precision == HODLR_PRECISION_FP64)
      e = mode == 0 ? gemm_tn_launch(dp, dt, (int)tiles.size(), 1, dws, split, s)
                    : gemm_nn_sub_launch(dp, dt, (int)tiles.size(), s);
    else
      e = mode == 0 ? umma_tn_launch(precision, dp, dt, (int)tiles.size(), 1, dws, split, derr, s)
                    : umma_nn_sub_launch(precision, dp, dt, (int)tiles.size(), derr, s);
    if (e || cudaStreamSynchronize(s) != cudaSuccess) rc = HODLR_ERR_CUDA;
    unsigned he = 0;
    if (!rc && cudaMemcpyAsync(&he, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess && he)
      rc = HODLR_ERR_TIMEOUT;
  }
  cudaFree(dp);
  cudaFree(dt);
  cudaFree(dws);
  cudaFree(derr);
  return rc;
}

int hodlr_set_rank_model(hodlr_t h, const float* params, double length_scale) {
  if (!h) return HODLR_ERR_ARG;
  if (!params) {
    dfree(h, h->d_model);
    return HODLR_OK;
  }
  if (h->dense) return fail(h, HODLR_ERR_UNSUPPORTED, "the rank model needs point coordinates");
  if (h->nsys) return fail(h, HODLR_ERR_UNSUPPORTED, "the rank model takes one length scale, not a forest");
  if (!(length_scale > 0)) return HODLR_ERR_ARG;
  for (int i = 0; i < HODLR_MLP_PARAMS; ++i)
    if (!std::isfinite(params[i])) return fail(h, HODLR_ERR_ARG, "non-finite model parameter");
  if (!h->d_model) CK(dalloc(h, &h->d_model, (size_t)HODLR_MLP_PARAMS));
  CK(h2d(h, h->d_model, params, sizeof(float) * HODLR_MLP_PARAMS));
  h->model_l = length_scale;
  return HODLR_OK;
}

int hodlr_get_predicted_ranks(hodlr_t h, int* ranks) {
  if (!h || !ranks) return HODLR_ERR_ARG;
  if (!h->d_model) return fail(h, HODLR_ERR_STATE, "no rank model set");
  int rc = predict_ranks(h);
  if (rc) return rc;
  std::copy(h->pred.begin(), h->pred.end(), ranks);
  return HODLR_OK;
}

int hodlr_block_features(hodlr_t h, double length_scale, float* features) {
  if (!h || !features || !(length_scale > 0)) return HODLR_ERR_ARG;
  if (h->dense) return fail(h, HODLR_ERR_UNSUPPORTED, "block features need point coordinates");
  const std::vector<int4> geom = block_geoms(h);
  const int nb = (int)geom.size();
  if (nb == 0) return HODLR_OK;
  float* d_F = nullptr;
  CK(dalloc(h, &d_F, (size_t)nb * HODLR_MLP_INPUTS));
  int rc = block_features_dev(h, geom, length_scale, d_F);
  if (rc) return rc;
  CK(d2h(h, features, d_F, sizeof(float) * nb * HODLR_MLP_INPUTS));
  dfree(h, d_F);
  return HODLR_OK;
}

int hodlr_mlp_scratch_floats(int batch, long long* floats) {
  if (batch < 1 || !floats) return HODLR_ERR_ARG;
  *floats = (long long)batch * mlp_sample_floats();
  return HODLR_OK;
}

int hodlr_mlp_forward(const float* d_params, const float* d_X, int batch, float* d_y,
                      void* stream) {
  if (!d_params || !d_X || !d_y || batch < 1) return HODLR_ERR_ARG;
  int e = mlp_forward_launch(d_params, d_X, batch, d_y, (cudaStream_t)stream);
  if (e || cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return HODLR_ERR_CUDA;
  return HODLR_OK;
}

int hodlr_mlp_train_step(float* d_params, float* d_m1, float* d_m2, const float* d_X,
                         const float* d_T, int batch, float* d_scratch, float lr, int step,
                         float* d_grad, float* d_loss, void* stream) {
  if (!d_params || !d_X || !d_T || !d_scratch || batch < 1) return HODLR_ERR_ARG;
  if (lr > 0 && (!d_m1 || !d_m2 || step < 1)) return HODLR_ERR_ARG;
  int e = mlp_train_launch(d_params, d_m1, d_m2, d_X, d_T, batch, d_scratch, lr, step, d_grad,
                           d_loss, (cudaStream_t)stream);
  return e ? HODLR_ERR_CUDA : HODLR_OK;
}

int hodlr_trim_device_memory(void) {
  cudaMemPool_t mp = device_pool();
  if (!mp) return HODLR_ERR_CUDA;
  if (cudaDeviceSynchronize() != cudaSuccess) return HODLR_ERR_CUDA;
  return cudaMemPoolTrimTo(mp, 0) == cudaSuccess ? HODLR_OK : HODLR_ERR_CUDA;
}

int hodlr_set_capacity_hint(hodlr_t h, const int* caps, int nlevels) {
  if (!h || nlevels < 0 || (nlevels > 0 && !caps)) return HODLR_ERR_ARG;
  h->cap_hint.assign(caps, caps + nlevels);
  return HODLR_OK;
}

int hodlr_set_wait_limit(hodlr_t h, unsigned polls, int unreachable) {
  if (!h || unreachable < 0 || unreachable > 1) return HODLR_ERR_ARG;
  h->spin_limit = polls;
  h->bar_unreachable = unreachable != 0;
  return HODLR_OK;
}

int hodlr_set_solver_form(hodlr_t h, int form) {
  if (!h || (form != HODLR_FORM_RECLU && form != HODLR_FORM_RECSM)) return HODLR_ERR_ARG;
  const bool sm = form == HODLR_FORM_RECSM;
  if (sm != h->sm_form) {
    CK(cudaStreamSynchronize(h->stream));
    free_factor(h);  // the compression is kept, unless a factorization overwrote W
    h->sm_form = sm;
  }
  return HODLR_OK;
}

int hodlr_get_solver_form(hodlr_t h, int* form) {
  if (!h || !form) return HODLR_ERR_ARG;
  *form = h->sm_form ? HODLR_FORM_RECSM : HODLR_FORM_RECLU;
  return HODLR_OK;
}

int hodlr_set_checked(hodlr_t h, int on) {
  if (!h || on < 0 || on > 1) return HODLR_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  h->checked = on != 0;
  return HODLR_OK;
}

int hodlr_set_aca_streaming(hodlr_t h, int on) {
  if (!h || on < 0 || on > 2) return HODLR_ERR_ARG;
  h->aca_ring = on != 0;
  h->aca_ring_tile = on == 2;
  return HODLR_OK;
}

int hodlr_set_factor_in_place(hodlr_t h, int mode) {
  if (!h || mode < -1 || mode > 1) return HODLR_ERR_ARG;
  if (mode != h->in_place) {
    h->in_place = mode;
    free_factor(h);
  }
  return HODLR_OK;
}

int hodlr_get_factor_in_place(hodlr_t h, int* levels) {
  if (!h || !levels) return HODLR_ERR_ARG;
  int c = 0;
  for (auto& L : h->lv) c += L.y_alias ? 1 : 0;
  *levels = c;
  return HODLR_OK;
}

int hodlr_get_launch_count(hodlr_t h, long long* count) {
  if (!h || !count) return HODLR_ERR_ARG;
  *count = h->nlaunch;
  return HODLR_OK;
}

int hodlr_set_lr_tolerance(hodlr_t h, double tol) {
  if (!h || !(tol > 0)) return HODLR_ERR_ARG;
  if (tol != h->tol) {
    h->tol = tol;
    free_compress(h);
  }
  return HODLR_OK;
}

int hodlr_set_min_pivot(hodlr_t h, double mp) {
  if (!h || mp < 0) return HODLR_ERR_ARG;
  int v = (int)mp;
  if (v != h->minPivot) {
    h->minPivot = v;
    free_compress(h);
  }
  return HODLR_OK;
}

int hodlr_set_lr_method(hodlr_t h, const char* method) {
  if (!h || !method) return HODLR_ERR_ARG;
  if (std::strcmp(method, "partialPiv_ACA") != 0)
    return fail(h, HODLR_ERR_UNSUPPORTED, std::string("low-rank method not on the GPU path: ") + method);
  return HODLR_OK;
}

int hodlr_compress(hodlr_t h) {
  if (!h) return HODLR_ERR_ARG;
  if (h->compressed) return HODLR_OK;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, h->stream));
  int rc = do_compress(h);
  CK(cudaEventRecord(b, h->stream));
  CK(cudaEventSynchronize(b));
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (!rc) h->t_lr = ms * 1e-3;
  return rc;
}

int hodlr_factorize(hodlr_t h) {
  if (!h) return HODLR_ERR_ARG;
  int rc = hodlr_compress(h);
  if (rc) return rc;
  return do_factorize(h);
}

int hodlr_solve(hodlr_t h, int nrhs, const double* b, int ldb, double* x, int ldx) {
  if (!h || nrhs < 1 || !b || !x || ldb < h->n || ldx < h->n) return HODLR_ERR_ARG;
  int rc = hodlr_factorize(h);
  if (rc) return rc;
  return do_solve_device(h, nrhs, b, ldb, x, ldx, true);
}

int hodlr_solve_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x, int ldx) {
  if (!h || nrhs < 1 || !d_b || !d_x || ldb < h->n || ldx < h->n) return HODLR_ERR_ARG;
  int rc = hodlr_factorize(h);
  if (rc) return rc;
  return do_solve_device(h, nrhs, d_b, ldb, d_x, ldx, false);
}

int hodlr_kernel_matvec_device(hodlr_t h, int nrhs, const double* d_x, int ldx, double* d_y,
                               int ldy) {
  if (!h || nrhs < 1 || nrhs > 16 || !d_x || !d_y || ldx < h->n || ldy < h->n)
    return HODLR_ERR_ARG;
  int rc = kmatvec_dev(h, nrhs, d_x, ldx, d_y, ldy);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return HODLR_OK;
}

int hodlr_solve_refined_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                               int ldx, double tol, int max_iter, int* iters, double* relres) {
  if (!h || nrhs < 1 || !d_b || !d_x || ldb < h->n || ldx < h->n || !(tol >= 0) || max_iter < 0)
    return HODLR_ERR_ARG;
  int rc = hodlr_factorize(h);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev0, h->stream));
  rc = refine_device(h, nrhs, d_b, ldb, d_x, ldx, tol, max_iter, iters, relres);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->t_solve = ms * 1e-3;
  return HODLR_OK;
}

int hodlr_iterative_solve_device(hodlr_t h, int nrhs, const double* d_b, int ldb, double* d_x,
                                 int ldx, double tol, int max_iter, int restart, int* iters,
                                 double* relres) {
  if (!h || nrhs < 1 || !d_b || !d_x || ldb < h->n || ldx < h->n || !(tol >= 0) ||
      max_iter < 0 || restart < 1 || restart > 256)
    return HODLR_ERR_ARG;
  int rc = hodlr_factorize(h);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev0, h->stream));
  rc = gmres_device(h, nrhs, d_b, ldb, d_x, ldx, tol, max_iter, restart, iters, relres);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->t_solve = ms * 1e-3;
  return HODLR_OK;
}

int hodlr_iterative_solve(hodlr_t h, int nrhs, const double* b, int ldb, double* x, int ldx,
                          double tol, int max_iter, int restart, int* iters, double* relres) {
  if (!h || nrhs < 1 || !b || !x || ldb < h->n || ldx < h->n) return HODLR_ERR_ARG;
  const int64_t N = h->n;
  double *db = nullptr, *dx = nullptr;
  CK(dalloc(h, &db, (size_t)(N * nrhs)));
  cudaError_t e = dalloc(h, &dx, (size_t)(N * nrhs));
  if (e != cudaSuccess) {
    dfree(h, db);
    return cuda_fail(h, e, "gmres alloc");
  }
  int rc = HODLR_OK;
  e = copy2d(h, db, sizeof(double) * N, b, sizeof(double) * ldb, sizeof(double) * N, nrhs,
             cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = hodlr_iterative_solve_device(h, nrhs, db, (int)N, dx, (int)N, tol, max_iter, restart,
                                      iters, relres);
    if (!rc)
      e = copy2d(h, x, sizeof(double) * ldx, dx, sizeof(double) * N, sizeof(double) * N, nrhs,
                 cudaMemcpyDeviceToHost);
  }
  dfree(h, db);
  dfree(h, dx);
  if (e != cudaSuccess) return cuda_fail(h, e, "gmres copy");
  return rc;
}

int hodlr_solve_refined(hodlr_t h, int nrhs, const double* b, int ldb, double* x, int ldx,
                        double tol, int max_iter, int* iters, double* relres) {
  if (!h || nrhs < 1 || !b || !x || ldb < h->n || ldx < h->n) return HODLR_ERR_ARG;
  const int64_t N = h->n;
  double *db = nullptr, *dx = nullptr;
  CK(dalloc(h, &db, (size_t)(N * nrhs)));
  cudaError_t e = dalloc(h, &dx, (size_t)(N * nrhs));
  if (e != cudaSuccess) {
    dfree(h, db);
    return cuda_fail(h, e, "refine alloc");
  }
  int rc = HODLR_OK;
  e = copy2d(h, db, sizeof(double) * N, b, sizeof(double) * ldb, sizeof(double) * N, nrhs,
             cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = hodlr_solve_refined_device(h, nrhs, db, (int)N, dx, (int)N, tol, max_iter, iters,
                                    relres);
    if (!rc)
      e = copy2d(h, x, sizeof(double) * ldx, dx, sizeof(double) * N, sizeof(double) * N, nrhs,
                 cudaMemcpyDeviceToHost);
  }
  dfree(h, db);
  dfree(h, dx);
  if (e != cudaSuccess) return cuda_fail(h, e, "refine copy");
  return rc;
}

int hodlr_residual(hodlr_t h, int nrhs, const double* b, int ldb, const double* x, int ldx,
                   double* relres) {
  if (!h || nrhs < 1 || !b || !x || !relres || ldb < h->n || ldx < h->n) return HODLR_ERR_ARG;
  const int64_t N = h->n;
  double *dx = nullptr, *dy = nullptr;
  CK(dalloc(h, &dx, (size_t)(N * nrhs)));
  cudaError_t e = dalloc(h, &dy, (size_t)(N * nrhs));
  if (e != cudaSuccess) {
    dfree(h, dx);
    return cuda_fail(h, e, "residual alloc");
  }
  int rc = HODLR_OK;
  std::vector<double> y((size_t)(N * nrhs));
  e = copy2d(h, dx, sizeof(double) * N, x, sizeof(double) * ldx, sizeof(double) * N, nrhs,
             cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    for (int c0 = 0; c0 < nrhs && !rc; c0 += 16) {
      int nc = std::min(16, nrhs - c0);
      rc = hodlr_kernel_matvec_device(h, nc, dx + c0 * N, (int)N, dy + c0 * N, (int)N);
    }
    if (!rc) e = d2h(h, y.data(), dy, sizeof(double) * N * nrhs);
  }
  dfree(h, dx);
  dfree(h, dy);
  if (e != cudaSuccess) return cuda_fail(h, e, "residual");
  if (rc) return rc;
  for (int c = 0; c < nrhs; ++c) {
    long double num = 0, den = 0;
    for (int64_t i = 0; i < N; ++i) {
      long double bi = b[c * (int64_t)ldb + i];
      long double r = (long double)y[c * N + i] - bi;
      num += r * r;
      den += bi * bi;
    }
    relres[c] = den > 0 ? (double)std::sqrt(num / den) : (double)std::sqrt(num);
  }
  return HODLR_OK;
}

int hodlr_get_times(hodlr_t h, double* lr, double* factor, double* solve, double* total) {
  if (!h) return HODLR_ERR_ARG;
  if (lr) *lr = h->t_lr;
  if (factor) *factor = h->t_fact;
  if (solve) *solve = h->t_solve;
  if (total) *total = h->t_lr + h->t_fact + h->t_solve;
  return HODLR_OK;
}

int hodlr_get_num_levels(hodlr_t h, int* levels) {
  if (!h || !levels) return HODLR_ERR_ARG;
  *levels = (int)h->lv.size();
  return HODLR_OK;
}

int hodlr_get_num_blocks(hodlr_t h, int* blocks) {
  if (!h || !blocks) return HODLR_ERR_ARG;
  int t = 0;
  for (auto& L : h->lv) t += L.nblocks();
  *blocks = t;
  return HODLR_OK;
}

static bool locate(hodlr_t h, int block, int& l, int& q) {
  if (block < 0) return false;
  int base = 0;
  for (l = 0; l < (int)h->lv.size(); ++l) {
    int nb = h->lv[l].nblocks();
    if (block < base + nb) {
      q = block - base;
      return true;
    }
    base += nb;
  }
  return false;
}

int hodlr_get_block_info(hodlr_t h, int block, int* level, int* row0, int* col0, int* m, int* n,
                         int* rank, int* iters) {
  int l, q;
  if (!h || !locate(h, block, l, q)) return HODLR_ERR_ARG;
  int r0, c0, mm, nn;
  block_geom(h->lv[l], q, r0, c0, mm, nn);
  if (level) *level = l;
  if (row0) *row0 = r0;
  if (col0) *col0 = c0;
  if (m) *m = mm;
  if (n) *n = nn;
  bool have = h->compressed;
  if (rank) *rank = have ? h->lv[l].st[q].rank : -1;
  if (iters) *iters = have ? h->lv[l].st[q].iters : -1;
  return HODLR_OK;
}

int hodlr_get_ranks(hodlr_t h, int* ranks) {
  if (!h || !ranks) return HODLR_ERR_ARG;
  if (!h->compressed) return fail(h, HODLR_ERR_STATE, "not compressed");
  int t = 0;
  for (auto& L : h->lv)
    for (auto& s : L.st) ranks[t++] = s.rank;
  return HODLR_OK;
}

int hodlr_get_pivots(hodlr_t h, int block, int* rows, int* cols, int* count) {
  int l, q;
  if (!h || !locate(h, block, l, q) || !count) return HODLR_ERR_ARG;
  if (!h->compressed) return fail(h, HODLR_ERR_STATE, "not compressed");
  Level& L = h->lv[l];
  int r0, c0, m, n;
  block_geom(L, q, r0, c0, m, n);
  const int k = L.st[q].k;
  *count = k;
  if (k > 0) {
    if (rows) CK(d2h(h, rows, L.prow + r0, 4 * (size_t)k));
    if (cols) CK(d2h(h, cols, L.pcol + c0, 4 * (size_t)k));
  }
  return HODLR_OK;
}

int hodlr_get_lowrank(hodlr_t h, int block, double* W, double* V) {
  int l, q;
  if (!h || !locate(h, block, l, q)) return HODLR_ERR_ARG;
  if (!h->compressed) return fail(h, HODLR_ERR_STATE, "not compressed");
  if (h->lv[l].y_alias)
    return fail(h, HODLR_ERR_STATE, "W of this level was overwritten by the in-place factorization");
  Level& L = h->lv[l];
  int r0, c0, m, n;
  block_geom(L, q, r0, c0, m, n);
  const int r = L.st[q].rank;
  const int64_t N = h->n;
  if (W) CK(copy2d(h, W, sizeof(double) * m, L.W + r0, sizeof(double) * N, sizeof(double) * m, r, cudaMemcpyDeviceToHost));
  if (V) CK(copy2d(h, V, sizeof(double) * n, L.V + c0, sizeof(double) * N, sizeof(double) * n, r, cudaMemcpyDeviceToHost));
  return HODLR_OK;
}

int hodlr_get_block_margin(hodlr_t h, int block, double* margin, int* near) {
  int l, q;
  if (!h || !locate(h, block, l, q)) return HODLR_ERR_ARG;
  if (!h->compressed) return fail(h, HODLR_ERR_STATE, "not compressed");
  if (margin) *margin = h->lv[l].st[q].margin;
  if (near) *near = h->lv[l].st[q].near;
  return HODLR_OK;
}

int hodlr_get_aca_stats(hodlr_t h, int* launches, double* seconds, double* bytes) {
  if (!h) return HODLR_ERR_ARG;
  if (launches) *launches = h->aca_launches;
  if (seconds) *seconds = h->aca_seconds;
  if (bytes) *bytes = h->aca_bytes;
  return HODLR_OK;
}

const char* hodlr_status_string(int s) {
  switch (s) {
    case HODLR_OK: return "ok";
    case HODLR_ERR_ARG: return "invalid argument";
    case HODLR_ERR_CUDA: return "CUDA error";
    case HODLR_ERR_ALLOC: return "device memory exhausted";
    case HODLR_ERR_UNSUPPORTED: return "unsupported on the GPU path";
    case HODLR_ERR_SINGULAR: return "exact-zero pivot";
    case HODLR_ERR_STATE: return "call out of order";
    case HODLR_ERR_NONFINITE: return "non-finite value";
    case HODLR_ERR_TIMEOUT: return "device wait timed out";
    case HODLR_ERR_IO: return "file could not be read or written";
    default: return "unknown status";
  }
}

const char* hodlr_last_error(hodlr_t h) { return h ? h->err.c_str() : "null handle"; }

}  // extern "C"
