// storeLRinTree (src/HODLR_Matrix.cpp:257-272,274-430): partial-pivot ACA of
// every off-diagonal block, level by level (aca.cu kernels).
#include "handle.h"

namespace hodlr_impl {

// Grow level L to `cap` columns, keeping the first kcap ones.
int grow_level(hodlr_t h, Level& L, int cap) {
  const int64_t N = h->n;
  double *W2 = nullptr, *V2 = nullptr;
  CK(dalloc(h, &W2, (size_t)(N * cap)));
  cudaError_t e = dalloc(h, &V2, (size_t)(N * cap));
  if (e != cudaSuccess) {
    dfree(h, W2);
    return cuda_fail(h, e, "grow_level");
  }
  if (L.W && L.kcap > 0) {
    CK(cudaMemcpyAsync(W2, L.W, sizeof(double) * N * L.kcap, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(V2, L.V, sizeof(double) * N * L.kcap, cudaMemcpyDeviceToDevice, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  dfree(h, L.W);
  dfree(h, L.V);
  L.W = W2;
  L.V = V2;
  L.kcap = cap;
  return HODLR_OK;
}

void fill_block(hodlr_t h, Level& L, int q, AcaBlock& B) {
  int r0, c0, m, n;
  block_geom(L, q, r0, c0, m, n);
  (void)h;
  B.st = L.d_st + q;
  B.W = L.W + r0;
  B.V = L.V + c0;
  B.cR = L.cR + r0;
  B.cC = L.cC + c0;
  B.prow = L.prow + r0;
  B.pcol = L.pcol + c0;
  B.r0 = r0;
  B.c0 = c0;
  B.m = m;
  B.n = n;
  B.kcap = L.kcap;
  B.level = 0;
  B.g0 = 0;
  B.G = 1;
  const int p = q >> 1;
  B.minRank = (q & 1) ? L.bmin[p] : L.tmin[p];
  B.maxRank = (q & 1) ? L.bmax[p] : L.tmax[p];
}

bool level_done(const Level& L) {
  for (auto& s : L.st)
    if (s.status != ACA_DONE) return false;
  return true;
}

// Run one ACA launch over `blocks` with group size G.
// One ACA launch over `blocks`: groups of G CTAs each, or, with `groups`,
// groups[i] CTAs for block i (a CTA table maps CTAs to blocks).
int run_aca(hodlr_t h, std::vector<AcaBlock>& blocks, int G, int nt, int kcap_max,
            bool ring, const std::vector<int>* groups, const Level* arena) {
  const int nb = (int)blocks.size();
  if (nb == 0) return HODLR_OK;
  int ncta = nb * G;
  if (groups) {
    ncta = 0;
    for (int i = 0; i < nb; ++i) {
      blocks[i].g0 = ncta;
      blocks[i].G = (*groups)[i];
      ncta += (*groups)[i];
    }
    std::vector<int> table((size_t)ncta);
    for (int i = 0; i < nb; ++i)
      for (int c = 0; c < blocks[i].G; ++c) table[(size_t)(blocks[i].g0 + c)] = i;
    if (ncta > h->cta_cap) {
      dfree(h, h->d_cta);
      CK(dalloc(h, &h->d_cta, (size_t)ncta));
      h->cta_cap = ncta;
    }
    CK(cudaMemcpyAsync(h->d_cta, table.data(), sizeof(int) * ncta, cudaMemcpyHostToDevice,
                       h->stream));
  }
  if (nb > h->blocks_cap) {
    dfree(h, h->d_blocks);
    CK(dalloc(h, &h->d_blocks, (size_t)nb));
    h->blocks_cap = nb;
  }
  CK(cudaMemcpyAsync(h->d_blocks, blocks.data(), sizeof(AcaBlock) * nb, cudaMemcpyHostToDevice,
                     h->stream));
  int64_t stride = 12 + 4 * (int64_t)kcap_max;  // args + two banks of dots and norms
  int64_t need = stride * ncta;
  if (need > h->part_cap) {
    dfree(h, h->part);
    CK(dalloc(h, &h->part, (size_t)need));
    h->part_cap = need;
  }
  if (nb > h->bar_cap) {
    dfree(h, h->bar);
    CK(dalloc(h, &h->bar, (size_t)nb));
    h->bar_cap = nb;
  }
  CK(cudaMemsetAsync(h->bar, 0, sizeof(unsigned) * nb, h->stream));
  AcaLaunch L;
  L.blocks = h->d_blocks;
  L.nblocks = nb;
  L.G = G;
  L.ld = h->n;
  L.tol = h->tol;
  L.minPivot = (double)h->minPivot;
  L.kcap_max = kcap_max;
  L.part = h->part;
  L.part_stride = stride;
  L.bar = h->bar;
  L.err = h->d_err;
  L.src = make_src(h);
  L.cta_block = groups ? h->d_cta : nullptr;
  L.ncta = ncta;
  L.dotg = nullptr;
  L.dotg_stride = 0;
  L.ring = ring ? 1 : 0;
  L.ring_stages = ring ? aca_ring_stages(kcap_max) : 0;
  // one tensor copy per ring tile needs every block's panels in the level's
  // arenas (fill_block: W + r0, V + c0); a map that cannot be encoded keeps
  // the per-column copies
  L.ring_tile = 0;
  if (ring && h->aca_ring_tile && arena && arena->kcap == kcap_max)
    L.ring_tile = aca_ring_tile_maps(L, arena->W, arena->V, h->n, arena->kcap) ? 1 : 0;
  // slices of a group shorter than 768 rows: the 2-element instance (512-row
  // chunks) leaves fewer lanes idle than the 4-element one (1024-row chunks)
  L.narrow = 0;
  if (!ring && nt == 256 && G > 1) {
    int longest = 0;
    for (auto& b : blocks) longest = std::max(longest, std::max(b.m, b.n));
    L.narrow = (longest + G - 1) / G < 768 ? 1 : 0;
  }
  L.spin_limit = h->spin_limit ? h->spin_limit : HODLR_SPIN_LIMIT;
  L.bar_extra = h->bar_unreachable ? 1u : 0u;
  if (aca_smem_bytes(nt, kcap_max, ring, false) > 227 * 1024)
    return fail(h, HODLR_ERR_UNSUPPORTED, "block rank above the shared-memory limit of ACA");
  if (aca_dots_global(nt, kcap_max, ring, false)) {
    L.dotg_stride = (int64_t)(nt / 32) * kcap_max;
    const int64_t dneed = L.dotg_stride * ncta;
    if (dneed > h->dotg_cap) {
      dfree(h, h->dotg);
      CK(dalloc(h, &h->dotg, (size_t)dneed));
      h->dotg_cap = dneed;
    }
    L.dotg = h->dotg;
  }
  bool coop = G > 1;
  if (groups)
    for (int g : *groups) coop |= g > 1;
  CK(cudaEventRecord(h->ev0, h->stream));
  int rc = aca_launch(L, nt, kcap_max, coop, h->stream);
  if (rc == (int)cudaErrorCooperativeLaunchTooLarge) return HODLR_ERR_RETRY_SMALLER;
  if (rc) return cuda_fail(h, (cudaError_t)rc, "aca_launch");
  h->nlaunch += 1;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->aca_seconds += ms * 1e-3;
  h->aca_launches += 1;
  return check_dev_err(h, "ACA");
}

// Allocate the per-level arrays of level L with `cap` low-rank columns.
int init_level(hodlr_t h, Level& L, int cap) {
  const int64_t N = h->n;
  int rc = grow_level(h, L, std::max(1, std::min(L.ub_max, cap)));
  if (rc) return rc;
  CK(dalloc(h, &L.cR, (size_t)N));
  CK(dalloc(h, &L.cC, (size_t)N));
  CK(dalloc(h, &L.prow, (size_t)N));
  CK(dalloc(h, &L.pcol, (size_t)N));
  CK(cudaMemsetAsync(L.cR, 0, N, h->stream));
  CK(cudaMemsetAsync(L.cC, 0, N, h->stream));
  const int nb = L.nblocks();
  CK(dalloc(h, &L.d_st, (size_t)nb));
  L.st.assign(nb, AcaState());
  for (auto& s : L.st) {
    s.frob2 = 0;
    s.eps = 1;
    s.margin = HUGE_VAL;
    s.swp = s.svp = 0;
    s.k = 0;
    s.cur = 0;
    s.status = ACA_RUNNING;
    s.iters = 0;
    s.rank = 0;
    s.near = 0;
    s.pending = 0;
    s.pad = 0;
  }
  CK(cudaMemcpyAsync(L.d_st, L.st.data(), sizeof(AcaState) * nb, cudaMemcpyHostToDevice,
                     h->stream));
  return HODLR_OK;
}

// Read the level's block states back; grow the level where blocks paused for
// capacity and re-arm them.  *done = every block of the level finished.
int sync_level(hodlr_t h, Level& L, bool* done) {
  const int nb = L.nblocks();
  CK(cudaMemcpyAsync(L.st.data(), L.d_st, sizeof(AcaState) * nb, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  int need = 0;
  *done = true;
  for (auto& s : L.st) {
    if (s.status == ACA_ERROR) return fail(h, HODLR_ERR_TIMEOUT, "ACA group failed");
    if (s.status == ACA_NEED_CAP) need = std::max(need, L.kcap + std::max(32, L.kcap / 2));
    if (s.status == ACA_NEED_CAP_POST) need = std::max(need, s.rank);
    if (s.status != ACA_DONE) *done = false;
  }
  if (need > 0) {
    int cap = std::min(std::max(need, L.kcap + 1), std::max(L.ub_max, L.kcap + 1));
    int rc = grow_level(h, L, cap);
    if (rc) return rc;
    for (auto& s : L.st) {
      if (s.status == ACA_NEED_CAP) s.status = ACA_RUNNING;
      if (s.status == ACA_NEED_CAP_POST) s.status = ACA_POST;
    }
    CK(cudaMemcpyAsync(L.d_st, L.st.data(), sizeof(AcaState) * nb, cudaMemcpyHostToDevice,
                       h->stream));
  }
  return HODLR_OK;
}

int level_kmax(const Level& L) {
  int k = 0;
  for (auto& s : L.st) k = std::max(k, s.rank);
  return k;
}

// storeLRinTree (src/HODLR_Matrix.cpp:257-272,274-430) for every block.
// Levels with many blocks run together in one launch, one CTA per block
// (G = 1); the top levels, with few large blocks, run one cooperative launch
// each with a group of CTAs per block.  They go bottom-up so that each
// level's W/V capacity can be sized from the ranks of the level below it
// (ranks shrink down the tree); a level that needs more grows and resumes.
std::vector<int4> block_geoms(hodlr_t h) {
  std::vector<int4> geom;
  for (auto& L : h->lv)
    for (int q = 0; q < L.nblocks(); ++q) {
      int r0, c0, m, n;
      block_geom(L, q, r0, c0, m, n);
      geom.push_back(make_int4(r0, c0, m, n));
    }
  return geom;
}

// Features of every block (nb x HODLR_MLP_INPUTS, device) for length scale l.
int block_features_dev(hodlr_t h, const std::vector<int4>& geom, double l, float* d_F) {
  const int nb = (int)geom.size();
  int4* d_geom = nullptr;
  CK(dalloc(h, &d_geom, (size_t)nb));
  CK(cudaMemcpyAsync(d_geom, geom.data(), sizeof(int4) * nb, cudaMemcpyHostToDevice, h->stream));
  int e = block_features_launch(h->d_pts, h->n, h->dim, d_geom, nb, (float)std::log(l),
                                (float)std::log(h->tol), d_F, h->stream);
  if (e) return cuda_fail(h, (cudaError_t)e, "block features");
  h->nlaunch += 1;
  dfree(h, d_geom);
  return HODLR_OK;
}

// Predicted ACA rank of every block (level-major order, as
// hodlr_get_block_info numbers them) from the rank model: block features on
// the device, the MLP forward, rank = exp(y) - 1 rounded and clamped.
int predict_ranks(hodlr_t h) {
  const std::vector<int4> geom = block_geoms(h);
  const int nb = (int)geom.size();
  h->pred.assign(nb, 0);
  if (nb == 0) return HODLR_OK;
  float *d_F = nullptr, *d_y = nullptr;
  CK(dalloc(h, &d_F, (size_t)nb * HODLR_MLP_INPUTS));
  CK(dalloc(h, &d_y, (size_t)nb));
  int rc = block_features_dev(h, geom, h->model_l, d_F);
  if (rc) return rc;
  int e = mlp_forward_launch(h->d_model, d_F, nb, d_y, h->stream);
  if (e) return cuda_fail(h, (cudaError_t)e, "rank prediction");
  h->nlaunch += 1;
  std::vector<float> y((size_t)nb);
  CK(d2h(h, y.data(), d_y, sizeof(float) * nb));
  dfree(h, d_F);
  dfree(h, d_y);
  for (int i = 0; i < nb; ++i) {
    const double r = std::expm1((double)std::min(y[i], 20.0f));
    const int ub = std::min(geom[i].z, geom[i].w);
    h->pred[i] = std::max(0, std::min(ub, (int)std::lround(r)));
  }
  return HODLR_OK;
}

int do_compress(hodlr_t h) {
  if (h->compressed) return HODLR_OK;
  free_compress(h);
  h->aca_launches = 0;
  h->aca_seconds = 0;
  h->aca_bytes = 0;
  const int nlev = (int)h->lv.size();
  // predicted ranks, when a rank model is set: level capacities and the
  // order of the pooled blocks (largest predicted work first) follow them;
  // ACA's stopping test still decides every rank (a block that needs more
  // columns pauses and resumes after its level grows)
  std::vector<int> lbase(nlev + 1, 0);
  for (int l = 0; l < nlev; ++l) lbase[l + 1] = lbase[l] + h->lv[l].nblocks();
  const bool have_pred = h->d_model != nullptr;
  if (have_pred) {
    int rc = predict_ranks(h);
    if (rc) return rc;
  }
  auto pred = [&](int l, int q) { return h->pred[(size_t)(lbase[l] + q)]; };
  auto pred_cap = [&](int l) {
    int mx = 0;
    for (int q = 0; q < h->lv[l].nblocks(); ++q) mx = std::max(mx, pred(l, q));
    return std::max(16, ((mx + mx / 4 + 8) + 7) / 8 * 8);
  };
  auto hint = [&](int l) {
    if (l < (int)h->cap_hint.size() && h->cap_hint[l] > 0) return h->cap_hint[l];
    return have_pred ? pred_cap(l) : 0;
  };
  auto pred_or = [&](int l, int q) -> int64_t { return have_pred ? pred(l, q) + 1 : 1; };
  int per_sm = 0;
  if (aca_max_coresident(256, 256, false, false, &per_sm))
    return fail(h, HODLR_ERR_CUDA, "occupancy query failed");
  const int P0 = std::max(1, per_sm) * h->num_sms;
  std::vector<int> pooled_levels, group_levels;
  for (int l = 0; l < nlev; ++l)
    (h->lv[l].nblocks() * 2 > P0 ? pooled_levels : group_levels).push_back(l);
  // 1. the many-block levels, together
  for (int l : pooled_levels) {
    int rc = init_level(h, h->lv[l], hint(l) ? hint(l) : 64);
    if (rc) return rc;
  }
  for (int round = 0; round < 64 && !pooled_levels.empty(); ++round) {
    int kcap_max = 1;
    std::vector<std::pair<int64_t, AcaBlock>> sorted;
    for (int l : pooled_levels) {
      Level& L = h->lv[l];
      kcap_max = std::max(kcap_max, L.kcap);
      L.G = 1;
      for (int q = 0; q < L.nblocks(); ++q) {
        if (L.st[q].status == ACA_DONE) continue;
        AcaBlock B;
        fill_block(h, L, q, B);
        const int64_t k1 = pred_or(l, q);
        sorted.push_back({have_pred ? (int64_t)(B.m + B.n) * k1 * k1 : (int64_t)B.m * B.n, B});
      }
    }
    if (sorted.empty()) break;
    std::stable_sort(sorted.begin(), sorted.end(),
                     [](const std::pair<int64_t, AcaBlock>& a,
                        const std::pair<int64_t, AcaBlock>& b) { return a.first > b.first; });
    std::vector<AcaBlock> blocks;
    for (auto& pb : sorted) blocks.push_back(pb.second);
    int rc = run_aca(h, blocks, 1, 128, kcap_max);
    if (rc) return rc;
    bool all = true;
    for (int l : pooled_levels) {
      bool done;
      rc = sync_level(h, h->lv[l], &done);
      if (rc) return rc;
      all &= done;
    }
    if (all) break;
  }
  // 2. the few-block levels, deepest first
  int kmax_below = 0;
  if (!pooled_levels.empty()) kmax_below = level_kmax(h->lv[pooled_levels.front()]);
  for (auto it = group_levels.rbegin(); it != group_levels.rend(); ++it) {
    const int l = *it;
    Level& L = h->lv[l];
    int guess = hint(l) ? hint(l) : std::max(64, (kmax_below * 3 + 1) / 2 + 16);
    int rc = init_level(h, L, guess);
    if (rc) return rc;
    for (int round = 0; round < 64; ++round) {
      // the group levels stream their panels through the bulk-copy ring
      // (16-byte aligned columns need an even N) while that still leaves at
      // least two of its one-per-SM CTAs to every block
      const int nb = L.nblocks();
      int ps = 0, ps_ring = 0;
      const bool ring_fits = aca_ring_stages(L.kcap) >= 2;
      if (aca_max_coresident(256, L.kcap, false, false, &ps) ||
          (ring_fits && aca_max_coresident(512, L.kcap, true, false, &ps_ring)))
        return fail(h, HODLR_ERR_CUDA, "occupancy query failed");
      const bool ring = h->aca_ring && ring_fits && (h->n % 2 == 0) &&
                        ps_ring * h->num_sms >= 2 * nb;
      if (ring) ps = ps_ring;
      // equal groups: CTAs sized by predicted work measured 2-8% slower on
      // 3D clouds than equal groups (per-step latency, not streamed bytes,
      // sets a block's time)
      int G = std::max(1, std::max(1, ps) * h->num_sms / nb);
      std::vector<AcaBlock> bl(nb);
      for (;;) {  // a cooperative launch the driver refuses is retried with half the groups
        L.G = G;
        for (int q = 0; q < nb; ++q) fill_block(h, L, q, bl[q]);
        rc = run_aca(h, bl, G, ring ? 512 : G > 1 ? 256 : 128, L.kcap, ring, nullptr, &L);
        if (rc != HODLR_ERR_RETRY_SMALLER) break;
        if (G == 1) return fail(h, HODLR_ERR_CUDA, "aca_launch: cooperative launch refused");
        G = std::max(1, G / 2);
      }
      if (rc) return rc;
      bool done;
      rc = sync_level(h, L, &done);
      if (rc) return rc;
      if (done) break;
    }
    kmax_below = level_kmax(L);
  }
  for (auto& L : h->lv)
    if (!level_done(L)) return fail(h, HODLR_ERR_STATE, "ACA did not converge in 64 rounds");
  // ranks, level widths, column offsets, algorithmic bytes
  int64_t coff = 0;
  double bytes = 0;
  const double es = 8.0;  // bytes of a panel element
  for (auto& L : h->lv) {
    L.kmax = 0;
    for (int q = 0; q < L.nblocks(); ++q) {
      L.kmax = std::max(L.kmax, L.st[q].rank);
      int r0, c0, m, n;
      block_geom(L, q, r0, c0, m, n);
      // one read of the W and V panels per step (the norm dots ride along),
      // the two new columns and the coordinates of the entries evaluated
      double K = L.st[q].iters;
      bytes += (double)(m + n) * (es / 2.0 * K * (K - 1) + es * K + 8.0 * K * h->dim);
    }
    L.coff = (int)coff;
    coff += L.kmax;
  }
  h->C = coff;
  h->aca_bytes = bytes;
  h->compressed = true;
  return HODLR_OK;
}

}  // namespace hodlr_impl
