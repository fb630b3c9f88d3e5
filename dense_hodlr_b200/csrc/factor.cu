// recLU_Factorize (src/HODLR_Matrix.cpp:505-518,612-692) as bottom-up level
// sweeps: leaf LUs, the K^-1 U panels, the capacitance matrices and their LUs;
// the log-determinant from those factors.
#include "handle.h"

namespace hodlr_impl {

// split: TN problems (C = A^T B), which may be split along K; else NN.
int upload_plan(hodlr_t h, std::vector<GemmProblem>& probs, bool split, DevPlan& out,
                const char* what) {
  std::vector<int4> tiles;
  int64_t ws = 0;
  if (h->gemm_prec == HODLR_GEMM_FP64)
    gemm_plan(probs, tiles, ws, split, 2 * h->num_sms * 4);
  else
    umma_plan(probs, tiles, ws, split, 2 * h->num_sms * 4);
  free_plan(h, out);
  out.nprob = (int)probs.size();
  out.ntiles = (int)tiles.size();
  out.ws_elems = ws;
  out.any_split = false;
  for (auto& p : probs) out.any_split |= p.splits > 1;
  if (out.nprob) {
    CK(dalloc(h, &out.probs, (size_t)out.nprob));
    CK(h2d_async(h, out.probs, probs.data(), sizeof(GemmProblem) * out.nprob));
  }
  if (out.ntiles) {
    CK(dalloc(h, &out.tiles, (size_t)out.ntiles));
    CK(h2d_async(h, out.tiles, tiles.data(), sizeof(int4) * out.ntiles));
  }
  int rc = ensure_ws(h, ws);
  if (rc) return rc;
  return check_gemm(h, probs, split, what);
}

int level_rank(const Level& L, int q) { return L.st[q].rank; }

// Launch a planned TN / NN-sub group in the handle's arithmetic.
int run_tn(hodlr_t h, const DevPlan& P) {
  if (P.ntiles == 0) return 0;
  h->nlaunch += 1 + (P.any_split ? 1 : 0);
  if (h->gemm_prec == HODLR_GEMM_FP64)
    return gemm_tn_launch(P.probs, P.tiles, P.ntiles, P.nprob, h->ws, P.any_split, h->stream);
  return umma_tn_launch(h->gemm_prec, P.probs, P.tiles, P.ntiles, P.nprob, h->ws, P.any_split,
                        h->d_err, h->stream);
}

int run_nn(hodlr_t h, const DevPlan& P) {
  if (P.ntiles == 0) return 0;
  h->nlaunch += 1;
  if (h->gemm_prec == HODLR_GEMM_FP64)
    return gemm_nn_sub_launch(P.probs, P.tiles, P.ntiles, h->stream);
  return umma_nn_sub_launch(h->gemm_prec, P.probs, P.tiles, P.ntiles, h->d_err, h->stream);
}

// Y_l[rows of block q, c] = W_l[rows, c] for c < rank(q), 0 for rank(q) <= c
// < kmax.  With Y == W (in place) only the padding is written.
__global__ void y_init_kernel(double* Y, const double* W, int64_t ld, int kmax, const int* r0s,
                              const int* ms, const int* ranks, int nb) {
  int q = blockIdx.y;
  if (q >= nb) return;
  const int r0 = r0s[q], m = ms[q], rank = ranks[q];
  for (int c = blockIdx.z; c < kmax; c += gridDim.z) {
    if (c < rank && Y == W) continue;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
      Y[(int64_t)c * ld + r0 + i] = c < rank ? W[(int64_t)c * ld + r0 + i] : 0.0;
  }
}

// log|det| pieces of the factorization: per leaf LU (column-major s x s,
// final row permutation perm) and per capacitance LU (sd x sd, LAPACK-style
// swaps piv): out = (sum_i log|u_ii|, #u_ii < 0, permutation parity).
__global__ void leaf_logdet_kernel(const double* lu, const int64_t* lu_off, const int* leaf_min,
                                   const int* leaf_size, const int* perm, double* out) {
  if (threadIdx.x != 0) return;
  const int q = blockIdx.x, s = leaf_size[q];
  const double* g = lu + lu_off[q];
  const int* pm = perm + leaf_min[q];
  double sum = 0.0;
  int neg = 0;
  for (int i = 0; i < s; ++i) {
    const double d = g[(int64_t)i * s + i];
    sum += log(fabs(d));
    neg += d < 0.0;
  }
  unsigned char seen[160];
  for (int i = 0; i < s; ++i) seen[i] = 0;
  int cycles = 0;
  for (int i = 0; i < s; ++i) {
    if (seen[i]) continue;
    ++cycles;
    for (int j = i; !seen[j]; j = pm[j]) seen[j] = 1;
  }
  out[3 * q] = sum;
  out[3 * q + 1] = neg;
  out[3 * q + 2] = (s - cycles) & 1;
}

__global__ void schur_logdet_kernel(const SchurNode* nodes, const double* S, const int* piv,
                                    double* out) {
  if (threadIdx.x != 0) return;
  const SchurNode N = nodes[blockIdx.x];
  const int n = N.kb + N.kt;
  const double* a = S + N.s_off;
  const int* p = piv + N.p_off;
  double sum = 0.0;
  int neg = 0, swaps = 0;
  for (int i = 0; i < n; ++i) {
    const double d = a[(int64_t)i * n + i];
    sum += log(fabs(d));
    neg += d < 0.0;
    swaps += p[i] != i;
  }
  out[3 * blockIdx.x] = sum;
  out[3 * blockIdx.x + 1] = neg;
  out[3 * blockIdx.x + 2] = swaps & 1;
}

// Identity blocks on the leaves' diagonal of an N x smax panel (zeroed):
// X[r0 + i, i] = 1 for every leaf (r0, s), i < s.
__global__ void leaf_identity_kernel(double* X, int64_t ldx, const int* leaf_min,
                                     const int* leaf_size) {
  const int r0 = leaf_min[blockIdx.x], s = leaf_size[blockIdx.x];
  for (int i = threadIdx.x; i < s; i += blockDim.x) X[r0 + i + (int64_t)i * ldx] = 1.0;
}

int do_factorize(hodlr_t h) {
  if (h->factored) return HODLR_OK;
  free_factor(h);  // first: a factorization that overwrote W also drops the compression
  int rc = do_compress(h);
  if (rc) return rc;
  const int64_t N = h->n;
  CK(cudaEventRecord(h->ev0, h->stream));
  // leaves: assemble + LU
  const int nl = (int)h->leaf_min.size();
  std::vector<int64_t> lu_off(nl);
  int64_t tot = 0;
  for (int p = 0; p < nl; ++p) {
    lu_off[p] = tot;
    tot += (int64_t)h->leaf_size[p] * h->leaf_size[p];
  }
  CK(dalloc(h, &h->d_lu, (size_t)tot));
  CK(dalloc(h, &h->d_lu_off, (size_t)nl));
  CK(dalloc(h, &h->d_perm, (size_t)N));
  CK(h2d_async(h, h->d_lu_off, lu_off.data(), sizeof(int64_t) * nl));
  // the assembled leaf blocks (N x smax, leaf (r0, s) at rows r0.., columns
  // 0..s-1): the residual of the refinement step of K^-1 U below
  double* Aleaf = nullptr;
  if (h->C > 0) CK(dalloc(h, &Aleaf, (size_t)(N * h->smax)));
  {
    LeafLULaunch L;
    L.leaf_min = h->d_leaf_min;
    L.leaf_size = h->d_leaf_size;
    L.lu_off = h->d_lu_off;
    L.lu = h->d_lu;
    L.perm = h->d_perm;
    L.src = make_src(h);
    L.err = h->d_err;
    L.a_copy = Aleaf;
    L.lda_copy = N;
    int e = leaf_lu_launch(L, nl, h->smax, h->stream);
    if (e) return cuda_fail(h, (cudaError_t)e, "leaf_lu_launch");
    h->nlaunch += 1;
    rc = check_phase(h, "factor: leaf LU");
    if (rc) return rc;
    if (h->checked) {  // every leaf's row permutation is a permutation of its rows
      std::vector<int> perm(N);
      CK(d2h(h, perm.data(), h->d_perm, sizeof(int) * N));
      for (int p = 0; p < nl; ++p) {
        const int r0 = h->leaf_min[p], s = h->leaf_size[p];
        std::vector<char> seen(s, 0);
        for (int i = 0; i < s; ++i) {
          const int v = perm[r0 + i];
          if (v < 0 || v >= s || seen[v]) {
            char msg[160];
            snprintf(msg, sizeof msg, "factor: leaf %d (rows %d..%d) permutation entry %d = %d", p,
                     r0, r0 + s - 1, i, v);
            return fail(h, HODLR_ERR_CHECK, msg);
          }
          seen[v] = 1;
        }
      }
    }
  }
  // Y_l = the U panel of every level, zero padded to kmax columns: its own
  // allocation, or W_l itself (in place) when that cannot be had
  if (h->C > 0) {
    for (auto& L : h->lv) {
      if (L.kmax == 0) continue;
      const int nb = L.nblocks();
      std::vector<int> r0s(nb), ms(nb), rk(nb);
      for (int q = 0; q < nb; ++q) {
        int r0, c0, m, n;
        block_geom(L, q, r0, c0, m, n);
        r0s[q] = r0;
        ms[q] = m;
        rk[q] = level_rank(L, q);
      }
      L.y_alias = h->in_place == 1;
      if (!L.y_alias) {
        cudaError_t ea = dalloc(h, &L.Yl, (size_t)(N * L.kmax));
        if (ea == cudaErrorMemoryAllocation && h->in_place == -1) {
          cudaGetLastError();
          L.y_alias = true;
        } else if (ea != cudaSuccess) {
          return cuda_fail(h, ea, "K^-1 U panel");
        }
      }
      if (L.y_alias) {
        L.Yl = L.W;
        h->w_consumed = true;
      }
      int *d_r0 = nullptr, *d_m = nullptr, *d_rk = nullptr;
      CK(dalloc(h, &d_r0, nb));
      CK(dalloc(h, &d_m, nb));
      CK(dalloc(h, &d_rk, nb));
      CK(h2d_async(h, d_r0, r0s.data(), 4 * nb));
      CK(h2d_async(h, d_m, ms.data(), 4 * nb));
      CK(h2d_async(h, d_rk, rk.data(), 4 * nb));
      int maxm = 0;
      for (int m : ms) maxm = std::max(maxm, m);
      dim3 grid(std::min(64, (maxm + 255) / 256), nb, std::min(L.kmax, 64));
      y_init_kernel<<<grid, 256, 0, h->stream>>>(L.Yl, L.W, N, L.kmax, d_r0, d_m, d_rk, nb);
      CK(cudaGetLastError());
      h->nlaunch += 1;
      dfree(h, d_r0);  // reused only after the stream has drained (DevPool)
      dfree(h, d_m);
      dfree(h, d_rk);
    }
    // Y <- blockdiag(leaf)^-1 Y on every column.  Each leaf's inverse is
    // formed once (its LU applied to identity columns, smax columns in all)
    // and applied as grouped GEMMs: Y1 = A^-1 U, then one refinement step
    // Y = Y1 + A^-1 (U - A Y1).  A product with an explicit inverse alone is
    // not backward stable: on ill-conditioned systems (rank-capped user
    // trees) it left residuals 28x the reference's LU solves; the refined
    // product matches them, at three products per column instead of the
    // per-column substitutions of a leaf solve (4x faster here).
    const int sm = h->smax;
    int CH = 1;  // Y columns per product pass
    for (auto& L : h->lv) CH = std::max(CH, std::min(L.kmax, 512));
    double *Xinv = nullptr, *Y2 = nullptr;
    CK(dalloc(h, &Xinv, (size_t)(N * sm)));
    CK(dalloc(h, &Y2, (size_t)(N * CH)));
    CK(cudaMemsetAsync(Xinv, 0, sizeof(double) * N * sm, h->stream));
    leaf_identity_kernel<<<nl, 128, 0, h->stream>>>(Xinv, N, h->d_leaf_min, h->d_leaf_size);
    CK(cudaGetLastError());
    LeafSolveLaunch S;
    S.leaf_min = h->d_leaf_min;
    S.leaf_size = h->d_leaf_size;
    S.lu_off = h->d_lu_off;
    S.lu = h->d_lu;
    S.perm = h->d_perm;
    S.X = Xinv;
    S.ldx = N;
    S.ncols = sm;
    S.err = h->d_err;
    int e = leaf_solve_launch(S, nl, sm, h->stream);
    if (e) return cuda_fail(h, (cudaError_t)e, "leaf_solve_launch");
    rc = check_phase(h, "factor: leaf inverses");
    if (rc) return rc;
    // per level, in passes of CH columns through an N x CH buffer
    // three problem lists per pass (the same tiles): Y2 = Xinv Y; Y -= A Y2
    // (Y now holds the residual U - A Y1); Y2 += Xinv Y
    GemmProblem* d_probs = nullptr;
    int4* d_tiles = nullptr;
    size_t tiles_cap = 0;
    CK(dalloc(h, &d_probs, (size_t)(3 * nl)));
    for (auto& L : h->lv) {
      for (int c0 = 0; c0 < L.kmax; c0 += CH) {
        const int nc = std::min(CH, L.kmax - c0);
        double* Yc = L.Yl + (int64_t)c0 * N;
        std::vector<GemmProblem> probs[3];
        for (int p = 0; p < nl; ++p) {
          const int r0 = h->leaf_min[p], s = h->leaf_size[p];
          GemmProblem g{};
          g.M = s;
          g.N = nc;
          g.K = s;
          g.lda = g.ldb = g.ldc = (int)N;
          g.A = Xinv + r0;  // Y2 = Xinv Y
          g.B = Yc + r0;
          g.C = Y2 + r0;
          probs[0].push_back(g);
          g.A = Aleaf + r0;  // Y -= A Y2
          g.B = Y2 + r0;
          g.C = Yc + r0;
          probs[1].push_back(g);
          g.A = Xinv + r0;  // Y2 += Xinv Y
          g.B = Yc + r0;
          g.C = Y2 + r0;
          probs[2].push_back(g);
        }
        std::vector<int4> tiles;
        int64_t ws = 0;
        for (auto& pr : probs) gemm_plan(pr, tiles, ws, false, 0);  // same tiles each time
        if (tiles.size() > tiles_cap) {
          dfree(h, d_tiles);
          CK(dalloc(h, &d_tiles, tiles.size()));
          tiles_cap = tiles.size();
        }
        for (int q = 0; q < 3; ++q)
          CK(h2d_async(h, d_probs + (size_t)q * nl, probs[q].data(), sizeof(GemmProblem) * nl));
        CK(h2d_async(h, d_tiles, tiles.data(), sizeof(int4) * tiles.size()));
        for (int q = 0; q < 3; ++q) {
          rc = check_gemm(h, probs[q], false, "factor: leaf inverse product");
          if (rc) return rc;
        }
        const int nt = (int)tiles.size();
        e = gemm_nn_launch(d_probs, d_tiles, nt, h->stream);
        if (!e) e = gemm_nn_sub_launch(d_probs + nl, d_tiles, nt, h->stream);
        if (!e) e = gemm_nn_add_launch(d_probs + 2 * nl, d_tiles, nt, h->stream);
        if (e) return cuda_fail(h, (cudaError_t)e, "leaf inverse product");
        rc = check_phase(h, "factor: leaf inverse product");
        if (rc) return rc;
        CK(cudaMemcpyAsync(Yc, Y2, sizeof(double) * N * nc, cudaMemcpyDeviceToDevice, h->stream));
        h->nlaunch += 3;
      }
    }
    h->nlaunch += 2;
    dfree(h, Y2);
    dfree(h, Xinv);
    dfree(h, Aleaf);
    dfree(h, d_probs);
    dfree(h, d_tiles);
  }
  // levels bottom-up
  for (int l = (int)h->lv.size() - 1; l >= 0; --l) {
    Level& L = h->lv[l];
    const int nn = (int)L.nmin.size();
    L.nodes.resize(nn);
    int64_t s_tot = 0, z_tot = 0, p_tot = 0;
    L.max_sd = 0;
    for (int p = 0; p < nn; ++p) {
      SchurNode& sn = L.nodes[p];
      sn.kt = level_rank(L, 2 * p);
      sn.kb = level_rank(L, 2 * p + 1);
      sn.coff = L.coff;
      sn.order = h->sm_form ? 1 : 0;
      const int sd = sn.kb + sn.kt;
      L.max_sd = std::max(L.max_sd, sd);
      sn.s_off = s_tot;
      s_tot += (int64_t)sd * sd;
      sn.z_off = z_tot;
      sn.r_off = z_tot;
      z_tot += (int64_t)sd * (L.coff + std::max(sn.kb, sn.kt));
      sn.p_off = p_tot;
      p_tot += sd;
    }
    CK(dalloc(h, &L.S, (size_t)s_tot));
    CK(dalloc(h, &L.piv, (size_t)p_tot));
    CK(dalloc(h, &L.d_nodes, (size_t)nn));
    CK(h2d_async(h, L.d_nodes, L.nodes.data(), sizeof(SchurNode) * nn));
    if (z_tot > h->z_cap) {
      dfree(h, h->Z);
      CK(dalloc(h, &h->Z, (size_t)z_tot));
      h->z_cap = z_tot;
    }
    // Z_h = V_h^T [Y_0 .. Y_{l-1} | own U columns of Y_l] on the node's rows:
    // Z columns [coff_a, coff_a + kmax_a) from level a < l, then the own
    // rank(U_h) columns at coff_l, one grouped-GEMM problem per panel
    std::vector<GemmProblem> tn;
    for (int p = 0; p < nn; ++p) {
      const SchurNode& sn = L.nodes[p];
      const int sd = sn.kb + sn.kt;
      const int mn = L.nmin[p], sp = L.nsplit[p], mx = L.nmax[p];
      for (int a = 0; a <= l; ++a) {
        const Level& A = h->lv[a];
        const int ncols_t = a < l ? A.kmax : sn.kt, ncols_b = a < l ? A.kmax : sn.kb;
        if (ncols_t > 0 && sn.kb > 0) {
          GemmProblem t{};
          t.A = L.V + mn;  // V of the bottom block lives on the top rows
          t.M = sn.kb;
          t.K = sp - mn + 1;
          t.lda = (int)N;
          t.B = A.Yl + mn;
          t.N = ncols_t;
          t.ldb = (int)N;
          t.C = h->Z + sn.z_off + (int64_t)A.coff * sd + (h->sm_form ? sn.kt : 0);
          t.ldc = sd;
          tn.push_back(t);
        }
        if (ncols_b > 0 && sn.kt > 0) {
          GemmProblem b{};
          b.A = L.V + sp + 1;  // V of the top block lives on the bottom rows
          b.M = sn.kt;
          b.K = mx - sp;
          b.lda = (int)N;
          b.B = A.Yl + sp + 1;
          b.N = ncols_b;
          b.ldb = (int)N;
          b.C = h->Z + sn.z_off + (int64_t)A.coff * sd + (h->sm_form ? 0 : sn.kb);
          b.ldc = sd;
          tn.push_back(b);
        }
      }
    }
    int rc2 = upload_plan(h, tn, true, L.tn, "factor: V^T Y products");
    if (rc2) return rc2;
    int e = run_tn(h, L.tn);
    if (e) return cuda_fail(h, (cudaError_t)e, "gemm_tn");
    rc2 = check_phase(h, "factor: V^T Y products");
    if (rc2) return rc2;
    rc2 = check_extent(h, L.S, sizeof(double) * s_tot, "capacitance matrices", "factor");
    if (!rc2) rc2 = check_extent(h, L.piv, sizeof(int) * p_tot, "capacitance pivots", "factor");
    if (!rc2) rc2 = check_extent(h, h->Z, sizeof(double) * z_tot, "Schur right-hand sides", "factor");
    if (rc2) return rc2;
    SchurLaunch S;
    S.nodes = L.d_nodes;
    S.S = L.S;
    S.Z = h->Z;
    S.R = h->Z;
    S.piv = L.piv;
    S.err = h->d_err;
    std::vector<int> sds(nn);
    for (int p = 0; p < nn; ++p) sds[p] = L.nodes[p].kb + L.nodes[p].kt;
    e = schur_factor_launch(S, nn, sds.data(), h->stream);
    if (e) return cuda_fail(h, (cudaError_t)e, "schur_factor");
    h->nlaunch += schur_factor_launches(sds.data(), nn);
    rc2 = check_phase(h, "factor: capacitance LU");
    if (rc2) return rc2;
    if (h->checked) {  // LAPACK-style interchanges: piv[p] in [p, sd)
      std::vector<int> piv(p_tot);
      CK(d2h(h, piv.data(), L.piv, sizeof(int) * p_tot));
      for (int p = 0; p < nn; ++p) {
        const SchurNode& sn = L.nodes[p];
        const int sd = sn.kb + sn.kt;
        for (int i = 0; i < sd; ++i) {
          const int q = piv[sn.p_off + i];
          if (q < i || q >= sd) {
            char msg[192];
            snprintf(msg, sizeof msg,
                     "factor: level %d node %d (sd %d, %s LU) pivot %d = %d", l, p, sd,
                     sd >= SCHUR_BIG_SD ? "multi-CTA" : "one-CTA", i, q);
            return fail(h, HODLR_ERR_CHECK, msg);
          }
        }
      }
    }
    if (L.coff > 0) {
      int nl_solve = 0;
      e = schur_solve_factor_launch(S, nn, sds.data(), L.coff, h->stream, &nl_solve);
      if (e) return cuda_fail(h, (cudaError_t)e, "schur_solve");
      h->nlaunch += nl_solve;
      rc2 = check_phase(h, "factor: ancestor-column solve");
      if (rc2) return rc2;
      // Y_a[rows_h] -= Y_l[rows_h, 0 : rank(U_h)] * y_h[:, level a's columns]
      // for every ancestor level a < l
      std::vector<GemmProblem> up;
      for (int p = 0; p < nn; ++p) {
        const SchurNode& sn = L.nodes[p];
        const int sd = sn.kb + sn.kt;
        const int mn = L.nmin[p], sp = L.nsplit[p], mx = L.nmax[p];
        for (int a = 0; a < l; ++a) {
          const Level& A = h->lv[a];
          if (A.kmax == 0) continue;
          if (sn.kt > 0) {
            GemmProblem t{};
            t.C = A.Yl + mn;
            t.ldc = (int)N;
            t.A = L.Yl + mn;
            t.lda = (int)N;
            t.M = sp - mn + 1;
            t.K = sn.kt;
            t.B = h->Z + sn.z_off + (h->sm_form ? 0 : sn.kb) + (int64_t)A.coff * sd;
            t.ldb = sd;
            t.N = A.kmax;
            up.push_back(t);
          }
          if (sn.kb > 0) {
            GemmProblem b{};
            b.C = A.Yl + sp + 1;
            b.ldc = (int)N;
            b.A = L.Yl + sp + 1;
            b.lda = (int)N;
            b.M = mx - sp;
            b.K = sn.kb;
            b.B = h->Z + sn.z_off + (h->sm_form ? sn.kt : 0) + (int64_t)A.coff * sd;
            b.ldb = sd;
            b.N = A.kmax;
            up.push_back(b);
          }
        }
      }
      rc2 = upload_plan(h, up, false, L.nn, "factor: Y updates");
      if (rc2) return rc2;
      e = run_nn(h, L.nn);
      if (e) return cuda_fail(h, (cudaError_t)e, "gemm_nn_sub");
      rc2 = check_phase(h, "factor: Y updates");
      if (rc2) return rc2;
    }
  }
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->t_fact = ms * 1e-3;
  rc = check_dev_err(h, "factorize");
  if (rc) return rc;
  h->factored = true;
  return HODLR_OK;
}

// log|det K| and its sign from the factorization's leaf and capacitance LUs.
int do_logdet(hodlr_t h, double* log_abs_det, int* sign) {
  int rc = do_factorize(h);
  if (rc) return rc;
  const int nl = (int)h->leaf_min.size();
  int nmax = nl;
  for (auto& L : h->lv) nmax = std::max(nmax, (int)L.nmin.size());
  double* d_out = nullptr;
  CK(dalloc(h, &d_out, (size_t)3 * nmax));
  std::vector<double> out((size_t)3 * nmax);
  leaf_logdet_kernel<<<nl, 32, 0, h->stream>>>(h->d_lu, h->d_lu_off, h->d_leaf_min,
                                               h->d_leaf_size, h->d_perm, d_out);
  CK(cudaGetLastError());
  CK(d2h(h, out.data(), d_out, sizeof(double) * 3 * nl));
  double sum = 0.0;
  long long flips = 0;
  for (int q = 0; q < nl; ++q) {
    sum += out[3 * q];
    flips += (long long)out[3 * q + 1] + (long long)out[3 * q + 2];
  }
  // det K = prod_leaves det(leaf) * prod_nodes det(S_node) (Sylvester's
  // identity at every node of the Woodbury recursion)
  for (auto& L : h->lv) {
    const int nn = (int)L.nmin.size();
    if (!nn) continue;
    schur_logdet_kernel<<<nn, 32, 0, h->stream>>>(L.d_nodes, L.S, L.piv, d_out);
    CK(cudaGetLastError());
    CK(d2h(h, out.data(), d_out, sizeof(double) * 3 * nn));
    for (int q = 0; q < nn; ++q) {
      sum += out[3 * q];
      flips += (long long)out[3 * q + 1] + (long long)out[3 * q + 2];
    }
  }
  h->nlaunch += 1 + (int)h->lv.size();
  dfree(h, d_out);
  *log_abs_det = sum;
  if (sign) *sign = (flips & 1) ? -1 : 1;
  return check_dev_err(h, "logdet");
}

}  // namespace hodlr_impl
