// Device memory, host<->device copies, error words and handle set-up shared
// by the host orchestration units (handle.h).
#include "handle.h"

namespace hodlr_impl {

// Device memory of every handle on a device comes from one stream-ordered
// pool owned by the library (cudaMallocFromPoolAsync / cudaFreeAsync) whose
// release threshold keeps freed memory reserved, so a new handle for the next
// system reuses the previous one's arenas instead of paying cudaMalloc /
// cudaFree for gigabytes.  hodlr_trim_device_memory hands it back.
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

cudaMemPool_t device_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) return it->second;
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  g_pools[dev] = pool;
  return pool;
}

int fail(hodlr_t h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(hodlr_t h, cudaError_t e, const char* where) {
  return fail(h, e == cudaErrorMemoryAllocation ? HODLR_ERR_ALLOC : HODLR_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorString(e));
}

void free_plan(hodlr_t h, DevPlan& p) {
  dfree(h, p.probs);
  dfree(h, p.tiles);
  p = DevPlan();
}

void drop_solve_graph(hodlr_t h) {
  if (h->sg_exec) cudaGraphExecDestroy(h->sg_exec);
  h->sg_exec = nullptr;
  h->sg_nrhs = -1;
}

void free_factor(hodlr_t h) {
  drop_solve_graph(h);
  ++h->factor_gen;
  for (auto& L : h->lv) {
    dfree(h, L.S);
    dfree(h, L.piv);
    dfree(h, L.d_nodes);
    dfree(h, L.d_snodes);
    free_plan(h, L.tn);
    free_plan(h, L.nn);
    free_plan(h, L.stn);
    free_plan(h, L.snn);
    L.solve_nrhs = -1;
    L.nodes.clear();
  }
  dfree(h, h->d_lu);
  dfree(h, h->d_lu_off);
  dfree(h, h->d_perm);
  for (auto& L : h->lv) {
    if (!L.y_alias) dfree(h, L.Yl);
    L.Yl = nullptr;
    L.y_alias = false;
  }
  if (h->w_consumed) h->compressed = false;  // the U panels are gone: compress again
  h->w_consumed = false;
  h->factored = false;
}

void free_compress(hodlr_t h) {
  free_factor(h);
  for (auto& L : h->lv) {
    dfree(h, L.W);
    dfree(h, L.V);
    dfree(h, L.cR);
    dfree(h, L.cC);
    dfree(h, L.prow);
    dfree(h, L.pcol);
    dfree(h, L.d_st);
    L.st.clear();
    L.kcap = 0;
  }
  h->compressed = false;
}

int ensure_ws(hodlr_t h, int64_t elems) {
  if (elems <= h->ws_cap) return HODLR_OK;
  dfree(h, h->ws);
  CK(dalloc(h, &h->ws, (size_t)elems));
  h->ws_cap = elems;
  return HODLR_OK;
}

// Host copies on the handle's stream.  The handle's own stream is a
// non-blocking stream, so a synchronous cudaMemcpy (legacy default stream) is
// not ordered with its kernels; every copy goes through these instead and
// returns after the stream has drained.
// Each of them drains the stream, after which the pinned staging memory of
// h2d_async is free again.
static cudaError_t drained(hodlr_t h, cudaError_t e) {
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) h->pin_used = 0;
  return e;
}
cudaError_t h2d(hodlr_t h, void* dst, const void* src, size_t bytes) {
  return drained(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
}
cudaError_t d2h(hodlr_t h, void* dst, const void* src, size_t bytes) {
  return drained(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
}

// A pageable cudaMemcpyAsync to the device synchronises the stream before it
// starts, so the host would wait for every queued kernel before planning the
// next launches.  These uploads go through pinned staging memory instead:
// the host copies the bytes there and queues the copy.  The staging area is
// reused once the stream has drained (any of the calls above), or here when
// it is full.
cudaError_t h2d_async(hodlr_t h, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return cudaSuccess;
  const size_t need = (bytes + 255) & ~(size_t)255;
  if (h->pin_used + need > h->pin_cap) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return e;
    h->pin_used = 0;
    if (need > h->pin_cap) {
      if (h->pin) cudaFreeHost(h->pin);
      h->pin = nullptr;
      h->pin_cap = 0;
      const size_t cap = std::max(need, (size_t)8 << 20);
      e = cudaMallocHost((void**)&h->pin, cap);
      if (e != cudaSuccess) {
        h->pin = nullptr;
        return e;
      }
      h->pin_cap = cap;
    }
  }
  char* p = h->pin + h->pin_used;
  memcpy(p, src, bytes);
  h->pin_used += need;
  return cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, h->stream);
}
cudaError_t copy2d(hodlr_t h, void* dst, size_t dpitch, const void* src, size_t spitch,
                   size_t width, size_t rows, cudaMemcpyKind kind) {
  return drained(h, cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, h->stream));
}

int check_dev_err(hodlr_t h, const char* where) {
  unsigned e = 0;
  CK(d2h(h, &e, h->d_err, sizeof(unsigned)));
  if (e == 0) return HODLR_OK;
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), h->stream));
  if (e & DEV_ERR_TIMEOUT) return fail(h, HODLR_ERR_TIMEOUT, std::string(where) + ": device wait timed out");
  if (e & DEV_ERR_NONFINITE) return fail(h, HODLR_ERR_NONFINITE, std::string(where) + ": non-finite value");
  if (e & DEV_ERR_SINGULAR) return fail(h, HODLR_ERR_SINGULAR, std::string(where) + ": exact-zero pivot");
  if (e & DEV_ERR_INDEX) {
    std::string at;
    if (e & DEV_ERR_AT_LEAF_PERM) at += " [leaf permutation]";
    if (e & DEV_ERR_AT_SOLVE_PIV) at += " [capacitance solve pivots]";
    if (e & DEV_ERR_AT_BLOCKED_PIV) at += " [blocked solve pivots]";
    if (e & DEV_ERR_AT_LU_SWAP) at += " [multi-CTA LU interchanges]";
    return fail(h, HODLR_ERR_CHECK, std::string(where) + ": pivot or permutation index out of range" + at);
  }
  return fail(h, HODLR_ERR_CUDA, where);
}

int check_phase(hodlr_t h, const char* where) {
  if (!h->checked) return HODLR_OK;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, where);
  return check_dev_err(h, where);
}

int check_extent(hodlr_t h, const void* p, size_t bytes, const char* what, const char* where) {
  if (!h->checked || bytes == 0 || h->pool.holds(p, bytes)) return HODLR_OK;
  char msg[256];
  snprintf(msg, sizeof msg, "%s: %s [%p, +%zu bytes) is outside the handle's allocations", where,
           what, p, bytes);
  return fail(h, HODLR_ERR_CHECK, msg);
}

int check_gemm(hodlr_t h, const std::vector<GemmProblem>& probs, bool tn, const char* where) {
  if (!h->checked) return HODLR_OK;
  const size_t e = sizeof(double);
  for (const auto& p : probs) {
    if (p.M <= 0 || p.N <= 0 || p.K <= 0) continue;
    // A: K x M (tn) or M x K, B: K x N, C: M x N, all column-major
    const size_t a = tn ? (size_t)(p.M - 1) * p.lda + p.K : (size_t)(p.K - 1) * p.lda + p.M;
    int rc = check_extent(h, p.A, a * e, "GEMM operand A", where);
    if (!rc) rc = check_extent(h, p.B, ((size_t)(p.N - 1) * p.ldb + p.K) * e, "GEMM operand B", where);
    if (!rc) rc = check_extent(h, p.C, ((size_t)(p.N - 1) * p.ldc + p.M) * e, "GEMM result C", where);
    if (!rc && p.splits > 1)
      rc = check_extent(h, h->ws + p.ws_off, (size_t)p.splits * p.M * p.N * e, "split-K slice",
                        where);
    if (rc) return rc;
  }
  return HODLR_OK;
}

EntrySrc make_src(hodlr_t h) {
  EntrySrc s;
  s.pts = h->d_pts;
  s.A = h->d_A;
  s.ld = h->n;
  s.kp = h->kp;
  s.dense = h->dense ? 1 : 0;
  s.kps = h->nsys ? h->d_kps : nullptr;
  s.psys = h->nsys ? h->d_psys : nullptr;
  return s;
}

int init_common(hodlr_t h) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev));
  int coop = 0;
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return fail(h, HODLR_ERR_UNSUPPORTED, "device lacks cooperative launch");
  const char* chk = getenv("HODLR_CHECKED");
  h->checked = chk && *chk && strcmp(chk, "0") != 0;
  // HODLR_ACA_STREAMING=0|1|2: the ACA panel streaming mode of new handles
  // (hodlr_set_aca_streaming); unset or anything else keeps the default
  const char* acs = getenv("HODLR_ACA_STREAMING");
  if (acs && acs[0] >= '0' && acs[0] <= '2' && acs[1] == 0) {
    h->aca_ring = acs[0] != '0';
    h->aca_ring_tile = acs[0] == '2';
  }
  CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
  h->stream = h->own_stream;
  CK(cudaEventCreate(&h->ev0));
  CK(cudaEventCreate(&h->ev1));
  CK(dalloc(h, &h->d_err, 1));
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), h->stream));
  build_tree(h);
  const int nl = (int)h->leaf_min.size();
  if (h->smax > 160) return fail(h, HODLR_ERR_UNSUPPORTED, "leaf size above 160");
  CK(dalloc(h, &h->d_leaf_min, (size_t)nl));
  CK(dalloc(h, &h->d_leaf_size, (size_t)nl));
  CK(h2d(h, h->d_leaf_min, h->leaf_min.data(), 4 * nl));
  CK(h2d(h, h->d_leaf_size, h->leaf_size.data(), 4 * nl));
  return HODLR_OK;
}

}  // namespace hodlr_impl
