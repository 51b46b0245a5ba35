// extern "C" entry points of include/mpsb.h.
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"
#include "ozaki.cuh"

namespace mpsb {

static thread_local std::string g_last_error;
static int64_t g_serial = 0;

void set_last_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_last_error = buf;
}

void set_last_message(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

static int bind(mpsb_ctx* ctx) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  MPSB_CUDA_TRY(cudaSetDevice(ctx->device));
  return MPSB_OK;
}

static int sync(mpsb_ctx* ctx) {
  int* hw = reinterpret_cast<int*>(ctx->h_scalars + 63);
  MPSB_CUDA_TRY(cudaMemcpyAsync(hw, ctx->err(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MPSB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (*hw != 0) {
    const int word = *hw;
    *hw = 0;
    cudaMemsetAsync(ctx->err(), 0, sizeof(int), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    set_last_message("a device-side wait timed out (%s); results of this stream are invalid",
                     (word & 4) ? "wait self-test" : (word & 2) ? "sliced GEMM pipeline" : "QR cluster exchange");
    return MPSB_ERR_CUDA;
  }
  return MPSB_OK;
}

static int dev_alloc(cd** p, int64_t elems) {
  *p = nullptr;
  if (elems <= 0) elems = 1;
  cudaError_t e = cudaMalloc((void**)p, (size_t)elems * sizeof(cd));
  if (e != cudaSuccess) {
    set_last_error(e, "cudaMalloc", __FILE__, __LINE__);
    return MPSB_ERR_OUT_OF_MEMORY;
  }
  return MPSB_OK;
}

// Stream-ordered: later work on the context stream sees the data.  From pageable memory the
// copy has left the host buffer when this returns; from pinned (page-locked) memory it has not,
// and the buffer must stay unchanged until the stream passes the copy (mpsb_sync).
static int upload(mpsb_ctx* ctx, cd* dst, const double* host, int64_t elems) {
  MPSB_CUDA_TRY(cudaMemcpyAsync(dst, host, (size_t)elems * sizeof(cd), cudaMemcpyHostToDevice, ctx->stream));
  return MPSB_OK;
}

// the same, waiting for the copy (small operator buffers the caller may reuse at once)
static int upload_wait(mpsb_ctx* ctx, cd* dst, const double* host, int64_t elems) {
  MPSB_TRY(upload(ctx, dst, host, elems));
  return sync(ctx);
}

static int download(mpsb_ctx* ctx, double* host, const cd* src, int64_t elems) {
  MPSB_CUDA_TRY(cudaMemcpyAsync(host, src, (size_t)elems * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

// <A|B> family: left env sweep with 2-index envs (scal_prod / scal_prod_no_conj)
static int scal_prod_impl(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mps* B, bool conj, double* out) {
  if (!A || !B || !out) return MPSB_ERR_INVALID_ARG;
  if (A->na != B->na || A->d != B->d) return MPSB_ERR_DIMENSION;
  const int na = A->na, d = A->d;
  int64_t maxE = 1, maxAL = 1;
  for (int k = 0; k <= na; ++k) maxE = std::max<int64_t>(maxE, A->dims[k] * B->dims[k]);
  for (int k = 0; k < na; ++k) maxAL = std::max<int64_t>(maxAL, A->dims[k] * d * B->dims[k + 1]);
  cd *e0, *e1, *al;
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV0, maxE * sizeof(cd), &e0));
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV1, maxE * sizeof(cd), &e1));
  MPSB_TRY(ensure_slot(ctx, SLOT_MISC, maxAL * sizeof(cd), &al));
  count_launch(&ctx->ws);
  MPSB_TRY(set_value(e0, cmk(1.0, 0.0), ctx->stream));
  cd* cur = e0;
  cd* nxt = e1;
  for (int k = 0; k < na; ++k) {
    int a0 = (int)A->dims[k], a1 = (int)A->dims[k + 1], b0 = (int)B->dims[k], b1 = (int)B->dims[k + 1];
    MPSB_TRY(op_L2_A3(ctx, cur, B->site(k), al, a0, b0, d * b1, cmk(1, 0), cmk(0, 0), false));
    MPSB_TRY(op_update_lenv(ctx, A->site(k), al, nxt, a0 * d, a1, b1, conj));
    std::swap(cur, nxt);
  }
  MPSB_CUDA_TRY(cudaMemcpyAsync(out, cur, sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

}  // namespace mpsb

using namespace mpsb;

extern "C" {

const char* mpsb_last_error(void) { return g_last_error.c_str(); }
int mpsb_version(void) { return 1; }

int mpsb_ctx_create(int device, mpsb_ctx** out) {
  if (!out) return MPSB_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || device < 0 || device >= n) {
    set_last_message("no CUDA device %d (%s)", device, e == cudaSuccess ? "out of range" : cudaGetErrorString(e));
    return MPSB_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  MPSB_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_last_message("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
    return MPSB_ERR_NO_DEVICE;
  }
  MPSB_CUDA_TRY(cudaSetDevice(device));
  mpsb_ctx* c = new mpsb_ctx();
  c->device = device;
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; set_last_error(e, "cudaStreamCreate", __FILE__, __LINE__); return MPSB_ERR_CUDA; }
  c->stream = c->own_stream;
  e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaStreamDestroy(c->own_stream);
    delete c;
    set_last_error(e, "cudaStreamCreate", __FILE__, __LINE__);
    return MPSB_ERR_CUDA;
  }
  if (const char* pe = getenv("MPSB_PIPELINE")) c->pipeline = atoi(pe) != 0;
  if (cudaMalloc((void**)&c->d_scalars, 64 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void**)&c->h_scalars, 64 * sizeof(double)) != cudaSuccess) {
    cudaStreamDestroy(c->own_stream);
    delete c;
    set_last_message("allocation of context scalars failed");
    return MPSB_ERR_OUT_OF_MEMORY;
  }
  cudaMemset(c->d_scalars, 0, 64 * sizeof(double));
  c->h_scalars[63] = 0.0;
  *out = c;
  return MPSB_OK;
}

int mpsb_ctx_destroy(mpsb_ctx* ctx) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->graphs_cache)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  cudaStreamSynchronize(ctx->side);
  for (auto& p : ctx->prof_events) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  ws_free(ctx->ws);
  ws_free(ctx->ws_side);
  if (ctx->vec.p) cudaFree(ctx->vec.p);
  for (cudaEvent_t ev : ctx->events) cudaEventDestroy(ev);
  cudaFree(ctx->d_scalars);
  cudaFreeHost(ctx->h_scalars);
  cudaStreamDestroy(ctx->side);
  cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return MPSB_OK;
}

int mpsb_sync(mpsb_ctx* ctx) {
  MPSB_TRY(bind(ctx));
  return sync(ctx);
}

int mpsb_ctx_set_stream(mpsb_ctx* ctx, void* stream) {
  MPSB_TRY(bind(ctx));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  for (auto& kv : ctx->graphs_cache)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs_cache.clear();
  return MPSB_OK;
}

int mpsb_ctx_set_graphs(mpsb_ctx* ctx, int enable) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  ctx->graphs = enable != 0;
  return MPSB_OK;
}

int mpsb_ctx_launch_count(mpsb_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return MPSB_ERR_INVALID_ARG;
  *out = ctx->ws.launches + ctx->ws_side.launches;
  return MPSB_OK;
}

int mpsb_ctx_set_profiling(mpsb_ctx* ctx, int enable) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  ctx->ws.prof = enable ? &ctx->prof_events : nullptr;
  ctx->ws_side.prof = ctx->ws.prof;
  return MPSB_OK;
}

int mpsb_ctx_profile_read(mpsb_ctx* ctx, double* ms, int64_t* launches, double* ops) {
  MPSB_TRY(bind(ctx));
  if (!ms || !launches) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(sync(ctx));
  MPSB_CUDA_TRY(cudaStreamSynchronize(ctx->side));
  double tot = 0.0, nops = 0.0;
  for (auto& p : ctx->prof_events) {
    float t = 0.f;
    MPSB_CUDA_TRY(cudaEventElapsedTime(&t, p.start, p.stop));
    tot += t;
    nops += p.ops;
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  *ms = tot;
  if (ops) *ops = nops;
  *launches = (int64_t)ctx->prof_events.size();
  ctx->prof_events.clear();
  return MPSB_OK;
}

int mpsb_wait_selftest(mpsb_ctx* ctx, double seconds) {
  MPSB_TRY(bind(ctx));
  count_launch(&ctx->ws);
  MPSB_TRY(wait_probe_launch(seconds, ctx->err(), ctx->stream));
  return sync(ctx);
}

int mpsb_ctx_set_precision(mpsb_ctx* ctx, int slices, int min_tiles) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  if (slices != 0 && (slices < OZ_MIN_SLICES || slices > OZ_MAX_SLICES)) {
    set_last_message("precision: slices must be 0 (FP64) or %d..%d", OZ_MIN_SLICES, OZ_MAX_SLICES);
    return MPSB_ERR_INVALID_ARG;
  }
  if (min_tiles < 1) return MPSB_ERR_INVALID_ARG;
  ctx->split_slices = slices;
  ctx->split_min_tiles = min_tiles;
  return MPSB_OK;
}

int mpsb_ctx_set_batched_split_threshold(mpsb_ctx* ctx, double min_flops) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  if (!(min_flops >= 0.0) || min_flops > 9.0e18) {
    set_last_message("batched split threshold must be a flop count in [0, 9e18]");
    return MPSB_ERR_INVALID_ARG;
  }
  ctx->split_min_flops = min_flops;
  return MPSB_OK;
}

int mpsb_ctx_set_pipeline(mpsb_ctx* ctx, int enable) {
  if (!ctx) return MPSB_ERR_INVALID_ARG;
  ctx->pipeline = enable != 0;
  return MPSB_OK;
}

// ---------------------------------------------------------------- MPS
static void register_slab(mpsb_ctx* ctx, const void* base, int64_t total, int batch) {
  const uintptr_t b = reinterpret_cast<uintptr_t>(base);
  ctx->slabs[b] = {b + (uintptr_t)(total * batch) * sizeof(cd), total};
}

static int mps_create(mpsb_ctx* ctx, int na, int d, const int64_t* dims, int batch, bool batched, mpsb_mps** out) {
  MPSB_TRY(bind(ctx));
  if (!out || !dims || na < 1 || d < 1 || batch < 1 || batch > 65535) return MPSB_ERR_INVALID_ARG;
  if (dims[0] != 1 || dims[na] != 1) return MPSB_ERR_DIMENSION;
  mpsb_mps* A = new mpsb_mps();
  A->ctx = ctx; A->serial = ++g_serial; A->na = na; A->d = d;
  A->batch = batch; A->batched = batched;
  A->dims.assign(dims, dims + na + 1);
  int64_t tot = 0;
  for (int k = 0; k < na; ++k) {
    if (dims[k] < 1) { delete A; return MPSB_ERR_DIMENSION; }
    A->off.push_back(tot);
    tot += dims[k] * d * dims[k + 1];
  }
  A->total = tot;
  int st = dev_alloc(&A->slab, tot * batch);
  if (st != MPSB_OK) { delete A; return st; }
  cudaMemsetAsync(A->slab, 0, tot * batch * sizeof(cd), ctx->stream);
  if (batched) register_slab(ctx, A->slab, tot, batch);
  *out = A;
  return MPSB_OK;
}

int mpsb_mps_create(mpsb_ctx* ctx, int na, int d, const int64_t* dims, mpsb_mps** out) {
  return mps_create(ctx, na, d, dims, 1, false, out);
}

int mpsb_mps_create_batch(mpsb_ctx* ctx, int na, int d, const int64_t* dims, int batch, mpsb_mps** out) {
  return mps_create(ctx, na, d, dims, batch, true, out);
}

int mpsb_mps_view(mpsb_mps* A, int copy, mpsb_mps** out) {
  if (!A || !out || copy < 0 || copy >= A->batch) return MPSB_ERR_INVALID_ARG;
  mpsb_mps* V = new mpsb_mps(*A);
  V->serial = ++g_serial;
  V->batch = 1;
  V->owns = false;
  V->slab = A->slab + (int64_t)copy * A->total;
  *out = V;
  return MPSB_OK;
}

int mpsb_mps_destroy(mpsb_mps* A) {
  if (!A) return MPSB_ERR_INVALID_ARG;
  cudaSetDevice(A->ctx->device);
  cudaStreamSynchronize(A->ctx->stream);
  if (A->owns) {
    A->ctx->slabs.erase(reinterpret_cast<uintptr_t>(A->slab));
    cudaFree(A->slab);
  }
  delete A;
  return MPSB_OK;
}

int mpsb_mps_batch(const mpsb_mps* A, int* batch) {
  if (!A || !batch) return MPSB_ERR_INVALID_ARG;
  *batch = A->batch;
  return MPSB_OK;
}

int mpsb_mps_set_site_copy(mpsb_mps* A, int copy, int site, const double* host) {
  if (!A || !host || site < 1 || site > A->na || copy < 0 || copy >= A->batch) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(A->ctx));
  return upload(A->ctx, A->site(site - 1) + (int64_t)copy * A->total, host, A->site_elems(site - 1));
}

int mpsb_mps_get_site_copy(const mpsb_mps* A, int copy, int site, double* host) {
  if (!A || !host || site < 1 || site > A->na || copy < 0 || copy >= A->batch) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(A->ctx));
  return download(A->ctx, host, A->site(site - 1) + (int64_t)copy * A->total, A->site_elems(site - 1));
}

int mpsb_mps_select(mpsb_mps* dst, mpsb_mps* const* srcs, int nsrc, const int* which) {
  if (!dst || !srcs || !which || nsrc < 1) return MPSB_ERR_INVALID_ARG;
  for (int i = 0; i < nsrc; ++i) {
    if (!srcs[i]) return MPSB_ERR_INVALID_ARG;
    if (srcs[i]->dims != dst->dims || srcs[i]->d != dst->d || srcs[i]->batch != dst->batch) return MPSB_ERR_DIMENSION;
  }
  MPSB_TRY(bind(dst->ctx));
  const int B = dst->batch;
  for (int b = 0; b < B;) {
    const int w = which[b];
    if (w >= nsrc) return MPSB_ERR_INVALID_ARG;
    int e = b + 1;
    while (e < B && which[e] == w) ++e;   // one copy per run of equal sources
    if (w >= 0 && srcs[w] != dst)
      MPSB_CUDA_TRY(cudaMemcpyAsync(dst->slab + (int64_t)b * dst->total, srcs[w]->slab + (int64_t)b * dst->total,
                                    (size_t)(e - b) * dst->total * sizeof(cd), cudaMemcpyDeviceToDevice,
                                    dst->ctx->stream));
    b = e;
  }
  return MPSB_OK;
}

int mpsb_mps_info(const mpsb_mps* A, int* na, int* d, int64_t* dims) {
  if (!A) return MPSB_ERR_INVALID_ARG;
  if (na) *na = A->na;
  if (d) *d = A->d;
  if (dims) for (int k = 0; k <= A->na; ++k) dims[k] = A->dims[k];
  return MPSB_OK;
}

int mpsb_mps_set_site(mpsb_mps* A, int site, const double* host) {
  if (!A || !host || site < 1 || site > A->na) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(A->ctx));
  return upload(A->ctx, A->site(site - 1), host, A->site_elems(site - 1));
}

int mpsb_mps_get_site(const mpsb_mps* A, int site, double* host) {
  if (!A || !host || site < 1 || site > A->na) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(A->ctx));
  return download(A->ctx, host, A->site(site - 1), A->site_elems(site - 1));
}

int mpsb_mps_site_ptr(const mpsb_mps* A, int site, void** dptr) {
  if (!A || !dptr || site < 1 || site > A->na) return MPSB_ERR_INVALID_ARG;
  *dptr = A->site(site - 1);
  return MPSB_OK;
}

int mpsb_mps_copy(mpsb_mps* dst, const mpsb_mps* src) {
  if (!dst || !src) return MPSB_ERR_INVALID_ARG;
  if (dst->na != src->na || dst->d != src->d || dst->dims != src->dims || dst->batch != src->batch)
    return MPSB_ERR_DIMENSION;
  MPSB_TRY(bind(dst->ctx));
  MPSB_CUDA_TRY(cudaMemcpyAsync(dst->slab, src->slab, src->total * src->batch * sizeof(cd), cudaMemcpyDeviceToDevice,
                                dst->ctx->stream));
  return MPSB_OK;
}

// ---------------------------------------------------------------- MPO
int mpsb_mpo_create(mpsb_ctx* ctx, int na, int d, const int64_t* w, mpsb_mpo** out) {
  MPSB_TRY(bind(ctx));
  if (!out || !w || na < 1 || d < 1) return MPSB_ERR_INVALID_ARG;
  if (w[0] != 1 || w[na] != 1) return MPSB_ERR_DIMENSION;
  mpsb_mpo* O = new mpsb_mpo();
  O->ctx = ctx; O->serial = ++g_serial; O->na = na; O->d = d;
  O->w.assign(w, w + na + 1);
  int64_t tot = 0;
  for (int k = 0; k < na; ++k) {
    if (w[k] < 1) { delete O; return MPSB_ERR_DIMENSION; }
    O->off.push_back(tot);
    tot += w[k] * d * w[k + 1] * d;
  }
  O->total = tot;
  int st = dev_alloc(&O->slab, tot);
  if (st != MPSB_OK) { delete O; return st; }
  cudaMemsetAsync(O->slab, 0, tot * sizeof(cd), ctx->stream);
  *out = O;
  return MPSB_OK;
}

int mpsb_mpo_destroy(mpsb_mpo* O) {
  if (!O) return MPSB_ERR_INVALID_ARG;
  cudaSetDevice(O->ctx->device);
  cudaStreamSynchronize(O->ctx->stream);
  cudaFree(O->slab);
  delete O;
  return MPSB_OK;
}

int mpsb_mpo_set_site(mpsb_mpo* O, int site, const double* host) {
  if (!O || !host || site < 1 || site > O->na) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(O->ctx));
  return upload(O->ctx, O->site(site - 1), host, O->site_elems(site - 1));
}

int mpsb_mpo_get_site(const mpsb_mpo* O, int site, double* host) {
  if (!O || !host || site < 1 || site > O->na) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(O->ctx));
  return download(O->ctx, host, O->site(site - 1), O->site_elems(site - 1));
}

// ---------------------------------------------------------------- environments
static int env_create(mpsb_ctx* ctx, int na, const int64_t* dims1, const int64_t* dims2, const int64_t* w, int batch,
                      bool batched, mpsb_env** out) {
  MPSB_TRY(bind(ctx));
  if (!out || !dims1 || !dims2 || na < 1 || batch < 1 || batch > 65535) return MPSB_ERR_INVALID_ARG;
  mpsb_env* E = new mpsb_env();
  E->ctx = ctx; E->serial = ++g_serial; E->na = na; E->three = (w != nullptr);
  E->batch = batch; E->batched = batched;
  int64_t tot = 0;
  for (int e = 0; e <= na; ++e) {
    bool end = (e == 0 || e == na);
    E->d1.push_back(end ? 1 : dims1[e]);
    E->d2.push_back(end ? 1 : dims2[e]);
    E->w.push_back(end ? 1 : (w ? w[e] : 1));
    E->off.push_back(tot);
    tot += E->d1.back() * E->w.back() * E->d2.back();
  }
  E->total = tot;
  int st = dev_alloc(&E->slab, tot * batch);
  if (st != MPSB_OK) { delete E; return st; }
  cudaMemsetAsync(E->slab, 0, tot * batch * sizeof(cd), ctx->stream);
  count_launch(&ctx->ws);
  set_value_strided(E->entry(0), tot, batch, cmk(1.0, 0.0), ctx->stream);
  count_launch(&ctx->ws);
  set_value_strided(E->entry(na), tot, batch, cmk(1.0, 0.0), ctx->stream);
  MPSB_CUDA_TRY(cudaGetLastError());
  if (batched) register_slab(ctx, E->slab, tot, batch);
  *out = E;
  return MPSB_OK;
}

int mpsb_env_create(mpsb_ctx* ctx, int na, const int64_t* dims1, const int64_t* dims2, const int64_t* w,
                    mpsb_env** out) {
  return env_create(ctx, na, dims1, dims2, w, 1, false, out);
}

int mpsb_env_create_batch(mpsb_ctx* ctx, int na, const int64_t* dims1, const int64_t* dims2, const int64_t* w,
                          int batch, mpsb_env** out) {
  return env_create(ctx, na, dims1, dims2, w, batch, true, out);
}

int mpsb_env_destroy(mpsb_env* E) {
  if (!E) return MPSB_ERR_INVALID_ARG;
  cudaSetDevice(E->ctx->device);
  cudaStreamSynchronize(E->ctx->stream);
  E->ctx->slabs.erase(reinterpret_cast<uintptr_t>(E->slab));
  cudaFree(E->slab);
  delete E;
  return MPSB_OK;
}

int mpsb_env_get(const mpsb_env* E, int entry, double* host) {
  if (!E || !host || entry < 1 || entry > E->na + 1) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(E->ctx));
  return download(E->ctx, host, E->entry(entry - 1), E->entry_elems(entry - 1));
}

int mpsb_env_set(mpsb_env* E, int entry, const double* host) {
  if (!E || !host || entry < 1 || entry > E->na + 1) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(bind(E->ctx));
  return upload(E->ctx, E->entry(entry - 1), host, E->entry_elems(entry - 1));
}

// ---------------------------------------------------------------- hot path
int mpsb_rk4stp_apply_H_half(mpsb_ctx* ctx, double dt, const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3,
                             mpsb_mps* psi0, mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2, mpsb_mps* psi3,
                             mpsb_env* env1, mpsb_env* env2, mpsb_env* env3, mpsb_env* envop) {
  MPSB_TRY(bind(ctx));
  return rk4_step(ctx, dt, H1, H2, H3, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop);
}

int mpsb_compress_var_apply_H_left(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain,
                                   const mpsb_mps* A, const mpsb_mpo* H) {
  MPSB_TRY(bind(ctx));
  return compress_var_apply_H_left(ctx, A0, envop, Ain, A, H);
}

static int sum_var(mpsb_ctx* ctx, bool right, mpsb_mps* A0, mpsb_env* const* env, mpsb_env* envop,
                   const mpsb_mps* Ain, const double* coef, int numv, mpsb_mps* const* A, const mpsb_mpo* H) {
  MPSB_TRY(bind(ctx));
  if (!coef || !A || numv < 1 || numv > 9) return MPSB_ERR_INVALID_ARG;
  std::vector<cd> c(numv);
  std::vector<const mpsb_mps*> t(numv);
  for (int i = 0; i < numv; ++i) {
    c[i] = cmk(coef[2 * i], coef[2 * i + 1]);
    t[i] = A[i];
  }
  return compress_sum_var_apply_H(ctx, right, A0, env, envop, Ain, c.data(), numv, t.data(), H);
}

int mpsb_compress_sum_var_apply_H_right(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* const* env, mpsb_env* envop,
                                        const mpsb_mps* Ain, const double* coef, int numv, mpsb_mps* const* A,
                                        const mpsb_mpo* H) {
  return sum_var(ctx, true, A0, env, envop, Ain, coef, numv, A, H);
}

int mpsb_compress_sum_var_apply_H_left(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* const* env, mpsb_env* envop,
                                       const mpsb_mps* Ain, const double* coef, int numv, mpsb_mps* const* A,
                                       const mpsb_mpo* H) {
  return sum_var(ctx, false, A0, env, envop, Ain, coef, numv, A, H);
}

int mpsb_compress_var_apply_H(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain, const mpsb_mps* A,
                              const mpsb_mpo* H, int maxsweeps) {
  MPSB_TRY(bind(ctx));
  return compress_var_apply_H(ctx, A0, envop, Ain, A, H, maxsweeps);
}

static int full_sum_var(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const double* coef, int numv,
                        mpsb_mps* const* A, const mpsb_mpo* H, int maxsweeps) {
  if (!coef || !A || numv < 1 || numv > 9) return MPSB_ERR_INVALID_ARG;
  std::vector<cd> c(numv);
  std::vector<const mpsb_mps*> t(numv);
  for (int i = 0; i < numv; ++i) {
    c[i] = cmk(coef[2 * i], coef[2 * i + 1]);
    t[i] = A[i];
  }
  return compress_sum_var_full(ctx, A0, envop, c.data(), numv, t.data(), H, maxsweeps);
}

int mpsb_compress_sum_var_apply_H(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const double* coef, int numv,
                                  mpsb_mps* const* A, const mpsb_mpo* H, int maxsweeps) {
  MPSB_TRY(bind(ctx));
  if (!H) return MPSB_ERR_INVALID_ARG;
  return full_sum_var(ctx, A0, envop, coef, numv, A, H, maxsweeps);
}

int mpsb_compress_sum_var(mpsb_ctx* ctx, mpsb_mps* A0, const mpsb_mps* Ain, const double* coef, int numv,
                          mpsb_mps* const* A, int maxsweeps) {
  MPSB_TRY(bind(ctx));
  if (!A0 || !Ain) return MPSB_ERR_INVALID_ARG;
  if (A0 != Ain) MPSB_TRY(mpsb_mps_copy(A0, Ain));   // the guess
  return full_sum_var(ctx, A0, nullptr, coef, numv, A, nullptr, maxsweeps);
}

int mpsb_ground_state_search(mpsb_ctx* ctx, mpsb_mps* At, const mpsb_mpo* H, int maxsweeps, double converge_rat,
                             double eigs_tol, double* ae) {
  MPSB_TRY(bind(ctx));
  double e = 0.0;
  MPSB_TRY(ground_state_search(ctx, At, H, maxsweeps, converge_rat, eigs_tol, &e));
  MPSB_TRY(sync(ctx));
  if (ae) *ae = e;
  return MPSB_OK;
}

// ---------------------------------------------------------------- gauge / norms
int mpsb_norm_lo(mpsb_ctx* ctx, const mpsb_mps* A, double* no) {
  MPSB_TRY(bind(ctx));
  if (!A || !no) return MPSB_ERR_INVALID_ARG;
  count_launch(&ctx->ws);
  MPSB_TRY(norm2(A->site(A->na - 1), A->site_elems(A->na - 1), ctx->d_scalars, ctx->stream));
  MPSB_CUDA_TRY(cudaMemcpyAsync(no, ctx->d_scalars, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MPSB_TRY(sync(ctx));
  if (!(*no == *no) || *no > 1e300) return MPSB_ERR_NONFINITE;
  return MPSB_OK;
}

int mpsb_normalize_lo_batch(mpsb_ctx* ctx, mpsb_mps* A, double* no) {
  MPSB_TRY(bind(ctx));
  if (!A || !no) return MPSB_ERR_INVALID_ARG;
  const int s = A->na - 1, B = A->batch;
  MPSB_TRY(devbuf_ensure(nullptr, ctx->vec, (size_t)B * sizeof(double)));
  double* dn = static_cast<double*>(ctx->vec.p);
  count_launch(&ctx->ws);
  MPSB_TRY(norm2_batched(A->site(s), A->site_elems(s), A->total, B, dn, ctx->stream));
  count_launch(&ctx->ws);
  MPSB_TRY(scale_by_rsqrt_batched(A->site(s), A->site_elems(s), A->total, B, dn, ctx->stream));
  MPSB_CUDA_TRY(cudaMemcpyAsync(no, dn, (size_t)B * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MPSB_TRY(sync(ctx));
  for (int b = 0; b < B; ++b)
    if (!(no[b] == no[b]) || no[b] > 1e300) return MPSB_ERR_NONFINITE;
  return MPSB_OK;
}

int mpsb_normalize_lo(mpsb_ctx* ctx, mpsb_mps* A, double* no) {
  MPSB_TRY(bind(ctx));
  if (!A) return MPSB_ERR_INVALID_ARG;
  const int s = A->na - 1;
  count_launch(&ctx->ws);
  MPSB_TRY(norm2(A->site(s), A->site_elems(s), ctx->d_scalars, ctx->stream));
  count_launch(&ctx->ws);
  MPSB_TRY(scale_by_rsqrt(A->site(s), A->site_elems(s), ctx->d_scalars, ctx->stream));
  double v = 0;
  MPSB_CUDA_TRY(cudaMemcpyAsync(&v, ctx->d_scalars, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MPSB_TRY(sync(ctx));
  if (no) *no = v;
  if (!(v == v) || v > 1e300) return MPSB_ERR_NONFINITE;
  return MPSB_OK;
}

int mpsb_leftorthogonalizeQR(mpsb_ctx* ctx, mpsb_mps* A, double* no) {
  MPSB_TRY(bind(ctx));
  if (!A) return MPSB_ERR_INVALID_ARG;
  const int na = A->na, d = A->d;
  int64_t maxR = 1, maxS = 1;
  for (int k = 0; k < na; ++k) {
    maxR = std::max<int64_t>(maxR, A->dims[k + 1] * A->dims[k + 1]);
    maxS = std::max<int64_t>(maxS, A->site_elems(k));
  }
  cd *R, *tmp;
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV0, maxR * sizeof(cd), &R));
  MPSB_TRY(ensure_slot(ctx, SLOT_MISC, maxS * sizeof(cd), &tmp));
  for (int k = 0; k < na - 1; ++k) {
    int Dl = (int)A->dims[k], Dr = (int)A->dims[k + 1], Dn = (int)A->dims[k + 2];
    MPSB_TRY(op_orth_left(ctx, A->site(k), Dl, d, Dr, R));
    MPSB_TRY(op_L2_A3(ctx, R, A->site(k + 1), tmp, Dr, Dr, d * Dn, cmk(1, 0), cmk(0, 0), false));
    count_launch(&ctx->ws);
    MPSB_TRY(copy(A->site(k + 1), tmp, A->site_elems(k + 1), ctx->stream));
  }
  return mpsb_norm_lo(ctx, A, no);
}

int mpsb_leftorthonormalizationQR(mpsb_ctx* ctx, mpsb_mps* A, double* no) {
  double tmp = 0;
  MPSB_TRY(mpsb_leftorthogonalizeQR(ctx, A, &tmp));
  return mpsb_normalize_lo(ctx, A, no);
}

int mpsb_apply_site_operator(mpsb_ctx* ctx, mpsb_mps* A, int site, const double* op) {
  MPSB_TRY(bind(ctx));
  if (!A || !op || site < 1 || site > A->na) return MPSB_ERR_INVALID_ARG;
  const int d = A->d, k = site - 1;
  cd* dop;
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV1, (size_t)d * d * sizeof(cd), &dop));
  MPSB_TRY(upload_wait(ctx, dop, op, (int64_t)d * d));
  MpoApply a;
  const int chiL = (int)A->dims[k], chiR = (int)A->dims[k + 1];
  a.X = chiL; a.Y = chiR; a.K1 = d; a.K2 = 1; a.M1 = d; a.M2 = 1;
  a.in = A->site(k); a.in_x = 1; a.in_k1 = chiL; a.in_k2 = 0; a.in_y = (int64_t)chiL * d;
  a.op = dop;
  a.out = A->site(k); a.out_x = 1; a.out_m1 = chiL; a.out_m2 = 0; a.out_y = (int64_t)chiL * d;
  count_launch(&ctx->ws);
  return mpo_apply_launch_strided(a, d, 0, 1, 0, ctx->stream);
}

// ---------------------------------------------------------------- observables
int mpsb_scal_prod(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mps* B, double* out) {
  MPSB_TRY(bind(ctx));
  return scal_prod_impl(ctx, A, B, true, out);
}

int mpsb_scal_prod_no_conj(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mps* B, double* out) {
  MPSB_TRY(bind(ctx));
  return scal_prod_impl(ctx, A, B, false, out);
}

int mpsb_scal_op_prod(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mpo* O, const mpsb_mps* B, double* out) {
  MPSB_TRY(bind(ctx));
  if (!A || !O || !B || !out) return MPSB_ERR_INVALID_ARG;
  if (A->na != B->na || A->na != O->na || A->d != B->d || A->d != O->d) return MPSB_ERR_DIMENSION;
  const int na = A->na, d = A->d;
  int64_t maxE = 1, maxAOL = 1, maxG = 1;
  for (int k = 0; k <= na; ++k) maxE = std::max<int64_t>(maxE, A->dims[k] * O->w[k] * B->dims[k]);
  for (int k = 0; k < na; ++k) {
    maxAOL = std::max<int64_t>(maxAOL, A->dims[k] * d * B->dims[k + 1] * O->w[k + 1]);
    maxG = std::max<int64_t>(maxG, O->w[k] * A->dims[k] * d * B->dims[k + 1]);
  }
  cd *e0, *e1, *aol;
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV0, maxE * sizeof(cd), &e0));
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV1, maxE * sizeof(cd), &e1));
  MPSB_TRY(ensure_slot(ctx, SLOT_MISC, maxAOL * sizeof(cd), &aol));
  count_launch(&ctx->ws);
  MPSB_TRY(set_value(e0, cmk(1.0, 0.0), ctx->stream));
  cd* cur = e0;
  cd* nxt = e1;
  for (int k = 0; k < na; ++k) {
    int a0 = (int)A->dims[k], a1 = (int)A->dims[k + 1], b0 = (int)B->dims[k], b1 = (int)B->dims[k + 1];
    int wl = (int)O->w[k], wr = (int)O->w[k + 1];
    MPSB_TRY(op_prod_AOL(ctx, B->site(k), O->site(k), cur, aol, b0, d, b1, wl, wr, a0));
    MPSB_TRY(op_update_le(ctx, A->site(k), aol, nxt, a0, d, b1, wr, a1));
    std::swap(cur, nxt);
  }
  MPSB_CUDA_TRY(cudaMemcpyAsync(out, cur, sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

int mpsb_measure_local(mpsb_ctx* ctx, const mpsb_mps* A, const double* op, double* out) {
  MPSB_TRY(bind(ctx));
  if (!A || !op || !out) return MPSB_ERR_INVALID_ARG;
  const int na = A->na, d = A->d;
  int64_t maxE = 1, maxS = 1;
  for (int k = 0; k <= na; ++k) maxE = std::max<int64_t>(maxE, A->dims[k] * A->dims[k]);
  for (int k = 0; k < na; ++k) maxS = std::max<int64_t>(maxS, A->site_elems(k));
  cd *e0, *e1, *aenv, *dop;
  // ENV0/ENV1 hold the envs, MISC the Aenv product; op and results share SLOT_T
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV0, maxE * sizeof(cd), &e0));
  MPSB_TRY(ensure_slot(ctx, SLOT_ENV1, maxE * sizeof(cd), &e1));
  MPSB_TRY(ensure_slot(ctx, SLOT_MISC, maxS * sizeof(cd), &aenv));
  MPSB_TRY(ensure_slot(ctx, SLOT_T, (size_t)(d * d + na) * sizeof(cd), &dop));
  cd* res = dop + d * d;
  MPSB_TRY(upload_wait(ctx, dop, op, (int64_t)d * d));
  count_launch(&ctx->ws);
  MPSB_TRY(set_value(e0, cmk(1.0, 0.0), ctx->stream));
  cd* cur = e0;
  cd* nxt = e1;
  for (int k = na - 1; k >= 0; --k) {
    int Dl = (int)A->dims[k], Dr = (int)A->dims[k + 1];
    MPSB_TRY(op_A3_R2(ctx, A->site(k), cur, aenv, Dl * d, Dr, Dr, cmk(1, 0), cmk(0, 0)));
    count_launch(&ctx->ws);
    MPSB_TRY(local_exp(aenv, A->site(k), dop, Dl, d, Dr, res + k, ctx->stream));
    MPSB_TRY(op_update_renv(ctx, A->site(k), aenv, nxt, Dl, Dl, d * Dr));
    std::swap(cur, nxt);
  }
  std::vector<cd> h(na);
  MPSB_CUDA_TRY(cudaMemcpyAsync(h.data(), res, na * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  MPSB_TRY(sync(ctx));
  for (int k = 0; k < na; ++k) out[k] = h[k].x;
  return MPSB_OK;
}

int mpsb_apply_mpo_to_mps(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mpo* O, mpsb_mps* out) {
  MPSB_TRY(bind(ctx));
  if (!A || !O || !out) return MPSB_ERR_INVALID_ARG;
  if (A->na != O->na || out->na != A->na || A->d != O->d || out->d != A->d) return MPSB_ERR_DIMENSION;
  const int na = A->na, d = A->d;
  for (int k = 0; k <= na; ++k)
    if (out->dims[k] != A->dims[k] * O->w[k]) return MPSB_ERR_DIMENSION;
  for (int k = 0; k < na; ++k) {
    const int dl = (int)A->dims[k], dr = (int)A->dims[k + 1], wl = (int)O->w[k], wr = (int)O->w[k + 1];
    MpoApply a;
    a.X = dl; a.Y = dr; a.K1 = d; a.K2 = 1; a.M1 = wl * d; a.M2 = wr;
    a.in = A->site(k); a.in_x = 1; a.in_k1 = dl; a.in_k2 = 0; a.in_y = (int64_t)dl * d;
    a.op = O->site(k);
    a.out = out->site(k); a.out_x = 1; a.out_m1 = dl; a.out_m2 = (int64_t)dl * wl * d * dr;
    a.out_y = (int64_t)dl * wl * d;
    count_launch(&ctx->ws);
    MPSB_TRY(mpo_apply_launch_strided(a, (int64_t)wl * d * wr, 0, 1, (int64_t)wl * d, ctx->stream));
  }
  return MPSB_OK;
}

// ---------------------------------------------------------------- op level
#define DP(x) static_cast<const cd*>(x)
#define DW(x) static_cast<cd*>(x)

int mpsb_op_prod_AOR(mpsb_ctx* ctx, const void* A, const void* O, const void* R, void* AOR, int chiL, int d, int chiR,
                     int wL, int wR, int chiR0) {
  MPSB_TRY(bind(ctx));
  return op_prod_AOR(ctx, DP(A), DP(O), DP(R), DW(AOR), chiL, d, chiR, wL, wR, chiR0);
}

int mpsb_op_prod_AOL(mpsb_ctx* ctx, const void* A, const void* O, const void* L, void* AOL, int chiL, int d, int chiR,
                     int wL, int wR, int chiL0) {
  MPSB_TRY(bind(ctx));
  return op_prod_AOL(ctx, DP(A), DP(O), DP(L), DW(AOL), chiL, d, chiR, wL, wR, chiL0);
}

int mpsb_op_prod_LR_3_4(mpsb_ctx* ctx, const void* L, const void* AOR, void* A0, int chiL, int wL, int chiL0, int d,
                        int chiR0) {
  MPSB_TRY(bind(ctx));
  return op_prod_LR_3_4(ctx, DP(L), DP(AOR), DW(A0), chiL, wL, chiL0, d, chiR0, cmk(1, 0), cmk(0, 0));
}

int mpsb_op_prod_LR_4_3(mpsb_ctx* ctx, const void* AOL, const void* R, void* A0, int chiL0, int d, int chiR, int wR,
                        int chiR0) {
  MPSB_TRY(bind(ctx));
  return op_prod_LR_4_3(ctx, DP(AOL), DP(R), DW(A0), chiL0, d, chiR, wR, chiR0, cmk(1, 0), cmk(0, 0));
}

int mpsb_op_update_re(mpsb_ctx* ctx, const void* A0, const void* AOR, void* env, int chiL, int wL, int d, int chiR0,
                      int chiL0) {
  MPSB_TRY(bind(ctx));
  return op_update_re(ctx, DP(A0), DP(AOR), DW(env), chiL, wL, d, chiR0, chiL0);
}

int mpsb_op_update_le(mpsb_ctx* ctx, const void* A0, const void* AOL, void* env, int chiL0, int d, int chiR, int wR,
                      int chiR0) {
  MPSB_TRY(bind(ctx));
  return op_update_le(ctx, DP(A0), DP(AOL), DW(env), chiL0, d, chiR, wR, chiR0);
}

int mpsb_compression_svd(mpsb_ctx* ctx, const mpsb_mps* in, int dmax, double tol, mpsb_mps** out, double* err_glob,
                         double* err_trim, double* ent_ent) {
  MPSB_TRY(bind(ctx));
  if (!in || !out) return MPSB_ERR_INVALID_ARG;
  std::vector<int64_t> dims;
  cd* sites = nullptr;
  MPSB_TRY(compression_svd(ctx, in, dmax, tol, dims, &sites, err_glob, err_trim, ent_ent));
  mpsb_mps* A = nullptr;
  MPSB_TRY(mpsb_mps_create(ctx, in->na, in->d, dims.data(), &A));
  for (int k = 0; k < in->na; ++k)
    MPSB_CUDA_TRY(cudaMemcpyAsync(A->site(k), sites + in->off[k], A->site_elems(k) * sizeof(cd),
                                  cudaMemcpyDeviceToDevice, ctx->stream));
  *out = A;
  return sync(ctx);
}

int mpsb_compress_var_apply_H_two_site(mpsb_ctx* ctx, const mpsb_mps* Ain, const mpsb_mps* A, const mpsb_mpo* H,
                                       int maxsweeps, double svd_tol, int dlim, mpsb_mps** out) {
  MPSB_TRY(bind(ctx));
  if (!out) return MPSB_ERR_INVALID_ARG;
  std::vector<int64_t> dims, offs;
  cd* sites = nullptr;
  MPSB_TRY(compress_two_site(ctx, Ain, A, H, maxsweeps, svd_tol, dlim, dims, offs, &sites));
  mpsb_mps* R = nullptr;
  MPSB_TRY(mpsb_mps_create(ctx, A->na, A->d, dims.data(), &R));
  for (int k = 0; k < A->na; ++k)
    MPSB_CUDA_TRY(cudaMemcpyAsync(R->site(k), sites + offs[k], R->site_elems(k) * sizeof(cd), cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  *out = R;
  return sync(ctx);
}

int mpsb_compress_sum_var_apply_H_two_site(mpsb_ctx* ctx, const mpsb_mps* Ain, const double* coef, int numv,
                                           const mpsb_mps* const* A, const mpsb_mpo* H, int maxsweeps,
                                           double svd_tol, int dlim, int half, mpsb_mps** out) {
  MPSB_TRY(bind(ctx));
  if (!out || !coef || !A || numv < 1 || numv > 9) return MPSB_ERR_INVALID_ARG;
  std::vector<cd> c(numv);
  for (int l = 0; l < numv; ++l) c[l] = cmk(coef[2 * l], coef[2 * l + 1]);
  std::vector<int64_t> dims, offs;
  cd* sites = nullptr;
  MPSB_TRY(compress_two_site_sum(ctx, Ain, numv, c.data(), A, H, maxsweeps, svd_tol, dlim, half, dims, offs, &sites));
  const mpsb_mps* T = A[numv - 1];
  mpsb_mps* R = nullptr;
  MPSB_TRY(mpsb_mps_create(ctx, T->na, T->d, dims.data(), &R));
  for (int k = 0; k < T->na; ++k)
    MPSB_CUDA_TRY(cudaMemcpyAsync(R->site(k), sites + offs[k], R->site_elems(k) * sizeof(cd), cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  *out = R;
  return sync(ctx);
}

int mpsb_op_svd(mpsb_ctx* ctx, const void* X, void* U, double* S, void* V, int m, int n) {
  MPSB_TRY(bind(ctx));
  if (!X || !U || !S || !V || m < 1 || n < 1) return MPSB_ERR_DIMENSION;
  void* before = ctx->ws.svd.p;
  int st = svd_launch(m, n, DP(X), 1, m, DW(U), 1, m, S, DW(V), 1, n, &ctx->ws, ctx->stream);
  if (ctx->ws.svd.p != before) ctx->ws_generation++;
  MPSB_TRY(st);
  return sync(ctx);
}

int mpsb_op_zgemm(mpsb_ctx* ctx, int M, int N, int K, const void* A, int64_t a_m, int64_t a_k, int conjA,
                  const void* B, int64_t b_k, int64_t b_n, int conjB, void* C, int64_t c_m, int64_t c_n,
                  const double* alpha, const double* beta, int slices) {
  MPSB_TRY(bind(ctx));
  if (!A || !B || !C || M < 1 || N < 1 || K < 0) return MPSB_ERR_DIMENSION;
  Gemm g;
  g.M = M; g.N = N; g.K = K;
  g.A = DP(A); g.a_m = a_m; g.a_k = a_k; g.conjA = conjA != 0;
  g.B = DP(B); g.b_k = b_k; g.b_n = b_n; g.conjB = conjB != 0;
  g.C = DW(C); g.c_m = c_m; g.c_n = c_n;
  if (alpha) g.alpha = cmk(alpha[0], alpha[1]);
  if (beta) g.beta = cmk(beta[0], beta[1]);
  if (slices == 0) return run_gemm(ctx, g);
  if (!ozgemm_supported(g, slices)) {
    set_last_message("zgemm: %d slices unsupported for M=%d N=%d K=%d", slices, M, N, K);
    return MPSB_ERR_UNSUPPORTED;
  }
  void* before = ctx->ws.oz.p;
  MPSB_TRY(devbuf_ensure(&ctx->ws, ctx->ws.oz, ozgemm_scratch_bytes(g, slices)));
  if (ctx->ws.oz.p != before) ctx->ws_generation++;
  return ozgemm_launch(g, slices, ctx->ws.oz.p, ctx->ws.oz.cap, ctx->err(), &ctx->ws, ctx->stream);
}

int mpsb_op_qr(mpsb_ctx* ctx, const void* X, void* Q, void* R, int m, int n) {
  MPSB_TRY(bind(ctx));
  if (!X || !Q || m < n || n < 1) return MPSB_ERR_DIMENSION;
  QrProblem p;
  p.m = m; p.n = n;
  p.X = DP(X); p.x_r = 1; p.x_c = m;
  p.Q = DW(Q); p.q_r = 1; p.q_c = m;
  if (R) { p.R = DW(R); p.r_r = 1; p.r_c = n; }
  p.err = ctx->err();
  return run_qr(ctx, p);
}

}  // extern "C"
