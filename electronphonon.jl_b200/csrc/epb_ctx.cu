// Context, workspace and error plumbing of the C ABI.
#include <cstdarg>
#include <cstring>

#include "epb_common.cuh"

namespace epb {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

void clear_error() { g_err[0] = 0; }

int make_current(epb_ctx* ctx) {
  int cur = -1;
  EPB_CUDA(cudaGetDevice(&cur));
  if (cur != ctx->device) EPB_CUDA(cudaSetDevice(ctx->device));
  return EPB_OK;
}

int ws_get(epb_ctx* ctx, int slot, size_t bytes, void** out) {
  if (bytes == 0) bytes = 256;
  if (ctx->ws_bytes[slot] >= bytes) {
    *out = ctx->ws[slot];
    return EPB_OK;
  }
  if (ctx->fail_alloc_nth > 0 && --ctx->fail_alloc_nth == 0) {
    set_error("workspace allocation of %zu bytes failed (injected by epb_debug_fail_alloc)", bytes);
    return EPB_ERR_OOM;
  }
  if (ctx->ws[slot]) {
    // The old buffer may still be read by queued work: free in stream order.
    cudaError_t e = cudaFreeAsync(ctx->ws[slot], ctx->stream);
    if (e != cudaSuccess) {
      set_error("cudaFreeAsync: %s", cudaGetErrorString(e));
      return EPB_ERR_CUDA;
    }
    ctx->ws[slot] = nullptr;
    ctx->ws_bytes[slot] = 0;
  }
  size_t want = bytes + bytes / 8;  // headroom so that slowly growing callers do not churn
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, want, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("workspace allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
    return EPB_ERR_OOM;
  }
  ctx->ws[slot] = p;
  ctx->ws_bytes[slot] = want;
  *out = p;
  return EPB_OK;
}

// The side stream and its events (non-blocking stream, timing-free events), created once.
int side_stream(epb_ctx* ctx) {
  if (ctx->side) return EPB_OK;
  // highest priority: when CTA slots free up, the side stream's (few, persistent) CTAs are placed first
  int lo = 0, hi = 0;
  EPB_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  cudaStream_t s = nullptr;
  EPB_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi));
  for (auto& e : ctx->side_ev) {
    cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (r != cudaSuccess) {
      cudaStreamDestroy(s);
      for (auto& f : ctx->side_ev)
        if (f) cudaEventDestroy(f), f = nullptr;
      EPB_CUDA(r);
    }
  }
  ctx->side = s;
  return EPB_OK;
}

// The pipeline stream of the mixed pass (high priority, like the side stream) and its events.
int pipe_streams(epb_ctx* ctx) {
  EPB_TRY(side_stream(ctx));
  if (ctx->tail) return EPB_OK;
  int lo = 0, hi = 0;
  EPB_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  cudaStream_t s = nullptr;
  EPB_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi));
  for (auto& e : ctx->pipe_ev) {
    cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (r != cudaSuccess) {
      cudaStreamDestroy(s);
      for (auto& f : ctx->pipe_ev)
        if (f) cudaEventDestroy(f), f = nullptr;
      EPB_CUDA(r);
    }
  }
  ctx->tail = s;
  return EPB_OK;
}

void prof_begin(epb_ctx* ctx, int id) {
  if (!ctx->prof_on) return;
  if (ctx->prof_used == ctx->prof.size()) {
    epb_prof_rec r;
    if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    ctx->prof.push_back(r);
  }
  epb_prof_rec& r = ctx->prof[ctx->prof_used];
  r.id = id;
  cudaEventRecord(r.a, ctx->stream);
}

void prof_end(epb_ctx* ctx) {
  if (!ctx->prof_on || ctx->prof_used == ctx->prof.size()) return;
  cudaEventRecord(ctx->prof[ctx->prof_used].b, ctx->stream);
  ++ctx->prof_used;
}

// Fold recorded event pairs into the per-id totals (synchronises on the events).
static int prof_flush(epb_ctx* ctx) {
  for (size_t i = 0; i < ctx->prof_used; ++i) {
    epb_prof_rec& r = ctx->prof[i];
    EPB_CUDA(cudaEventSynchronize(r.b));
    float ms = 0.f;
    EPB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    ctx->prof_ms[r.id] += ms;
    ctx->prof_cnt[r.id] += 1;
  }
  ctx->prof_used = 0;
  return EPB_OK;
}

}  // namespace epb

using namespace epb;

extern "C" {

const char* epb_last_error(void) { return g_err; }

int epb_version(void) { return 100; }

int epb_create(epb_ctx** out, int device, void* stream) {
  clear_error();
  EPB_CHECK_ARG(out != nullptr, "epb_create: ctx pointer is NULL");
  int ndev = 0;
  EPB_CUDA(cudaGetDeviceCount(&ndev));
  EPB_CHECK_ARG(device >= 0 && device < ndev, "epb_create: device %d out of range (%d devices)",
                device, ndev);
  EPB_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  EPB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("epb200 is built for sm_100a (B200); device %d is sm_%d%d", device, prop.major,
              prop.minor);
    return EPB_ERR_UNSUPPORTED;
  }
  epb_ctx* c = new epb_ctx();
  c->device = device;
  c->stream = (cudaStream_t)stream;
  c->sm_count = prop.multiProcessorCount;
  c->cc_major = prop.major;
  c->cc_minor = prop.minor;
  if (cudaMallocHost(&c->pinned, 64 * sizeof(int64_t)) != cudaSuccess ||
      cudaMalloc(&c->dstat, 64 * sizeof(int)) != cudaSuccess ||
      cudaMemset(c->dstat, 0, 64 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->dstat) cudaFree(c->dstat);
    delete c;
    set_error("epb_create: status/scratch allocation failed");
    return EPB_ERR_OOM;
  }
  *out = c;
  return EPB_OK;
}

int epb_destroy(epb_ctx* ctx) {
  if (!ctx) return EPB_OK;
  make_current(ctx);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  for (auto& e : ctx->side_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->tail) {
    cudaStreamSynchronize(ctx->tail);
    cudaStreamDestroy(ctx->tail);
  }
  for (auto& e : ctx->pipe_ev)
    if (e) cudaEventDestroy(e);
  for (auto& r : ctx->prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  cublas_release(ctx);
  for (int i = 0; i < EPB_WS_NSLOTS; ++i)
    if (ctx->ws[i]) cudaFree(ctx->ws[i]);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->dstat) cudaFree(ctx->dstat);
  delete ctx;
  return EPB_OK;
}

int epb_set_stream(epb_ctx* ctx, void* stream) {
  EPB_CHECK_ARG(ctx, "epb_set_stream: NULL ctx");
  ctx->stream = (cudaStream_t)stream;
  return EPB_OK;
}

int epb_free_bytes(epb_ctx* ctx, uint64_t* free_host, uint64_t* total_host) {
  EPB_CHECK_ARG(ctx && free_host && total_host, "epb_free_bytes: NULL argument");
  EPB_TRY(make_current(ctx));
  size_t f = 0, t = 0;
  EPB_CUDA(cudaMemGetInfo(&f, &t));
  *free_host = f;
  *total_host = t;
  return EPB_OK;
}

int epb_synchronize(epb_ctx* ctx) {
  EPB_CHECK_ARG(ctx, "epb_synchronize: NULL ctx");
  EPB_TRY(make_current(ctx));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  return EPB_OK;
}

int epb_workspace_bytes(epb_ctx* ctx, uint64_t* bytes_host) {
  EPB_CHECK_ARG(ctx && bytes_host, "epb_workspace_bytes: NULL argument");
  uint64_t s = 0;
  for (int i = 0; i < EPB_WS_NSLOTS; ++i) s += ctx->ws_bytes[i];
  *bytes_host = s;
  return EPB_OK;
}

int epb_launch_count(epb_ctx* ctx, int64_t* count_host) {
  EPB_CHECK_ARG(ctx && count_host, "epb_launch_count: NULL argument");
  *count_host = ctx->launches;
  return EPB_OK;
}

int epb_profile_enable(epb_ctx* ctx, int on) {
  EPB_CHECK_ARG(ctx, "epb_profile_enable: NULL ctx");
  EPB_TRY(make_current(ctx));
  if (ctx->prof_on && !on) EPB_TRY(prof_flush(ctx));
  ctx->prof_on = on != 0;
  return EPB_OK;
}

int epb_profile_read(epb_ctx* ctx, double* ms_host, int64_t* count_host, int n, int reset) {
  EPB_CHECK_ARG(ctx && ms_host && count_host && n >= 1, "epb_profile_read: bad argument");
  EPB_TRY(make_current(ctx));
  EPB_TRY(prof_flush(ctx));
  for (int i = 0; i < n && i < EPB_PROF_N; ++i) {
    ms_host[i] = ctx->prof_ms[i];
    count_host[i] = ctx->prof_cnt[i];
    if (reset) {
      ctx->prof_ms[i] = 0;
      ctx->prof_cnt[i] = 0;
    }
  }
  return EPB_OK;
}

int epb_debug_fail_alloc(epb_ctx* ctx, int nth) {
  EPB_CHECK_ARG(ctx, "epb_debug_fail_alloc: NULL ctx");
  ctx->fail_alloc_nth = nth < 0 ? 0 : nth;
  return EPB_OK;
}

int epb_rset_create(epb_ctx* ctx, const int64_t* irvec_host, int64_t nr, epb_rset** out) {
  clear_error();
  EPB_CHECK_ARG(ctx && irvec_host && out, "epb_rset_create: NULL argument");
  EPB_CHECK_ARG(nr >= 1 && nr <= (1 << 24), "epb_rset_create: nr=%lld out of range", (long long)nr);
  EPB_TRY(make_current(ctx));
  epb_rset* r = new epb_rset();
  r->ctx = ctx;
  r->nr = nr;
  r->host.assign(irvec_host, irvec_host + 3 * nr);
  std::vector<int4> packed(nr);
  for (int d = 0; d < 3; ++d) {
    r->lo[d] = 1 << 30;
    r->hi[d] = -(1 << 30);
  }
  for (int64_t i = 0; i < nr; ++i) {
    int v[3];
    for (int d = 0; d < 3; ++d) {
      int64_t x = irvec_host[3 * i + d];
      if (x < -1023 || x > 1023) {
        delete r;
        set_error("epb_rset_create: |R| component %lld exceeds 1023", (long long)x);
        return EPB_ERR_ARG;
      }
      v[d] = (int)x;
      r->lo[d] = v[d] < r->lo[d] ? v[d] : r->lo[d];
      r->hi[d] = v[d] > r->hi[d] ? v[d] : r->hi[d];
    }
    packed[i] = make_int4(v[0], v[1], v[2], 0);
  }
  cudaError_t e = cudaMalloc(&r->dev, nr * sizeof(int4));
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete r;
    set_error("epb_rset_create: allocation failed");
    return EPB_ERR_OOM;
  }
  e = cudaMemcpy(r->dev, packed.data(), nr * sizeof(int4), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(r->dev);
    delete r;
    set_error("epb_rset_create: copy failed: %s", cudaGetErrorString(e));
    return EPB_ERR_CUDA;
  }
  *out = r;
  return EPB_OK;
}

int epb_rset_destroy(epb_rset* r) {
  if (!r) return EPB_OK;
  if (r->ctx) make_current(r->ctx);
  if (r->dev) cudaFree(r->dev);
  delete r;
  return EPB_OK;
}

}  // extern "C"
