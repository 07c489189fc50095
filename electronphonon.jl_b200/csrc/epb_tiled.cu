// Device-resident calculator output tiled over outer-k states: the residency decision (whole output in HBM
// or one outer-k tile at a time), the per-batch tile range with its contiguity check, the zeroing of the
// active tile region and its device->host download (src/calculator/tiled_device_output.jl, the state
// range of src/band_states.jl:416-428). Element size 4, 8 or 16 bytes; column-major arrays; the tiled axis
// may be any axis.
#include <algorithm>
#include <vector>

#include "epb_common.cuh"

struct epb_tiled {
  epb_ctx* ctx = nullptr;
  std::vector<int64_t> dims;
  int i_axis = 0, narr = 1, force_block = -1;
  int64_t elem = 8, n_full = 0, nk = 0, n_batch_max = 1;
  double headroom = 1.2;
  // per-k state ranges: first / last state index (1-based, 0 when none) and count
  std::vector<int64_t> kfirst, klast, kcount;
  std::vector<void*> dev;
  bool decided = false, block = false;
  int64_t ni_cap = 0, tile_i0 = 0, tile_ni = 0;
  int64_t inner = 1, outer = 1;  // elements before / after the tiled axis
};

namespace epb {

// States of the 1-based k range [kstart, kend]: (first, last), 1-based; (1, 0) when there are none; an
// error when they do not form a contiguous index range.
static int range_for(const epb_tiled* t, int64_t kstart, int64_t kend, int64_t* first, int64_t* last) {
  int64_t imin = INT64_MAX, imax = 0, count = 0;
  for (int64_t k = std::max<int64_t>(kstart, 1); k <= std::min(kend, t->nk); ++k) {
    if (t->kcount[k - 1] == 0) continue;
    imin = std::min(imin, t->kfirst[k - 1]);
    imax = std::max(imax, t->klast[k - 1]);
    count += t->kcount[k - 1];
  }
  if (count == 0) {
    *first = 1;
    *last = 0;
    return EPB_OK;
  }
  EPB_CHECK_ARG(imax - imin + 1 == count,
                "ind_range_for_k_range: k-range %lld:%lld maps to a non-contiguous state range (%lld states span %lld "
                "indices)",
                (long long)kstart, (long long)kend, (long long)count, (long long)(imax - imin + 1));
  *first = imin;
  *last = imax;
  return EPB_OK;
}

static int fill_ranges(epb_tiled* t, const int64_t* iks, int64_t n, int64_t nk) {
  t->nk = nk;
  t->kfirst.assign(nk, 0);
  t->klast.assign(nk, 0);
  t->kcount.assign(nk, 0);
  for (int64_t i = 1; i <= n; ++i) {
    const int64_t k = iks[i - 1];
    EPB_CHECK_ARG(k >= 1 && k <= nk, "tiled output: state %lld has k index %lld outside 1..%lld", (long long)i,
                  (long long)k, (long long)nk);
    if (t->kcount[k - 1] == 0 || i < t->kfirst[k - 1]) t->kfirst[k - 1] = i;
    t->klast[k - 1] = std::max(t->klast[k - 1], i);
    t->kcount[k - 1] += 1;
  }
  return EPB_OK;
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_ind_range_for_k_range(const int64_t* iks, int64_t n, int64_t nk, int64_t kstart, int64_t kend, int64_t* first,
                              int64_t* last) {
  clear_error();
  EPB_CHECK_ARG((n == 0 || iks) && first && last && n >= 0 && nk >= 0, "epb_ind_range_for_k_range: bad argument");
  epb_tiled t;
  EPB_TRY(fill_ranges(&t, iks, n, nk));
  return range_for(&t, kstart, kend, first, last);
}

int epb_tiled_plan(const int64_t* iks, int64_t n, int64_t nk, int64_t n_batch_max, int64_t* ni_cap) {
  clear_error();
  EPB_CHECK_ARG((n == 0 || iks) && ni_cap && n >= 0 && nk >= 0 && n_batch_max >= 1, "epb_tiled_plan: bad argument");
  epb_tiled t;
  EPB_TRY(fill_ranges(&t, iks, n, nk));
  int64_t cap = 0;
  for (int64_t ks = 1; ks <= nk; ks += n_batch_max) {
    int64_t a = 0, b = 0;
    EPB_TRY(range_for(&t, ks, std::min(ks + n_batch_max - 1, nk), &a, &b));
    cap = std::max(cap, b - a + 1);
  }
  *ni_cap = cap;
  return EPB_OK;
}

int epb_residency_use_block(epb_ctx* ctx, int64_t full_bytes, double headroom, int* use_block) {
  clear_error();
  EPB_CHECK_ARG(ctx && use_block && full_bytes >= 0 && headroom > 0, "epb_residency_use_block: bad argument");
  EPB_TRY(make_current(ctx));
  size_t f = 0, tot = 0;
  EPB_CUDA(cudaMemGetInfo(&f, &tot));
  *use_block = headroom * (double)full_bytes > (double)f ? 1 : 0;
  return EPB_OK;
}

int epb_tiled_create(epb_ctx* ctx, const int64_t* dims, int ndims, int i_axis, int narr, int64_t elem_bytes,
                     int force_block, double headroom, const int64_t* iks, int64_t n_states, int64_t nk,
                     int64_t n_batch_max, epb_tiled** out) {
  clear_error();
  EPB_CHECK_ARG(ctx && dims && out && ndims >= 1 && ndims <= 8, "epb_tiled_create: bad argument");
  EPB_CHECK_ARG(i_axis >= 0 && i_axis < ndims, "epb_tiled_create: i_axis %d out of range for %d dims", i_axis, ndims);
  EPB_CHECK_ARG(narr >= 1 && (elem_bytes == 4 || elem_bytes == 8 || elem_bytes == 16) && headroom > 0 &&
                    force_block >= -1 && force_block <= 1 && n_batch_max >= 1 && nk >= 0 && n_states >= 0 &&
                    (n_states == 0 || iks),
                "epb_tiled_create: bad argument");
  for (int d = 0; d < ndims; ++d) EPB_CHECK_ARG(dims[d] >= 0, "epb_tiled_create: negative dimension");
  EPB_CHECK_ARG(dims[i_axis] == n_states, "epb_tiled_create: dims[i_axis] = %lld must equal the number of states %lld",
                (long long)dims[i_axis], (long long)n_states);
  epb_tiled* t = new epb_tiled();
  t->ctx = ctx;
  t->dims.assign(dims, dims + ndims);
  t->i_axis = i_axis;
  t->narr = narr;
  t->elem = elem_bytes;
  t->force_block = force_block;
  t->headroom = headroom;
  t->n_full = dims[i_axis];
  t->n_batch_max = n_batch_max;
  for (int d = 0; d < i_axis; ++d) t->inner *= dims[d];
  for (int d = i_axis + 1; d < ndims; ++d) t->outer *= dims[d];
  const int st = fill_ranges(t, iks, n_states, nk);
  if (st != EPB_OK) {
    delete t;
    return st;
  }
  *out = t;
  return EPB_OK;
}

int epb_tiled_free(epb_tiled* t) {
  if (!t) return EPB_OK;
  if (t->ctx) make_current(t->ctx);
  for (void* p : t->dev) cudaFree(p);
  t->dev.clear();
  t->decided = t->block = false;
  t->ni_cap = t->tile_i0 = t->tile_ni = 0;
  return EPB_OK;
}

int epb_tiled_destroy(epb_tiled* t) {
  epb_tiled_free(t);
  delete t;
  return EPB_OK;
}

int epb_tiled_begin(epb_ctx* ctx, epb_tiled* t, int64_t kstart, int64_t kend) {
  clear_error();
  EPB_CHECK_ARG(ctx && t && ctx == t->ctx, "epb_tiled_begin: bad context or object");
  EPB_TRY(make_current(ctx));
  if (!t->decided) {
    const int64_t full = t->narr * t->elem * t->inner * t->n_full * t->outer;
    if (t->force_block >= 0) {
      t->block = t->force_block == 1;
    } else {
      int b = 0;
      EPB_TRY(epb_residency_use_block(ctx, full, t->headroom, &b));
      t->block = b != 0;
    }
    int64_t ext = t->n_full;
    if (t->block) {
      int64_t cap = 0;
      for (int64_t ks = 1; ks <= t->nk; ks += t->n_batch_max) {
        int64_t a = 0, b = 0;
        EPB_TRY(range_for(t, ks, std::min(ks + t->n_batch_max - 1, t->nk), &a, &b));
        cap = std::max(cap, b - a + 1);
      }
      t->ni_cap = ext = cap;
    }
    const size_t bytes = (size_t)(t->elem * t->inner * ext * t->outer);
    for (int a = 0; a < t->narr; ++a) {
      void* p = nullptr;
      if (bytes) {
        EPB_CUDA(cudaMalloc(&p, bytes));
        if (!t->block) EPB_CUDA(cudaMemsetAsync(p, 0, bytes, ctx->stream));
      }
      t->dev.push_back(p);
    }
    t->decided = true;
  }
  if (t->block) {
    int64_t a = 0, b = 0;
    EPB_TRY(range_for(t, kstart, kend, &a, &b));
    t->tile_i0 = a - 1;
    t->tile_ni = b - a + 1;
    EPB_CHECK_ARG(t->tile_ni <= t->ni_cap, "epb_tiled_begin: k range %lld:%lld holds %lld states, above the tile "
                  "capacity %lld (a batch wider than n_batch_max)", (long long)kstart, (long long)kend,
                  (long long)t->tile_ni, (long long)t->ni_cap);
    const size_t pitch = (size_t)(t->elem * t->inner * t->ni_cap), width = (size_t)(t->elem * t->inner * t->tile_ni);
    for (void* p : t->dev)
      if (p && width && t->outer)
        EPB_CUDA(cudaMemset2DAsync(p, pitch, 0, width, (size_t)t->outer, ctx->stream));
  }
  return EPB_OK;
}

int epb_tiled_get_info(const epb_tiled* t, epb_tiled_info* info) {
  clear_error();
  EPB_CHECK_ARG(t && info, "epb_tiled_get_info: NULL argument");
  info->allocated = t->dev.empty() ? 0 : 1;
  info->block = t->block ? 1 : 0;
  info->ni_cap = t->ni_cap;
  info->tile_offset = t->tile_i0;
  info->tile_length = t->tile_ni;
  info->tile_stride = t->block ? t->ni_cap : t->n_full;
  return EPB_OK;
}

int epb_tiled_device_array(const epb_tiled* t, int k, void** ptr) {
  clear_error();
  EPB_CHECK_ARG(t && ptr, "epb_tiled_device_array: NULL argument");
  EPB_CHECK_ARG(!t->dev.empty(), "epb_tiled_device_array: no buffers before the first epb_tiled_begin");
  EPB_CHECK_ARG(k >= 0 && k < t->narr, "epb_tiled_device_array: array %d out of 0..%d", k, t->narr - 1);
  *ptr = t->dev[k];
  return EPB_OK;
}

int epb_tiled_download(epb_ctx* ctx, const epb_tiled* t, int k, void* host) {
  clear_error();
  EPB_CHECK_ARG(ctx && t && host && ctx == t->ctx, "epb_tiled_download: bad argument");
  EPB_CHECK_ARG(!t->dev.empty(), "epb_tiled_download: no buffers before the first epb_tiled_begin");
  EPB_CHECK_ARG(k >= 0 && k < t->narr, "epb_tiled_download: array %d out of 0..%d", k, t->narr - 1);
  EPB_TRY(make_current(ctx));
  const int64_t ext = t->block ? t->tile_ni : t->n_full;
  const int64_t cap = t->block ? t->ni_cap : t->n_full;
  const size_t width = (size_t)(t->elem * t->inner * ext), spitch = (size_t)(t->elem * t->inner * cap);
  if (width && t->outer && t->dev[k])
    EPB_CUDA(cudaMemcpy2DAsync(host, width, t->dev[k], spitch, width, (size_t)t->outer, cudaMemcpyDeviceToHost,
                               ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  return EPB_OK;
}

}  // extern "C"
