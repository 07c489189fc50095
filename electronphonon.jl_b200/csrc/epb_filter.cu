// Energy-window selection with fused compaction, and the grid iq hash.
//
// Window (src/filter.jl:19,40-72): for sorted band energies E[:, k], the in-window range is
// searchsortedfirst(E, wmin) : searchsortedlast(E, wmax) (inclusive at both ends); k is kept iff it
// is non-empty. The reference copies all eigenvalues to the host and loops there; here one pass over
// E writes the per-k band range and the ascending list of kept k (block-local ballot/popc scan,
// block offsets from a tiny second pass), so only the kept count ever needs to leave the device.
#include "epb_common.cuh"

namespace epb {

constexpr int W_THREADS = 1024;

__device__ __forceinline__ void window_range(const double* e, int nw, double wmin, double wmax,
                                             int& first, int& last) {
  // e ascending; first = #(e < wmin) + 1, last = #(e <= wmax)
  int lo = 0, hi = 0;
  for (int i = 0; i < nw; ++i) {
    double v = e[i];
    lo += v < wmin;
    hi += v <= wmax;
  }
  first = lo + 1;
  last = hi;
}

__global__ void window_count_kernel(const double* __restrict__ E, int64_t nw, int64_t nk, double wmin,
                                    double wmax, int32_t* __restrict__ bmin, int32_t* __restrict__ bmax,
                                    double* __restrict__ nbelow, int32_t* __restrict__ block_count) {
  int64_t k = (int64_t)blockIdx.x * W_THREADS + threadIdx.x;
  int keep = 0;
  if (k < nk) {
    int first, last;
    window_range(E + k * nw, (int)nw, wmin, wmax, first, last);
    keep = last >= first;
    bmin[k] = keep ? first : 0;
    bmax[k] = keep ? last : 0;
    if (nbelow) nbelow[k] = (double)(first - 1);
  }
  __shared__ int wsum[W_THREADS / 32];
  unsigned bal = __ballot_sync(0xffffffffu, keep);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < W_THREADS / 32; ++w) s += wsum[w];
    block_count[blockIdx.x] = s;
  }
}

// single block: exclusive scan of block counts (in place) and the total.
__global__ void window_scan_kernel(int32_t* __restrict__ block_count, int64_t nblocks,
                                   int64_t* __restrict__ total) {
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  __shared__ int64_t buf[W_THREADS];
  for (int64_t base = 0; base < nblocks; base += W_THREADS) {
    int64_t i = base + threadIdx.x;
    int64_t v = i < nblocks ? block_count[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < W_THREADS; off <<= 1) {
      int64_t t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nblocks) block_count[i] = (int32_t)(carry + buf[threadIdx.x] - v);
    __syncthreads();
    if (threadIdx.x == W_THREADS - 1) carry += buf[W_THREADS - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void window_scatter_kernel(const int32_t* __restrict__ bmin, int64_t nk,
                                      const int32_t* __restrict__ block_off, int32_t* __restrict__ keep_idx) {
  int64_t k = (int64_t)blockIdx.x * W_THREADS + threadIdx.x;
  int keep = (k < nk) && bmin[k] > 0;
  unsigned bal = __ballot_sync(0xffffffffu, keep);
  __shared__ int wsum[W_THREADS / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wsum[warp] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < W_THREADS / 32; ++w) {
      int t = wsum[w];
      wsum[w] = s;
      s += t;
    }
  }
  __syncthreads();
  if (keep) {
    int pos = block_off[blockIdx.x] + wsum[warp] + __popc(bal & ((1u << lane) - 1u));
    keep_idx[pos] = (int32_t)k;
  }
}

int window_filter(epb_ctx* ctx, const double* E, int64_t nw, int64_t nk, double wmin, double wmax,
                  int32_t* bmin, int32_t* bmax, int32_t* keep_idx, int64_t* nkeep, double* nbelow) {
  if (nk == 0) {
    EPB_CUDA(cudaMemsetAsync(nkeep, 0, sizeof(int64_t), ctx->stream));
    return EPB_OK;
  }
  int64_t nblocks = cdiv(nk, W_THREADS);
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_FLAGS, 64 + sizeof(int32_t) * nblocks, &ws));
  int32_t* bc = (int32_t*)((char*)ws + 64);
  window_count_kernel<<<(unsigned)nblocks, W_THREADS, 0, ctx->stream>>>(E, nw, nk, wmin, wmax, bmin, bmax,
                                                                        nbelow, bc);
  EPB_LAUNCH_CHECK();
  window_scan_kernel<<<1, W_THREADS, 0, ctx->stream>>>(bc, nblocks, nkeep);
  EPB_LAUNCH_CHECK();
  window_scatter_kernel<<<(unsigned)nblocks, W_THREADS, 0, ctx->stream>>>(bmin, nk, bc, keep_idx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// ---------------------------------------------------------------------------------------------
__global__ void fill_iqs_kernel(const int64_t* __restrict__ xkq_int, int64_t nkq, int64_t k1, int64_t k2,
                                int64_t k3, int64_t ng1, int64_t ng2, int64_t ng3,
                                const int64_t* __restrict__ dense, int64_t* __restrict__ iqs,
                                int* __restrict__ miss) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nkq) return;
  int64_t d1 = xkq_int[3 * j] - k1, d2 = xkq_int[3 * j + 1] - k2, d3 = xkq_int[3 * j + 2] - k3;
  bool ok = (-ng1 < d1 && d1 < 2 * ng1) && (-ng2 < d2 && d2 < 2 * ng2) && (-ng3 < d3 && d3 < 2 * ng3);
  int64_t iq = 0;
  if (ok) {
    d1 = d1 < 0 ? d1 + ng1 : (d1 >= ng1 ? d1 - ng1 : d1);
    d2 = d2 < 0 ? d2 + ng2 : (d2 >= ng2 ? d2 - ng2 : d2);
    d3 = d3 < 0 ? d3 + ng3 : (d3 >= ng3 ? d3 - ng3 : d3);
    iq = dense[(d1 * ng2 + d2) * ng3 + d3];
  }
  iqs[j] = iq;
  if (iq < 1) atomicAdd(miss, 1);
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_window_filter(epb_ctx* ctx, const double* E, int64_t nw, int64_t nk, double wmin,
                      double wmax, int32_t* band_min, int32_t* band_max, int32_t* keep_idx,
                      int64_t* nkeep_dev, double* nbelow) {
  clear_error();
  EPB_CHECK_ARG(ctx && nkeep_dev, "epb_window_filter: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nw <= 4096 && nk >= 0, "epb_window_filter: bad sizes");
  EPB_CHECK_ARG(nk == 0 || (E && band_min && band_max && keep_idx), "epb_window_filter: NULL buffer");
  EPB_CHECK_ARG(nk < (int64_t)1 << 31, "epb_window_filter: nk must be < 2^31");
  EPB_TRY(make_current(ctx));
  return window_filter(ctx, E, nw, nk, wmin, wmax, band_min, band_max, keep_idx, nkeep_dev, nbelow);
}

int epb_fill_iqs(epb_ctx* ctx, const int64_t* xkq_int, int64_t nkq, const int64_t* xk_int_host,
                 int64_t ng1, int64_t ng2, int64_t ng3, const int64_t* dense_hash_to_iq,
                 int64_t* iqs) {
  clear_error();
  EPB_CHECK_ARG(ctx && xk_int_host, "epb_fill_iqs: NULL argument");
  EPB_CHECK_ARG(ng1 >= 1 && ng2 >= 1 && ng3 >= 1 && nkq >= 0, "epb_fill_iqs: bad sizes");
  EPB_CHECK_ARG(nkq == 0 || (xkq_int && dense_hash_to_iq && iqs), "epb_fill_iqs: NULL buffer");
  EPB_TRY(make_current(ctx));
  if (nkq == 0) return EPB_OK;
  int* miss = ctx->dstat + 3;
  EPB_CUDA(cudaMemsetAsync(miss, 0, sizeof(int), ctx->stream));
  fill_iqs_kernel<<<(unsigned)cdiv(nkq, 256), 256, 0, ctx->stream>>>(
      xkq_int, nkq, xk_int_host[0], xk_int_host[1], xk_int_host[2], ng1, ng2, ng3, dense_hash_to_iq, iqs, miss);
  EPB_LAUNCH_CHECK();
  int* h = (int*)ctx->pinned;
  EPB_CUDA(cudaMemcpyAsync(h, miss, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*h > 0) {
    set_error("kq - k = q point not found in precomputed qpts (%d misses)", *h);
    return EPB_ERR_ARG;
  }
  return EPB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// FilteredStates on the device (src/band_states.jl:85-121, 283-287): from the per-k in-window band ranges
// of the window filter, the states ordered by k then band (state i = 1, 2, ...), their k and band indices,
// and the index map in the physical-band form the device calculators read, indmap[b - 1, k] = i for the
// states, 0 elsewhere (the reference builds it on the host and uploads it, _indmap_to_device). One pass
// counts the states per k with a block-local scan, one block scans the block totals, one pass writes.
namespace epb {

__device__ __forceinline__ int fs_count(const int32_t* bmin, const int32_t* bmax, int64_t k, int64_t nk, int nw) {
  if (k >= nk) return 0;
  const int lo = bmin[k], hi = bmax[k];
  return (lo >= 1 && hi >= lo && hi <= nw) ? hi - lo + 1 : 0;
}

// exclusive prefix of v over the block (W_THREADS threads); returns it, and the block total in *tot
__device__ __forceinline__ int64_t block_excl_scan(int v, int64_t* tot) {
  __shared__ int64_t wsum[W_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t s = 0;
    for (int w = 0; w < W_THREADS / 32; ++w) {
      const int64_t t = wsum[w];
      wsum[w] = s;
      s += t;
    }
    *tot = s;  // wsum[w] now holds the exclusive warp offsets
  }
  __syncthreads();
  return wsum[warp] + (incl - v);
}

__global__ void fs_count_kernel(const int32_t* __restrict__ bmin, const int32_t* __restrict__ bmax, int64_t nk,
                                int nw, int64_t* __restrict__ block_tot, int* __restrict__ minmax) {
  const int64_t k = (int64_t)blockIdx.x * W_THREADS + threadIdx.x;
  const int c = fs_count(bmin, bmax, k, nk, nw);
  __shared__ int64_t tot;
  block_excl_scan(c, &tot);
  if (c > 0) {
    atomicMin(&minmax[0], bmin[k]);
    atomicMax(&minmax[1], bmax[k]);
  }
  if (threadIdx.x == 0) block_tot[blockIdx.x] = tot;
}

// single block: exclusive scan of the block totals (in place); counts[0] = number of states,
// counts[1] = nband_ignore, counts[2] = nband of the compact map (0, 0 when no state is kept)
__global__ void fs_scan_kernel(int64_t* __restrict__ block_tot, int64_t nblocks, const int* __restrict__ minmax,
                               int64_t* __restrict__ counts) {
  __shared__ int64_t carry;
  __shared__ int64_t buf[W_THREADS];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nblocks; base += W_THREADS) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < nblocks ? block_tot[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < W_THREADS; off <<= 1) {
      const int64_t t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nblocks) block_tot[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == W_THREADS - 1) carry += buf[W_THREADS - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    counts[0] = carry;
    const bool any = carry > 0;
    counts[1] = any ? (int64_t)minmax[0] - 1 : 0;
    counts[2] = any ? (int64_t)minmax[1] - (int64_t)minmax[0] + 1 : 0;
  }
}

__global__ void fs_write_kernel(const int32_t* __restrict__ bmin, const int32_t* __restrict__ bmax, int64_t nk,
                                int nw, const int64_t* __restrict__ block_off, int64_t* __restrict__ indmap,
                                int64_t* __restrict__ iks, int64_t* __restrict__ ibands, int64_t cap) {
  const int64_t k = (int64_t)blockIdx.x * W_THREADS + threadIdx.x;
  const int c = fs_count(bmin, bmax, k, nk, nw);
  __shared__ int64_t tot;
  const int64_t base = block_off[blockIdx.x] + block_excl_scan(c, &tot);  // 0-based index of k's first state
  if (k >= nk) return;
  const int lo = c > 0 ? bmin[k] : 1;
  int64_t* col = indmap + k * (int64_t)nw;
  for (int b = 1; b <= nw; ++b) col[b - 1] = (c > 0 && b >= lo && b < lo + c) ? base + (b - lo) + 1 : 0;
  for (int j = 0; j < c; ++j) {
    const int64_t i = base + j;
    if (i < cap) {
      if (iks) iks[i] = k + 1;
      if (ibands) ibands[i] = lo + j;
    }
  }
}

}  // namespace epb

extern "C" int epb_filtered_states(epb_ctx* ctx, const int32_t* band_min, const int32_t* band_max, int64_t nw,
                                   int64_t nk, int64_t* indmap, int64_t* iks, int64_t* ibands, int64_t capacity,
                                   int64_t* counts_dev) {
  using namespace epb;
  clear_error();
  EPB_CHECK_ARG(ctx && counts_dev, "epb_filtered_states: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nw <= 4096 && nk >= 0 && capacity >= 0, "epb_filtered_states: bad sizes");
  EPB_CHECK_ARG(nk == 0 || (band_min && band_max && indmap), "epb_filtered_states: NULL buffer");
  EPB_TRY(make_current(ctx));
  if (nk == 0) {
    EPB_CUDA(cudaMemsetAsync(counts_dev, 0, 3 * sizeof(int64_t), ctx->stream));
    return EPB_OK;
  }
  const int64_t nblocks = cdiv(nk, W_THREADS);
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_FLAGS, 64 + sizeof(int64_t) * nblocks, &ws));
  int* minmax = (int*)ws;
  int64_t* bt = (int64_t*)((char*)ws + 64);
  EPB_CUDA(cudaMemsetAsync(minmax, 0x7f, sizeof(int), ctx->stream));  // min band: 0x7f7f7f7f
  EPB_CUDA(cudaMemsetAsync(minmax + 1, 0, sizeof(int), ctx->stream));   // max band
  fs_count_kernel<<<(unsigned)nblocks, W_THREADS, 0, ctx->stream>>>(band_min, band_max, nk, (int)nw, bt, minmax);
  EPB_LAUNCH_CHECK();
  fs_scan_kernel<<<1, W_THREADS, 0, ctx->stream>>>(bt, nblocks, minmax, counts_dev);
  EPB_LAUNCH_CHECK();
  fs_write_kernel<<<(unsigned)nblocks, W_THREADS, 0, ctx->stream>>>(band_min, band_max, nk, (int)nw, bt, indmap, iks,
                                                                    ibands, capacity);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}
