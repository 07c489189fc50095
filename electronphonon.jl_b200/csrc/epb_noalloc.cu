// Energy-window filter that allocates nothing (epb_window_filter_noalloc).
//
// Some callers cannot let a library allocate device memory: a host program whose device memory is
// owned by its own caching allocator (a Julia CUDA.jl pool or a PyTorch caching pool that has
// already reserved the free memory, so a library cudaMalloc fails or evicts the pool), or a hot loop
// that must not pay an allocation's latency, implicit synchronisation or out-of-memory failure. For
// them this entry point keeps its only scratch -- one int32 count per 1024-point block of the
// window compaction -- in a file-scope device array of fixed size, and takes a plain CUDA stream
// instead of an epb_ctx (creating a context allocates).
//
// Limits and behaviour:
//  * at most EPB_NOALLOC_MAX_BLOCKS = 16384 blocks, i.e. nk <= 16384 * 1024 = 16,777,216 points;
//    larger nk is rejected with EPB_ERR_ARG before anything is launched;
//  * the array lives on every GPU that loads the library, for the life of the process (64 KB);
//  * every call shares it: two calls whose kernels overlap on the GPU (different streams, or
//    different host threads on the same device) race on it and give undefined results; calls on
//    one stream are ordered and safe. Each call rewrites every count it later reads, so nothing
//    needs clearing between calls;
//  * the first call on a device resolves the array's device address (cudaGetSymbolAddress) with
//    that device current; make that first call before any stream capture on the device;
//  * that address is kept for the life of the process: after a cudaDeviceReset of a device (CUDA.jl
//    `device_reset!`), which unloads this module's device memory, do not call this entry point on that
//    device again in the same process.
#include <cuda_runtime.h>

#include <mutex>

#include "epb_common.cuh"

#define EPB_NOALLOC_MAX_BLOCKS 16384
#define EPB_NOALLOC_MAX_DEVICES 64

namespace epb {

// The three kernels of the window compaction (epb_filter.cu).
__global__ void window_count_kernel(const double* __restrict__ E, int64_t nw, int64_t nk, double wmin,
                                    double wmax, int32_t* __restrict__ bmin, int32_t* __restrict__ bmax,
                                    double* __restrict__ nbelow, int32_t* __restrict__ block_count);
__global__ void window_scan_kernel(int32_t* __restrict__ block_count, int64_t nblocks,
                                   int64_t* __restrict__ total);
__global__ void window_scatter_kernel(const int32_t* __restrict__ bmin, int64_t nk,
                                      const int32_t* __restrict__ block_off, int32_t* __restrict__ keep_idx);

// Fixed scratch of the allocation-free filter (block counts, then their exclusive scan).
static __device__ __align__(256) int32_t g_window_scratch[EPB_NOALLOC_MAX_BLOCKS];

// Device address of g_window_scratch per device, resolved once with that device current. Host code
// must not pass the symbol itself to a kernel: on the host it only stands in for the device array.
static int32_t* g_window_scratch_dev[EPB_NOALLOC_MAX_DEVICES] = {};
static std::mutex g_window_scratch_mu;

static int window_scratch_ptr(int32_t** out) {
  int dev = -1;
  EPB_CUDA(cudaGetDevice(&dev));
  EPB_CHECK_ARG(dev >= 0 && dev < EPB_NOALLOC_MAX_DEVICES, "epb_window_filter_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_window_scratch_mu);
  if (!g_window_scratch_dev[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_window_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      set_error("epb_window_filter_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                cudaGetErrorString(e));
      return EPB_ERR_CUDA;
    }
    g_window_scratch_dev[dev] = (int32_t*)p;
  }
  *out = g_window_scratch_dev[dev];
  return EPB_OK;
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_window_filter_noalloc(void* stream, const double* E, int64_t nw, int64_t nk, double wmin, double wmax,
                              int32_t* band_min, int32_t* band_max, int32_t* keep_idx, int64_t* nkeep_dev,
                              double* nbelow) {
  clear_error();
  EPB_CHECK_ARG(nkeep_dev, "epb_window_filter_noalloc: nkeep_dev is NULL");
  EPB_CHECK_ARG(nw >= 1 && nw <= 4096 && nk >= 0, "epb_window_filter_noalloc: bad sizes (nw=%lld, nk=%lld)",
                (long long)nw, (long long)nk);
  EPB_CHECK_ARG(nk == 0 || (E && band_min && band_max && keep_idx), "epb_window_filter_noalloc: NULL buffer");
  const int64_t nblocks = (nk + 1023) / 1024;
  EPB_CHECK_ARG(nblocks <= EPB_NOALLOC_MAX_BLOCKS,
                "epb_window_filter_noalloc: nk=%lld exceeds the fixed scratch (at most %lld points)",
                (long long)nk, (long long)EPB_NOALLOC_MAX_BLOCKS * 1024);
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* counts = nullptr;
  EPB_TRY(window_scratch_ptr(&counts));
  if (nk == 0) {
    EPB_CUDA(cudaMemsetAsync(nkeep_dev, 0, sizeof(int64_t), s));
    return EPB_OK;
  }
  window_count_kernel<<<(unsigned)nblocks, 1024, 0, s>>>(E, nw, nk, wmin, wmax, band_min, band_max, nbelow, counts);
  EPB_CUDA(cudaGetLastError());
  window_scan_kernel<<<1, 1024, 0, s>>>(counts, nblocks, nkeep_dev);
  EPB_CUDA(cudaGetLastError());
  window_scatter_kernel<<<(unsigned)nblocks, 1024, 0, s>>>(band_min, nk, counts, keep_idx);
  EPB_CUDA(cudaGetLastError());
  return EPB_OK;
}

}  // extern "C"
