// EPW e-ph matrix reader (src/model_new.jl:487-568, read_epmat): streams the binary `<prefix>.epmatwp`
// file (complex128, EPW order (iw, jw, iRe, imode, iRp), iRp slowest) from disk through two pinned host
// buffers into HBM; a scatter kernel applies the R-vector sort (ind_el, ind_ep), the Wigner-Seitz
// degeneracy divisions in the reference's order (phonon side first, then electron side; zero where the
// degeneracy is 0) and writes the "el" layout (i, j, nu, Rp, Re) or the "ph" layout (i, j, nu, Re, Rp)
// directly. File reads of one chunk overlap the copy and scatter of the previous one.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "epb_common.cuh"

namespace epb {

struct EpmatScatter {
  const double2* chunk;  // (nw, nw, nr_el, nmc): modes m0 .. m0 + nmc - 1 of one file Rp
  int64_t nw, nm, nr_el, nr_ep, nmc, m0;
  int64_t rp_new;            // sorted index of this Rp (0-based)
  const int32_t* inv_el;     // file Re index -> sorted index (0-based)
  const int32_t* ndeg_ep;    // (d1, d2, nr_ep) sorted order, or nullptr (no phonon-side division)
  int64_t d1, d2;
  const int32_t* ndeg_el;    // (de, de, nr_el) sorted order, or nullptr
  int64_t de;
  int layout;                // 0 "el", 1 "ph"
  double2* out;
};

__global__ void epmat_scatter_kernel(EpmatScatter a) {
  const int64_t nw2 = a.nw * a.nw;
  const int64_t total = nw2 * a.nr_el * a.nmc;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ij = e % nw2, iw = ij % a.nw, jw = ij / a.nw;
    const int64_t re_f = (e / nw2) % a.nr_el;
    const int64_t mode = a.m0 + e / (nw2 * a.nr_el);
    const int64_t re = a.inv_el[re_f];
    double2 v = a.chunk[e];
    if (a.ndeg_ep) {
      const int64_t iatm = mode / 3;
      const int32_t d = a.d1 == 1 ? a.ndeg_ep[a.rp_new * a.d1 * a.d2]
                                  : a.ndeg_ep[iw + a.d1 * (iatm + a.d2 * a.rp_new)];
      v = d == 0 ? make_double2(0.0, 0.0) : make_double2(v.x / (double)d, v.y / (double)d);
    }
    if (a.ndeg_el) {
      const int32_t d = a.de == 1 ? a.ndeg_el[re] : a.ndeg_el[iw + a.de * (jw + a.de * re)];
      v = d == 0 ? make_double2(0.0, 0.0) : make_double2(v.x / (double)d, v.y / (double)d);
    }
    const int64_t b = ij + nw2 * mode;
    const int64_t nd = nw2 * a.nm;
    const int64_t o = a.layout == 0 ? b + nd * (a.rp_new + a.nr_ep * re) : b + nd * (re + a.nr_el * a.rp_new);
    a.out[o] = v;
  }
}

// pread of [off, off + bytes) into dst by `nt` threads on disjoint slices; false on a short read.
static bool pread_parallel(int fd, char* dst, int64_t bytes, int64_t off, int nt) {
  std::atomic<bool> ok{true};
  auto part = [&](int t) {
    const int64_t a = bytes * t / nt, b = bytes * (t + 1) / nt;
    int64_t got = a;
    while (got < b) {
      const ssize_t r = pread(fd, dst + got, (size_t)(b - got), (off_t)(off + got));
      if (r <= 0) {
        ok = false;
        return;
      }
      got += r;
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(part, t);
  part(0);
  for (auto& x : th) x.join();
  return ok;
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_read_epmat(epb_ctx* ctx, const char* filename, int64_t nw, int64_t nmodes, int64_t nr_el, int64_t nr_ep,
                   const int64_t* ind_el, const int64_t* ind_ep, const int32_t* ndegen_el, int64_t ndegen_el_dim,
                   const int32_t* ndegen_ep, int64_t ndegen_ep_dim1, int64_t ndegen_ep_dim2, int skip_ndegen_ep,
                   int ndegen_pre_divided, int layout, double* out) {
  clear_error();
  EPB_CHECK_ARG(ctx && filename && ind_el && ind_ep && out, "epb_read_epmat: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nmodes >= 1 && nr_el >= 1 && nr_ep >= 1, "epb_read_epmat: bad sizes");
  EPB_CHECK_ARG(layout == 0 || layout == 1, "epb_read_epmat: layout must be 0 (el) or 1 (ph)");
  const bool div_ep = !(skip_ndegen_ep || ndegen_pre_divided), div_el = !ndegen_pre_divided;
  if (div_ep)
    EPB_CHECK_ARG(ndegen_ep && (ndegen_ep_dim1 == 1 || ndegen_ep_dim1 == nw) && ndegen_ep_dim2 >= 1 &&
                      (ndegen_ep_dim1 == 1 || ndegen_ep_dim2 * 3 >= nmodes),
                  "epb_read_epmat: ndegen_ep must be (1, 1, nr_ep) or (nw, nat, nr_ep)");
  if (div_el)
    EPB_CHECK_ARG(ndegen_el && (ndegen_el_dim == 1 || ndegen_el_dim == nw),
                  "epb_read_epmat: ndegen_el must be (1, 1, nr_el) or (nw, nw, nr_el)");
  // sort permutations (1-based "new <- old" as Julia's sortperm) and their inverses
  std::vector<int32_t> inv_el(nr_el, -1);
  std::vector<int64_t> inv_ep(nr_ep, -1);
  for (int64_t i = 0; i < nr_el; ++i) {
    EPB_CHECK_ARG(ind_el[i] >= 1 && ind_el[i] <= nr_el && inv_el[ind_el[i] - 1] < 0,
                  "epb_read_epmat: ind_el is not a permutation of 1..%lld", (long long)nr_el);
    inv_el[ind_el[i] - 1] = (int32_t)i;
  }
  for (int64_t i = 0; i < nr_ep; ++i) {
    EPB_CHECK_ARG(ind_ep[i] >= 1 && ind_ep[i] <= nr_ep && inv_ep[ind_ep[i] - 1] < 0,
                  "epb_read_epmat: ind_ep is not a permutation of 1..%lld", (long long)nr_ep);
    inv_ep[ind_ep[i] - 1] = i;
  }
  const int64_t nw2 = nw * nw;
  const int64_t per_mode = 16 * nw2 * nr_el;  // bytes of one (Rp, mode) slab in the file
  const int64_t total = per_mode * nmodes * nr_ep;
  const int fd = open(filename, O_RDONLY);
  EPB_CHECK_ARG(fd >= 0, "epb_read_epmat: cannot open %s", filename);
  struct stat sb;
  if (fstat(fd, &sb) != 0 || (int64_t)sb.st_size < total) {
    close(fd);
    set_error("epb_read_epmat: %s holds %lld bytes, %lld expected for nw=%lld nmodes=%lld nr_el=%lld nr_ep=%lld",
              filename, (long long)sb.st_size, (long long)total, (long long)nw, (long long)nmodes, (long long)nr_el,
              (long long)nr_ep);
    return EPB_ERR_ARG;
  }
  int st = make_current(ctx);
  if (st != EPB_OK) {
    close(fd);
    return st;
  }
  // chunks: a run of modes of one Rp, at most 256 MB (at least one mode)
  const int64_t nmc = std::max<int64_t>(1, std::min<int64_t>(nmodes, ((int64_t)256 << 20) / per_mode));
  const int64_t cbytes = per_mode * nmc;
  void* host[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  int32_t* d_inv = nullptr;
  int32_t* d_nep = nullptr;
  int32_t* d_nel = nullptr;
  void* dstage = nullptr;
  auto cleanup = [&]() {
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < 2; ++i) {
      if (host[i]) cudaFreeHost(host[i]);
      if (done[i]) cudaEventDestroy(done[i]);
    }
    if (d_inv) cudaFree(d_inv);
    if (d_nep) cudaFree(d_nep);
    if (d_nel) cudaFree(d_nel);
    if (dstage) cudaFree(dstage);
    close(fd);
  };
#define EPW_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      set_error("%s failed: %s", #call, cudaGetErrorString(_e));                            \
      cleanup();                                                                             \
      return EPB_ERR_CUDA;                                                                   \
    }                                                                                        \
  } while (0)
  for (int i = 0; i < 2; ++i) {
    EPW_CUDA(cudaHostAlloc(&host[i], cbytes, cudaHostAllocDefault));
    EPW_CUDA(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
  }
  EPW_CUDA(cudaMalloc(&dstage, 2 * cbytes));
  EPW_CUDA(cudaMalloc(&d_inv, 4 * nr_el));
  EPW_CUDA(cudaMemcpyAsync(d_inv, inv_el.data(), 4 * nr_el, cudaMemcpyHostToDevice, ctx->stream));
  if (div_ep) {
    const int64_t n = ndegen_ep_dim1 * ndegen_ep_dim2 * nr_ep;
    EPW_CUDA(cudaMalloc(&d_nep, 4 * n));
    EPW_CUDA(cudaMemcpyAsync(d_nep, ndegen_ep, 4 * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (div_el) {
    const int64_t n = ndegen_el_dim * ndegen_el_dim * nr_el;
    EPW_CUDA(cudaMalloc(&d_nel, 4 * n));
    EPW_CUDA(cudaMemcpyAsync(d_nel, ndegen_el, 4 * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  // the pinned buffers are reused only after the copy out of them has finished (event per buffer); the
  // page-cache -> pinned copy of a chunk runs on several threads (one thread reaches ~5 GB/s)
  const int nthreads = (int)std::max<unsigned>(1, std::min<unsigned>(16, std::thread::hardware_concurrency()));
  int64_t c = 0;
  for (int64_t rp_f = 0; rp_f < nr_ep; ++rp_f) {
    for (int64_t m0 = 0; m0 < nmodes; m0 += nmc, ++c) {
      const int64_t nm_here = std::min(nmc, nmodes - m0);
      const int64_t bytes = per_mode * nm_here;
      const int b = (int)(c & 1);
      EPW_CUDA(cudaEventSynchronize(done[b]));
      const int64_t off = per_mode * (nmodes * rp_f + m0);
      if (!pread_parallel(fd, (char*)host[b], bytes, off, nthreads)) {
        set_error("epb_read_epmat: read of %s failed in bytes %lld..%lld", filename, (long long)off,
                  (long long)(off + bytes));
        cleanup();
        return EPB_ERR_ARG;
      }
      double2* dchunk = (double2*)((char*)dstage + b * cbytes);
      EPW_CUDA(cudaMemcpyAsync(dchunk, host[b], bytes, cudaMemcpyHostToDevice, ctx->stream));
      EPW_CUDA(cudaEventRecord(done[b], ctx->stream));
      EpmatScatter a;
      a.chunk = dchunk;
      a.nw = nw;
      a.nm = nmodes;
      a.nr_el = nr_el;
      a.nr_ep = nr_ep;
      a.nmc = nm_here;
      a.m0 = m0;
      a.rp_new = inv_ep[rp_f];
      a.inv_el = d_inv;
      a.ndeg_ep = div_ep ? d_nep : nullptr;
      a.d1 = ndegen_ep_dim1;
      a.d2 = ndegen_ep_dim2;
      a.ndeg_el = div_el ? d_nel : nullptr;
      a.de = ndegen_el_dim;
      a.layout = layout;
      a.out = (double2*)out;
      const int64_t n = nw2 * nr_el * nm_here;
      const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)ctx->sm_count * 16));
      epmat_scatter_kernel<<<grid, 256, 0, ctx->stream>>>(a);
      ++ctx->launches;
      EPW_CUDA(cudaGetLastError());
    }
  }
#undef EPW_CUDA
  cleanup();
  return EPB_OK;
}

}  // extern "C"
