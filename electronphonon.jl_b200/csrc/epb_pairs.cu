// Energy-window selection of k points and of (k, q) pairs, with the optional learned pre-filter.
//
// Reference semantics (src/filter.jl:19,40-72; src/electron_state.jl:118-128; the pair skip of
// src/run_eph_over_k_and_q.jl:303-307): the in-window band range of a point is
// searchsortedfirst(e, wmin) : searchsortedlast(e, wmax) of its ascending band energies, inclusive at
// both ends; a k point is kept iff the range is non-empty; a (k, q) pair is kept iff the range at
// x_k + x_q is non-empty (the caller passes only the kept k). Band ranges are 1-based, 0 / 0 when
// empty.
//
// The plain evaluation of a point is H(x) by the R -> k Fourier sum and the two Sturm counts at the
// window edges on its Householder tridiagonal (epb_tridiag.cu), which give exactly
// #(e < wmin) + 1 and #(e <= wmax):
//   EPB_PREC_FP64 : FP64 Fourier sum, FP64 reduction and counts;
//   EPB_PREC_MIXED: split-BF16x3 tensor-core Fourier sum, FP32 reduction and counts at wmin -/+ guard
//                   and wmax -/+ guard; a point whose counts differ across a guard interval (an
//                   eigenvalue may lie within `guard` of an edge) is re-evaluated in FP64. With the
//                   guard above the mixed path's eigenvalue error, the ranges equal the FP64 ones.
// The learned pre-filter (epb_mlp.cu) predicts the band energies of every pair point; a point whose
// predicted bands all lie outside [wmin - margin_n, wmax + margin_n] (margin_n = calibrated maximum
// held-out error of band n) has an empty window and is culled; the plain evaluation runs on the rest.
// Every evaluated point's result does not depend on which other points are evaluated with it, so the
// kept set with the pre-filter equals the kept set without it whenever the margins hold.
#include <algorithm>

#include "epb_common.cuh"

struct epb_bands {
  epb_ctx* ctx = nullptr;
  int64_t nw = 0, nr = 0;
  const double2* ham = nullptr;  // (nw^2, nr) caller-owned
  epb_rset* rs = nullptr;
  void* planes = nullptr;        // tensor-core operand planes of H(R)
};

namespace epb {

int band_planes_prepare(epb_ctx* ctx, const double2* ham, int nw, const epb_rset* rs, void** out);
void band_planes_free(void* p);
int64_t band_hk_chunk(const epb_rset* rs);
int band_hk_packed(epb_ctx* ctx, const void* planes, const epb_rset* rs, int nw, const double* xa, const double* xb,
                   int64_t nb, const int64_t* pidx, int64_t pair0, int64_t N, float* Hp);
int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* xk,
                int64_t nk, double2* out, int64_t ldo);
int tridiag_window(epb_ctx* ctx, const float* Hp, const double2* A, int n, int64_t batch, double wmin, double wmax,
                   double delta, int32_t* bmin, int32_t* bmax, int32_t* flag);
int tridiag_eigvals(epb_ctx* ctx, const float* Hp, const double2* A, int n, int64_t batch, double* E);
int tridiag_band(epb_ctx* ctx, const float* Hp, const double2* A, int n, int64_t batch, int band, double* Dt,
                 double* E2t, double* out);
int mlp_predict_norm(epb_ctx* ctx, const epb_mlp* m, const double* xa, const double* xb, int64_t nb,
                     const int64_t* pidx, int64_t pair0, int64_t n, float* out_all);
int split_gemm_check(epb_ctx* ctx);
int mlp_tc_check(epb_ctx* ctx);
int mlp_screen_params(const epb_mlp* m, const float** mu, const float** sc, const double** margin, int* nout,
                      bool* calibrated);

constexpr int CMP_THREADS = 1024;
constexpr int64_t EPB_AUDIT_STRIDE = 64;  // one culled pair in 64 is re-evaluated by the plain path

static unsigned grid_pts(epb_ctx* ctx, int64_t total) {
  int64_t b = cdiv(total, 256);
  const int64_t cap = (int64_t)ctx->sm_count * 16;
  return (unsigned)std::max<int64_t>(1, std::min(b, cap));
}

// x_j (3 x N) of listed points: position q = pos[j] (or j); pair p = pidx[q] (or pair0 + q);
// x = xa[p / nb] + xb[p % nb], or xa[p] when xb == null.
__global__ void gather_points_kernel(const double* __restrict__ xa, const double* __restrict__ xb, int64_t nb,
                                     const int64_t* __restrict__ pidx, int64_t pair0, const int64_t* __restrict__ pos,
                                     int64_t N, double* __restrict__ x) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < N; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = pos ? pos[j] : j;
    const int64_t p = pidx ? pidx[q] : pair0 + q;
    if (xb) {
      const int64_t a = p / nb, b = p % nb;
      for (int d = 0; d < 3; ++d) x[3 * j + d] = xa[3 * a + d] + xb[3 * b + d];
    } else {
      for (int d = 0; d < 3; ++d) x[3 * j + d] = xa[3 * p + d];
    }
  }
}

// ---- stable compaction: block counts, one-block scan onto a running device total, scatter ---------
__global__ void cmp_count_kernel(const int32_t* __restrict__ flag, int64_t n, int32_t* __restrict__ bcount) {
  const int64_t j = (int64_t)blockIdx.x * CMP_THREADS + threadIdx.x;
  const int f = j < n ? (flag[j] != 0) : 0;
  __shared__ int ws[CMP_THREADS / 32];
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < CMP_THREADS / 32; ++w) s += ws[w];
    bcount[blockIdx.x] = s;
  }
}

// bcount[i] <- running + exclusive prefix; running += total.
__global__ void cmp_scan_kernel(int32_t* __restrict__ bcount, int64_t nblocks, int64_t* __restrict__ running,
                                int64_t* __restrict__ boff) {
  __shared__ int64_t buf[CMP_THREADS];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = *running;
  __syncthreads();
  for (int64_t base = 0; base < nblocks; base += CMP_THREADS) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < nblocks ? bcount[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < CMP_THREADS; o <<= 1) {
      const int64_t t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nblocks) boff[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += buf[CMP_THREADS - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *running = carry;
}

// out[pos] = src index of each flagged j (pidx[j] or base + j); optional band ranges alongside.
// Positions at or beyond `cap` are counted but not written.
__global__ void cmp_scatter_kernel(const int32_t* __restrict__ flag, int64_t n, const int64_t* __restrict__ boff,
                                   const int64_t* __restrict__ pidx, int64_t base, int64_t* __restrict__ out,
                                   const int32_t* __restrict__ bmin, const int32_t* __restrict__ bmax,
                                   int32_t* __restrict__ omin, int32_t* __restrict__ omax, int64_t cap) {
  const int64_t j = (int64_t)blockIdx.x * CMP_THREADS + threadIdx.x;
  const int f = j < n ? (flag[j] != 0) : 0;
  __shared__ int ws[CMP_THREADS / 32];
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = __popc(bal);
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = threadIdx.x < CMP_THREADS / 32 ? ws[threadIdx.x] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, v, o);
      if (threadIdx.x >= o) v += t;
    }
    if (threadIdx.x < CMP_THREADS / 32) ws[threadIdx.x] = v;  // inclusive
  }
  __syncthreads();
  if (f) {
    const int before = (w > 0 ? ws[w - 1] : 0) + __popc(bal & ((1u << lane) - 1u));
    const int64_t pos = boff[blockIdx.x] + before;
    if (pos < cap) {
      out[pos] = pidx ? pidx[j] : base + j;
      if (omin) {
        omin[pos] = bmin[j];
        omax[pos] = bmax[j];
      }
    }
  }
}

// keep flag from band ranges
__global__ void range_nonempty_kernel(const int32_t* __restrict__ bmin, int64_t n, int32_t* __restrict__ flag) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    flag[j] = bmin[j] > 0;
}

// Results of the FP64 re-evaluation back into the chunk arrays.
__global__ void recheck_merge_kernel(const int64_t* __restrict__ list, int64_t n, const int32_t* __restrict__ rmin,
                                     const int32_t* __restrict__ rmax, int32_t* __restrict__ bmin,
                                     int32_t* __restrict__ bmax) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = list[i];
    bmin[j] = rmin[i];
    bmax[j] = rmax[i];
  }
}

__global__ void i64_to_i32_kernel(const int64_t* __restrict__ a, int64_t n, int32_t* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (int32_t)a[i];
}

// Audit sample: every `stride`-th pair of the chunk that the surrogate culled.
__global__ void audit_mark_kernel(const int32_t* __restrict__ flag, int64_t n, int64_t stride,
                                  int32_t* __restrict__ aflag) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    aflag[j] = flag[j] == 0 && j % stride == 0;
}

__global__ void count_nonempty_kernel(const int32_t* __restrict__ bmin, int64_t n, int64_t* __restrict__ count) {
  int c = 0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    c += bmin[j] > 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd((unsigned long long*)count, (unsigned long long)c);
}

__global__ void fill_one_kernel(int32_t* __restrict__ flag, int64_t n) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    flag[j] = 1;
}

// Surrogate screen: flag[j] = 1 unless every predicted band lies outside [wmin - m_b, wmax + m_b].
__global__ void mlp_screen_kernel(const float* __restrict__ out, int nout, int64_t n, const float* __restrict__ mu,
                                  const float* __restrict__ sc, const double* __restrict__ margin, double wmin,
                                  double wmax, int32_t* __restrict__ flag) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    int f = 0;
    for (int b = 0; b < nout; ++b) {
      const double e = (double)out[j * nout + b] * (double)sc[b] + (double)mu[b];
      f |= (e >= wmin - margin[b]) && (e <= wmax + margin[b]);
    }
    flag[j] = f;
  }
}

// Device compaction of n flags into out (appending at *running); returns nothing to the host.
struct Compactor {
  int32_t* bcount = nullptr;
  int64_t* boff = nullptr;
};

static int compact(epb_ctx* ctx, const Compactor& c, const int32_t* flag, int64_t n, const int64_t* pidx, int64_t base,
                   int64_t* running, int64_t* out, const int32_t* bmin, const int32_t* bmax, int32_t* omin,
                   int32_t* omax, int64_t cap) {
  if (n == 0) return EPB_OK;
  const int64_t nb = cdiv(n, CMP_THREADS);
  cmp_count_kernel<<<(unsigned)nb, CMP_THREADS, 0, ctx->stream>>>(flag, n, c.bcount);
  EPB_LAUNCH_CHECK();
  cmp_scan_kernel<<<1, CMP_THREADS, 0, ctx->stream>>>(c.bcount, nb, running, c.boff);
  EPB_LAUNCH_CHECK();
  cmp_scatter_kernel<<<(unsigned)nb, CMP_THREADS, 0, ctx->stream>>>(flag, n, c.boff, pidx, base, out, bmin, bmax, omin,
                                                                     omax, cap);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

static int64_t read_i64(epb_ctx* ctx, const int64_t* d) {
  int64_t v = -1;
  if (cudaMemcpyAsync(ctx->pinned, d, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return -1;
  v = *ctx->pinned;
  return v;
}

// Workspace of the point evaluator for up to `cap` points per call.
struct EvalWs {
  int64_t cap = 0;
  float* Hp = nullptr;      // cap x nw^2 (mixed)
  double2* Hc = nullptr;    // recheck c128 (cap x nw^2 when FP64)
  double* x = nullptr;      // 3 x cap
  int32_t* flag = nullptr;  // cap
  int64_t* list = nullptr;  // cap
  int32_t* rmin = nullptr;
  int32_t* rmax = nullptr;
  int64_t* cnt = nullptr;   // device counter
  Compactor cmp;
};

static int eval_ws(epb_ctx* ctx, const epb_bands* bd, int64_t cap, EvalWs& w) {
  const int64_t n2 = bd->nw * bd->nw;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_hp = take((size_t)cap * n2 * sizeof(float));
  const size_t o_hc = take((size_t)cap * n2 * sizeof(double2));
  const size_t o_x = take((size_t)cap * 3 * sizeof(double));
  const size_t o_f = take((size_t)cap * sizeof(int32_t));
  const size_t o_l = take((size_t)cap * sizeof(int64_t));
  const size_t o_r0 = take((size_t)cap * sizeof(int32_t));
  const size_t o_r1 = take((size_t)cap * sizeof(int32_t));
  const size_t o_c = take(64);
  const size_t o_bc = take((size_t)(cdiv(cap, CMP_THREADS) + 1) * sizeof(int32_t));
  const size_t o_bo = take((size_t)(cdiv(cap, CMP_THREADS) + 1) * sizeof(int64_t));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PAIR1, off + 256, &ws));
  uint8_t* b = (uint8_t*)ws;
  w.cap = cap;
  w.Hp = (float*)(b + o_hp);
  w.Hc = (double2*)(b + o_hc);
  w.x = (double*)(b + o_x);
  w.flag = (int32_t*)(b + o_f);
  w.list = (int64_t*)(b + o_l);
  w.rmin = (int32_t*)(b + o_r0);
  w.rmax = (int32_t*)(b + o_r1);
  w.cnt = (int64_t*)(b + o_c);
  w.cmp.bcount = (int32_t*)(b + o_bc);
  w.cmp.boff = (int64_t*)(b + o_bo);
  return EPB_OK;
}

// Band ranges of ncand points (position c: pair pidx[c], or pair0 + c; see gather_points_kernel)
// into cmin / cmax [0, ncand), in sub-chunks of at most w.cap points. In the mixed mode the flagged
// positions of every sub-chunk are appended to rc_list (capacity ncand) and re-evaluated in FP64
// together at the end (one count read-back per call).
static int eval_candidates(epb_ctx* ctx, const epb_bands* bd, EvalWs& w, const double* xa, const double* xb,
                           int64_t nb, const int64_t* pidx, int64_t pair0, int64_t ncand, double wmin, double wmax,
                           int prec, double guard, int32_t* cmin, int32_t* cmax, int64_t* rc_list,
                           int64_t* rechecked) {
  if (ncand == 0) return EPB_OK;
  const int nw = (int)bd->nw;
  const int64_t n2 = bd->nw * bd->nw;
  if (prec == EPB_PREC_FP64) {
    for (int64_t c0 = 0; c0 < ncand; c0 += w.cap) {
      const int64_t n = std::min(w.cap, ncand - c0);
      gather_points_kernel<<<grid_pts(ctx, n), 256, 0, ctx->stream>>>(xa, xb, nb, pidx ? pidx + c0 : nullptr,
                                                                      pair0 + c0, nullptr, n, w.x);
      EPB_LAUNCH_CHECK();
      EPB_TRY(fourier_f64(ctx, bd->ham, n2, n2, bd->rs, w.x, n, w.Hc, n2));
      EPB_TRY(tridiag_window(ctx, nullptr, w.Hc, nw, n, wmin, wmax, 0.0, cmin + c0, cmax + c0, nullptr));
    }
    return EPB_OK;
  }
  EPB_CUDA(cudaMemsetAsync(w.cnt, 0, sizeof(int64_t), ctx->stream));
  for (int64_t c0 = 0; c0 < ncand; c0 += w.cap) {
    const int64_t n = std::min(w.cap, ncand - c0);
    EPB_TRY(band_hk_packed(ctx, bd->planes, bd->rs, nw, xa, xb, nb, pidx ? pidx + c0 : nullptr, pair0 + c0, n, w.Hp));
    EPB_TRY(tridiag_window(ctx, w.Hp, nullptr, nw, n, wmin, wmax, guard, cmin + c0, cmax + c0, w.flag));
    EPB_TRY(compact(ctx, w.cmp, w.flag, n, nullptr, c0, w.cnt, rc_list, nullptr, nullptr, nullptr, nullptr, ncand));
  }
  const int64_t nf = read_i64(ctx, w.cnt);
  if (nf < 0) {
    set_error("window evaluation: reading the re-evaluation count failed");
    return EPB_ERR_CUDA;
  }
  *rechecked += nf;
  for (int64_t r0 = 0; r0 < nf; r0 += w.cap) {
    const int64_t n = std::min(w.cap, nf - r0);
    gather_points_kernel<<<grid_pts(ctx, n), 256, 0, ctx->stream>>>(xa, xb, nb, pidx, pair0, rc_list + r0, n, w.x);
    EPB_LAUNCH_CHECK();
    EPB_TRY(fourier_f64(ctx, bd->ham, n2, n2, bd->rs, w.x, n, w.Hc, n2));
    EPB_TRY(tridiag_window(ctx, nullptr, w.Hc, nw, n, wmin, wmax, 0.0, w.rmin, w.rmax, nullptr));
    recheck_merge_kernel<<<grid_pts(ctx, n), 256, 0, ctx->stream>>>(rc_list + r0, n, w.rmin, w.rmax, cmin, cmax);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

// Points per evaluator call.
static int64_t eval_chunk(const epb_bands* bd) {
  int64_t c = band_hk_chunk(bd->rs);
  // c128 recheck buffer of the same count: keep both below ~1.5 GB
  const int64_t per = bd->nw * bd->nw * (int64_t)(sizeof(float) + sizeof(double2));
  const int64_t lim = ((int64_t)1536 << 20) / per;
  return std::max<int64_t>(128, std::min(c, lim) / 128 * 128);
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_bands_create(epb_ctx* ctx, const double* ham_op, int64_t nw, const int64_t* irvec_host, int64_t nr,
                     epb_bands** out) {
  clear_error();
  EPB_CHECK_ARG(ctx && ham_op && irvec_host && out, "epb_bands_create: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nw <= 32 && nr >= 1, "epb_bands_create: unsupported sizes (nw=%lld, nr=%lld)",
                (long long)nw, (long long)nr);
  EPB_TRY(make_current(ctx));
  epb_bands* b = new epb_bands();
  b->ctx = ctx;
  b->nw = nw;
  b->nr = nr;
  b->ham = (const double2*)ham_op;
  int st = epb_rset_create(ctx, irvec_host, nr, &b->rs);
  if (st == EPB_OK) st = band_planes_prepare(ctx, b->ham, (int)nw, b->rs, &b->planes);
  if (st != EPB_OK) {
    if (b->rs) epb_rset_destroy(b->rs);
    delete b;
    return st;
  }
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  *out = b;
  return EPB_OK;
}

int epb_bands_destroy(epb_bands* b) {
  if (!b) return EPB_OK;
  band_planes_free(b->planes);
  if (b->rs) epb_rset_destroy(b->rs);
  delete b;
  return EPB_OK;
}

int epb_bands_eigvals(epb_ctx* ctx, const epb_bands* bd, const double* xk, int64_t nk, double* E, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && bd, "epb_bands_eigvals: NULL argument");
  EPB_CHECK_ARG(nk >= 0 && (nk == 0 || (xk && E)), "epb_bands_eigvals: bad arguments");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_bands_eigvals: unknown precision %d", prec);
  if (nk == 0) return EPB_OK;
  EPB_TRY(make_current(ctx));
  const int64_t ch = eval_chunk(bd);
  EvalWs w;
  EPB_TRY(eval_ws(ctx, bd, std::min(ch, nk), w));
  const int64_t n2 = bd->nw * bd->nw;
  for (int64_t k0 = 0; k0 < nk; k0 += ch) {
    const int64_t n = std::min(ch, nk - k0);
    if (prec == EPB_PREC_FP64) {
      EPB_TRY(fourier_f64(ctx, bd->ham, n2, n2, bd->rs, xk + 3 * k0, n, w.Hc, n2));
      EPB_TRY(tridiag_eigvals(ctx, nullptr, w.Hc, (int)bd->nw, n, E + k0 * bd->nw));
    } else {
      EPB_TRY(band_hk_packed(ctx, bd->planes, bd->rs, (int)bd->nw, xk + 3 * k0, nullptr, 1, nullptr, 0, n, w.Hp));
      EPB_TRY(tridiag_eigvals(ctx, w.Hp, nullptr, (int)bd->nw, n, E + k0 * bd->nw));
    }
  }
  return prec == EPB_PREC_MIXED ? split_gemm_check(ctx) : EPB_OK;
}

int epb_bands_band_energy(epb_ctx* ctx, const epb_bands* bd, const double* xk, int64_t nk, int64_t band,
                          double* E, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && bd, "epb_bands_band_energy: NULL argument");
  EPB_CHECK_ARG(nk >= 0 && (nk == 0 || (xk && E)), "epb_bands_band_energy: bad arguments");
  EPB_CHECK_ARG(band >= 1 && band <= bd->nw, "epb_bands_band_energy: band %lld outside 1..%lld", (long long)band,
                (long long)bd->nw);
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_bands_band_energy: unknown precision %d", prec);
  if (nk == 0) return EPB_OK;
  EPB_TRY(make_current(ctx));
  const int64_t ch = eval_chunk(bd);
  EvalWs w;
  EPB_TRY(eval_ws(ctx, bd, std::min(ch, nk), w));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PAIR2, (size_t)std::min(ch, nk) * 64 * sizeof(double) + 256, &ws));
  double* Dt = (double*)ws;
  double* E2t = Dt + std::min(ch, nk) * 32;
  const int64_t n2 = bd->nw * bd->nw;
  for (int64_t k0 = 0; k0 < nk; k0 += ch) {
    const int64_t n = std::min(ch, nk - k0);
    if (prec == EPB_PREC_FP64) {
      EPB_TRY(fourier_f64(ctx, bd->ham, n2, n2, bd->rs, xk + 3 * k0, n, w.Hc, n2));
      EPB_TRY(tridiag_band(ctx, nullptr, w.Hc, (int)bd->nw, n, (int)band - 1, Dt, E2t, E + k0));
    } else {
      EPB_TRY(band_hk_packed(ctx, bd->planes, bd->rs, (int)bd->nw, xk + 3 * k0, nullptr, 1, nullptr, 0, n, w.Hp));
      EPB_TRY(tridiag_band(ctx, w.Hp, nullptr, (int)bd->nw, n, (int)band - 1, Dt, E2t, E + k0));
    }
  }
  return prec == EPB_PREC_MIXED ? split_gemm_check(ctx) : EPB_OK;
}

int epb_bands_window(epb_ctx* ctx, const epb_bands* bd, const double* xk, int64_t nk, double wmin, double wmax,
                     int prec, double guard, int32_t* bmin, int32_t* bmax, int32_t* keep_idx, int64_t* nkeep_host,
                     epb_window_stats* stats) {
  clear_error();
  EPB_CHECK_ARG(ctx && bd && nkeep_host, "epb_bands_window: NULL argument");
  EPB_CHECK_ARG(nk >= 0 && (nk == 0 || (xk && bmin && bmax && keep_idx)), "epb_bands_window: bad arguments");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || (prec == EPB_PREC_MIXED && guard > 0),
                "epb_bands_window: prec %d / guard %g (mixed needs guard > 0)", prec, guard);
  EPB_TRY(make_current(ctx));
  epb_window_stats st{};
  st.tested = nk;
  *nkeep_host = 0;
  if (nk == 0) {
    if (stats) *stats = st;
    return EPB_OK;
  }
  const int64_t ch = eval_chunk(bd);
  EvalWs w;
  EPB_TRY(eval_ws(ctx, bd, std::min(ch, nk), w));
  EPB_CHECK_ARG(nk <= INT32_MAX, "epb_bands_window: nk too large for int32 indices");
  // nk flags | running count | kept list (int64) | re-evaluation list | compaction scratch
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_f = take((size_t)nk * sizeof(int32_t));
  const size_t o_r = take(64);
  const size_t o_k = take((size_t)nk * sizeof(int64_t));
  const size_t o_l = take((size_t)nk * sizeof(int64_t));
  const size_t o_bc = take((size_t)(cdiv(nk, CMP_THREADS) + 1) * sizeof(int32_t));
  const size_t o_bo = take((size_t)(cdiv(nk, CMP_THREADS) + 1) * sizeof(int64_t));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PAIR0, off + 256, &ws));
  uint8_t* base = (uint8_t*)ws;
  int32_t* kflag = (int32_t*)(base + o_f);
  int64_t* running = (int64_t*)(base + o_r);
  int64_t* kidx = (int64_t*)(base + o_k);
  int64_t* rc_list = (int64_t*)(base + o_l);
  Compactor kc;
  kc.bcount = (int32_t*)(base + o_bc);
  kc.boff = (int64_t*)(base + o_bo);
  EPB_CUDA(cudaMemsetAsync(running, 0, sizeof(int64_t), ctx->stream));
  prof_begin(ctx, EPB_PROF_PAIRS);
  EPB_TRY(eval_candidates(ctx, bd, w, xk, nullptr, 1, nullptr, 0, nk, wmin, wmax, prec, guard, bmin, bmax, rc_list,
                          &st.rechecked));
  range_nonempty_kernel<<<grid_pts(ctx, nk), 256, 0, ctx->stream>>>(bmin, nk, kflag);
  EPB_LAUNCH_CHECK();
  EPB_TRY(compact(ctx, kc, kflag, nk, nullptr, 0, running, kidx, nullptr, nullptr, nullptr, nullptr, nk));
  prof_end(ctx);
  const int64_t nkeep = read_i64(ctx, running);
  if (nkeep < 0) {
    set_error("epb_bands_window: reading the kept count failed");
    return EPB_ERR_CUDA;
  }
  if (nkeep > 0) {
    i64_to_i32_kernel<<<grid_pts(ctx, nkeep), 256, 0, ctx->stream>>>(kidx, nkeep, keep_idx);
    EPB_LAUNCH_CHECK();
  }
  if (prec == EPB_PREC_MIXED) EPB_TRY(split_gemm_check(ctx));
  st.evaluated = nk;
  st.kept = nkeep;
  *nkeep_host = nkeep;
  if (stats) *stats = st;
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  return EPB_OK;
}

int epb_pair_window(epb_ctx* ctx, const epb_bands* bd, const double* xk, int64_t nk, const double* xq, int64_t nq,
                    double wmin, double wmax, const epb_mlp* mlp, int prec, double guard, int64_t* pairs,
                    int32_t* bmin, int32_t* bmax, int64_t capacity, int64_t* npairs_host, epb_window_stats* stats) {
  clear_error();
  EPB_CHECK_ARG(ctx && bd && npairs_host, "epb_pair_window: NULL argument");
  EPB_CHECK_ARG(nk >= 0 && nq >= 0 && capacity >= 0, "epb_pair_window: bad sizes");
  EPB_CHECK_ARG(nk * nq == 0 || (xk && xq), "epb_pair_window: NULL point list");
  EPB_CHECK_ARG(capacity == 0 || (pairs && bmin && bmax), "epb_pair_window: NULL output");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || (prec == EPB_PREC_MIXED && guard > 0),
                "epb_pair_window: prec %d / guard %g (mixed needs guard > 0)", prec, guard);
  const float *mu = nullptr, *sc = nullptr;
  const double* margin = nullptr;
  int nout = 0;
  if (mlp) {
    bool cal = false;
    mlp_screen_params(mlp, &mu, &sc, &margin, &nout, &cal);
    EPB_CHECK_ARG(cal, "epb_pair_window: the surrogate has not been calibrated (epb_mlp_calibrate)");
    EPB_CHECK_ARG(nout == bd->nw, "epb_pair_window: surrogate predicts %d bands, model has %lld", nout,
                  (long long)bd->nw);
  }
  EPB_TRY(make_current(ctx));
  epb_window_stats st{};
  st.tested = nk * nq;
  *npairs_host = 0;
  if (nk * nq == 0) {
    if (stats) *stats = st;
    return EPB_OK;
  }
  const int64_t ech = eval_chunk(bd);
  // pair chunk: whole k rows, about 2^20 pairs
  const int64_t krows = std::max<int64_t>(1, ((int64_t)1 << 20) / nq);
  const int64_t pch = krows * nq;
  EvalWs w;
  EPB_TRY(eval_ws(ctx, bd, std::min(ech, nk * nq), w));
  // chunk buffers: candidate list, band ranges, keep flags, surrogate outputs
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_c = take((size_t)pch * sizeof(int64_t));
  const size_t o_b0 = take((size_t)pch * sizeof(int32_t));
  const size_t o_b1 = take((size_t)pch * sizeof(int32_t));
  const size_t o_f = take((size_t)pch * sizeof(int32_t));
  const size_t o_o = take(mlp ? (size_t)pch * nout * sizeof(float) : 0);
  const size_t o_rc = take((size_t)pch * sizeof(int64_t));
  const size_t o_af = take(mlp ? (size_t)pch * sizeof(int32_t) : 0);
  const size_t o_r = take(64);
  const size_t o_bc = take((size_t)(cdiv(pch, CMP_THREADS) + 1) * sizeof(int32_t));
  const size_t o_bo = take((size_t)(cdiv(pch, CMP_THREADS) + 1) * sizeof(int64_t));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PAIR0, off + 256, &ws));
  uint8_t* base = (uint8_t*)ws;
  int64_t* cand = (int64_t*)(base + o_c);
  int32_t* cmin = (int32_t*)(base + o_b0);
  int32_t* cmax = (int32_t*)(base + o_b1);
  int32_t* flag = (int32_t*)(base + o_f);
  float* pred = (float*)(base + o_o);
  int64_t* running = (int64_t*)(base + o_r);
  int64_t* ccount = running + 1;
  int64_t* rc_list = (int64_t*)(base + o_rc);
  int32_t* aflag = (int32_t*)(base + o_af);
  int64_t* vcount = running + 2;
  Compactor cc;
  cc.bcount = (int32_t*)(base + o_bc);
  cc.boff = (int64_t*)(base + o_bo);
  EPB_CUDA(cudaMemsetAsync(running, 0, sizeof(int64_t), ctx->stream));

  // The screen pays only where it culls: inference costs about a quarter of the plain evaluation of a pair
  // (H(x) GEMM + Householder/Sturm), so once 2^20 screened pairs have culled under a fifth of them the
  // remaining chunks skip it. Skipping never changes the kept set (culling only removes pairs the plain
  // evaluation would reject).
  bool screen = mlp != nullptr;
  for (int64_t k0 = 0; k0 < nk; k0 += krows) {
    const int64_t nkr = std::min(krows, nk - k0);
    const int64_t np = nkr * nq, pair0 = k0 * nq;
    int64_t ncand = np;
    const int64_t* cl = nullptr;  // candidate list (null: all pairs of the chunk)
    if (screen) {
      prof_begin(ctx, EPB_PROF_MLP_INFER);
      EPB_TRY(mlp_predict_norm(ctx, mlp, xk, xq, nq, nullptr, pair0, np, pred));
      mlp_screen_kernel<<<grid_pts(ctx, np), 256, 0, ctx->stream>>>(pred, nout, np, mu, sc, margin, wmin, wmax, flag);
      prof_end(ctx);
      EPB_LAUNCH_CHECK();
      // the plain path judges the surrogate: evaluate an evenly spaced sample of the culled pairs; a
      // culled pair with a non-empty window sends the whole chunk to the plain evaluation
      audit_mark_kernel<<<grid_pts(ctx, np), 256, 0, ctx->stream>>>(flag, np, EPB_AUDIT_STRIDE, aflag);
      EPB_LAUNCH_CHECK();
      EPB_CUDA(cudaMemsetAsync(ccount, 0, 2 * sizeof(int64_t), ctx->stream));  // ccount, vcount
      EPB_TRY(compact(ctx, cc, aflag, np, nullptr, pair0, ccount, cand, nullptr, nullptr, nullptr, nullptr, np));
      const int64_t na = read_i64(ctx, ccount);
      if (na < 0) {
        set_error("epb_pair_window: reading the audit count failed");
        return EPB_ERR_CUDA;
      }
      int64_t viol = 0;
      if (na > 0) {
        EPB_TRY(eval_candidates(ctx, bd, w, xk, xq, nq, cand, 0, na, wmin, wmax, prec, guard, cmin, cmax, rc_list,
                                &st.rechecked));
        count_nonempty_kernel<<<grid_pts(ctx, na), 256, 0, ctx->stream>>>(cmin, na, vcount);
        EPB_LAUNCH_CHECK();
        viol = read_i64(ctx, vcount);
        if (viol < 0) {
          set_error("epb_pair_window: reading the audit result failed");
          return EPB_ERR_CUDA;
        }
      }
      st.audited += na;
      st.violations += viol;
      if (viol > 0) {
        ++st.fallback_chunks;
        fill_one_kernel<<<grid_pts(ctx, np), 256, 0, ctx->stream>>>(flag, np);
        EPB_LAUNCH_CHECK();
      }
      EPB_CUDA(cudaMemsetAsync(ccount, 0, sizeof(int64_t), ctx->stream));
      prof_begin(ctx, EPB_PROF_PAIRS);
      EPB_TRY(compact(ctx, cc, flag, np, nullptr, pair0, ccount, cand, nullptr, nullptr, nullptr, nullptr, np));
      prof_end(ctx);
      ncand = read_i64(ctx, ccount);
      if (ncand < 0) {
        set_error("epb_pair_window: reading the candidate count failed");
        return EPB_ERR_CUDA;
      }
      cl = cand;
      st.culled += np - ncand;
      st.screened += np;
      if (st.screened >= (int64_t(1) << 20) && st.culled * 5 < st.screened) screen = false;
    }
    st.evaluated += ncand;
    EPB_TRY(eval_candidates(ctx, bd, w, xk, xq, nq, cl, pair0, ncand, wmin, wmax, prec, guard, cmin, cmax, rc_list,
                            &st.rechecked));
    prof_begin(ctx, EPB_PROF_PAIRS);
    range_nonempty_kernel<<<grid_pts(ctx, ncand), 256, 0, ctx->stream>>>(cmin, ncand, flag);
    EPB_LAUNCH_CHECK();
    EPB_TRY(compact(ctx, cc, flag, ncand, cl, pair0, running, pairs, cmin, cmax, bmin, bmax, capacity));
    prof_end(ctx);
  }
  if (prec == EPB_PREC_MIXED) EPB_TRY(split_gemm_check(ctx));
  if (mlp) EPB_TRY(mlp_tc_check(ctx));
  const int64_t nk_out = read_i64(ctx, running);
  if (nk_out < 0) {
    set_error("epb_pair_window: reading the kept count failed");
    return EPB_ERR_CUDA;
  }
  st.kept = nk_out;
  *npairs_host = nk_out;
  if (stats) *stats = st;
  if (nk_out > capacity) {
    set_error("epb_pair_window: %lld kept pairs exceed the output capacity %lld", (long long)nk_out,
              (long long)capacity);
    return EPB_ERR_ARG;
  }
  return EPB_OK;
}

}  // extern "C"
