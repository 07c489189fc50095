// Wannier -> Bloch Fourier transform, FP64 path.
//
// out[i, j] = sum_r op_r[i, r] * exp(2 pi i R_r . x_j)   (src/wannier/batched_fourier_core.jl:117-139)
//
// The reference materialises the phase matrix (fourier_phase!, batched_fourier_core.jl:24-30) and
// calls ZGEMM. Here the phase never touches HBM: each CTA builds, for its BN k-points, the 1-D
// tables exp(2 pi i m x_{d,j}) for m in [lo_d, hi_d] of each axis once, and forms every phase
// element of a K-tile as the product of three table entries while staging it into shared memory.
// The GEMM itself is a register-tiled FP64 complex GEMM (4 DFMA per complex MAC).
#include <algorithm>

#include "epb_common.cuh"

namespace epb {

// ---------------------------------------------------------------------------------------------
// Standalone phase (for epb_fourier_phase): direct exact-reduction cispi, as in the reference.
__global__ void phase_kernel(const int4* __restrict__ rv, int64_t nr, const double* __restrict__ xk,
                             int64_t nk, double2* __restrict__ phase) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t total = nr * nk;
  if (idx >= total) return;
  int64_t ir = idx % nr, j = idx / nr;
  int4 r = rv[ir];
  phase[idx] = cis2pi(rdotx(r.x, r.y, r.z, xk[3 * j], xk[3 * j + 1], xk[3 * j + 2]));
}

// The same phase from the reference's own operands: R as an FP64 (nr x 3) column-major device matrix
// (leading dimension ldr) and x as (3 x nk) with column stride ldx, the output with column stride ldp.
__global__ void phase_mat_kernel(const double* __restrict__ rm, int64_t ldr, int64_t nr, const double* __restrict__ x,
                                 int64_t ldx, int64_t nk, double2* __restrict__ phase, int64_t ldp) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nr * nk;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ir = idx % nr, j = idx / nr;
    const double* xj = x + j * ldx;
    const double t = __dadd_rn(__dadd_rn(__dmul_rn(rm[ir], xj[0]), __dmul_rn(rm[ir + ldr], xj[1])),
                               __dmul_rn(rm[ir + 2 * ldr], xj[2]));
    phase[ir + j * ldp] = cis2pi(t);
  }
}

// ---------------------------------------------------------------------------------------------
// FP64 GEMM with on-the-fly phase.
constexpr int F_BM = 64, F_BN = 64, F_BK = 8, F_THREADS = 256;
constexpr int F_TAB = 16;  // max per-axis extent of R handled by the table path

struct FourierArgs {
  const double2* op;   // column-major, leading dimension ld
  int64_t ld, M, K, N;
  const int4* rv;      // K lattice vectors
  const double* xk;    // 3 x N
  double2* out;        // M x N, leading dimension ldo
  int64_t ldo;
  int lo0, lo1, lo2, L0, L1, L2;
};

template <bool TABLE>
__global__ void __launch_bounds__(F_THREADS, 2) fourier_f64_kernel(FourierArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* As = reinterpret_cast<double2*>(smem_raw);      // [2][F_BK][F_BM]
  double2* Bs = As + 2 * F_BK * F_BM;                      // [2][F_BK][F_BN]
  double2* tab = Bs + 2 * F_BK * F_BN;                     // [3][F_TAB][F_BN]
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  // warp covers a 4 (rows) x 8 (cols) grid of 4x4 thread tiles
  const int ty = 4 * (warp & 3) + (lane >> 3);
  const int tx = 8 * (warp >> 2) + (lane & 7);
  const int64_t m0 = (int64_t)blockIdx.y * F_BM;
  const int64_t n0 = (int64_t)blockIdx.x * F_BN;

  if (TABLE) {
    const int L[3] = {a.L0, a.L1, a.L2};
    const int lo[3] = {a.lo0, a.lo1, a.lo2};
    for (int e = tid; e < 3 * F_TAB * F_BN; e += F_THREADS) {
      int j = e % F_BN, m = (e / F_BN) % F_TAB, d = e / (F_BN * F_TAB);
      int64_t col = n0 + j;
      double2 v = make_double2(1.0, 0.0);
      if (m < L[d] && col < a.N) v = cis2pi((double)(lo[d] + m) * a.xk[3 * col + d]);
      tab[e] = v;
    }
  }

  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);

  const int64_t ktiles = (a.K + F_BK - 1) / F_BK;

  auto load_tile = [&](int64_t kt, int buf) {
    const int64_t k0 = kt * F_BK;
    // A tile: F_BK x F_BM, 512 elements, 2 per thread; rows contiguous in global.
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      int e = tid + t * F_THREADS;
      int mm = e % F_BM, kk = e / F_BM;
      int64_t row = m0 + mm, k = k0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (row < a.M && k < a.K) v = a.op[row + k * a.ld];
      As[(buf * F_BK + kk) * F_BM + mm] = v;
    }
    // B tile: phase for F_BK vectors x F_BN points
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      int e = tid + t * F_THREADS;
      int jj = e % F_BN, kk = e / F_BN;
      int64_t col = n0 + jj, k = k0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (col < a.N && k < a.K) {
        int4 r = a.rv[k];
        if (TABLE) {
          double2 p0 = tab[(0 * F_TAB + (r.x - a.lo0)) * F_BN + jj];
          double2 p1 = tab[(1 * F_TAB + (r.y - a.lo1)) * F_BN + jj];
          double2 p2 = tab[(2 * F_TAB + (r.z - a.lo2)) * F_BN + jj];
          v = cmul(cmul(p0, p1), p2);
        } else {
          const double* x = a.xk + 3 * col;
          v = cis2pi(rdotx(r.x, r.y, r.z, x[0], x[1], x[2]));
        }
      }
      Bs[(buf * F_BK + kk) * F_BN + jj] = v;
    }
  };

  if (TABLE) __syncthreads();
  load_tile(0, 0);
  __syncthreads();
  for (int64_t kt = 0; kt < ktiles; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) load_tile(kt + 1, buf ^ 1);
#pragma unroll
    for (int kk = 0; kk < F_BK; ++kk) {
      double2 av[4], bv[4];
      const double2* ap = As + (buf * F_BK + kk) * F_BM + ty * 4;
      const double2* bp = Bs + (buf * F_BK + kk) * F_BN + tx * 4;
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = ap[i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = bp[j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }

#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int64_t col = n0 + tx * 4 + j;
    if (col >= a.N) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int64_t row = m0 + ty * 4 + i;
      if (row < a.M) a.out[row + col * a.ldo] = acc[i][j];
    }
  }
}

int launch_phase(epb_ctx* ctx, const epb_rset* rs, const double* xk, int64_t nk, double2* phase) {
  int64_t total = rs->nr * nk;
  if (total == 0) return EPB_OK;
  phase_kernel<<<(unsigned)cdiv(total, 256), 256, 0, ctx->stream>>>(rs->dev, rs->nr, xk, nk, phase);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

static size_t fourier_smem_bytes() {
  return sizeof(double2) * (2 * F_BK * F_BM + 2 * F_BK * F_BN + 3 * F_TAB * F_BN);
}

// Internal entry used by the e-ph drivers as well.
int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                const double* xk, int64_t N, double2* out, int64_t ldo) {
  if (M == 0 || N == 0) return EPB_OK;
  FourierArgs a;
  a.op = op;
  a.ld = ld;
  a.M = M;
  a.K = rs->nr;
  a.N = N;
  a.rv = rs->dev;
  a.xk = xk;
  a.out = out;
  a.ldo = ldo;
  a.lo0 = rs->lo[0];
  a.lo1 = rs->lo[1];
  a.lo2 = rs->lo[2];
  a.L0 = rs->hi[0] - rs->lo[0] + 1;
  a.L1 = rs->hi[1] - rs->lo[1] + 1;
  a.L2 = rs->hi[2] - rs->lo[2] + 1;
  bool table = a.L0 <= F_TAB && a.L1 <= F_TAB && a.L2 <= F_TAB;
  dim3 grid((unsigned)cdiv(N, F_BN), (unsigned)cdiv(M, F_BM));
  EPB_CHECK_ARG(grid.y <= 65535, "fourier: ndata=%lld too large for one launch", (long long)M);
  size_t smem = fourier_smem_bytes();
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(fourier_f64_kernel<true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EPB_CUDA(cudaFuncSetAttribute(fourier_f64_kernel<false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  prof_begin(ctx, EPB_PROF_FOURIER_F64);
  if (table) {
    fourier_f64_kernel<true><<<grid, F_THREADS, smem, ctx->stream>>>(a);
  } else {
    fourier_f64_kernel<false><<<grid, F_THREADS, smem, ctx->stream>>>(a);
  }
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int fourier_mixed(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                  const double* xk, int64_t N, double2* out, int64_t ldo);

}  // namespace epb

using namespace epb;

extern "C" {

int epb_fourier_phase_mat(epb_ctx* ctx, const double* irvec_mat, int64_t ld_r, int64_t nr, const double* xkmat,
                          int64_t ld_x, int64_t nk, double* phase, int64_t ld_p) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_fourier_phase_mat: NULL ctx");
  EPB_CHECK_ARG(nr >= 0 && nk >= 0, "epb_fourier_phase_mat: negative size");
  EPB_CHECK_ARG(nr == 0 || nk == 0 || (irvec_mat && xkmat && phase), "epb_fourier_phase_mat: NULL buffer");
  EPB_CHECK_ARG(ld_r >= nr && ld_x >= 3 && ld_p >= nr, "epb_fourier_phase_mat: leading dimension too small");
  EPB_TRY(make_current(ctx));
  if (nr == 0 || nk == 0) return EPB_OK;
  const int64_t total = nr * nk;
  const unsigned grid = (unsigned)std::min<int64_t>(cdiv(total, 256), (int64_t)ctx->sm_count * 16);
  phase_mat_kernel<<<grid, 256, 0, ctx->stream>>>(irvec_mat, ld_r, nr, xkmat, ld_x, nk, (double2*)phase, ld_p);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_fourier_phase(epb_ctx* ctx, const epb_rset* rset, const double* xk, int64_t nk,
                      double* phase) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset && (nk == 0 || (xk && phase)), "epb_fourier_phase: NULL argument");
  EPB_CHECK_ARG(nk >= 0, "epb_fourier_phase: nk < 0");
  EPB_TRY(make_current(ctx));
  int64_t total = rset->nr * nk;
  if (total == 0) return EPB_OK;
  phase_kernel<<<(unsigned)cdiv(total, 256), 256, 0, ctx->stream>>>(rset->dev, rset->nr, xk, nk,
                                                                    (double2*)phase);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_fourier(epb_ctx* ctx, const double* op_r, int64_t ld_op, int64_t ndata,
                const epb_rset* rset, const double* xk, int64_t nk, double* out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset, "epb_fourier: NULL ctx or rset");
  EPB_CHECK_ARG(ndata >= 0 && nk >= 0 && ld_op >= ndata, "epb_fourier: bad sizes");
  EPB_CHECK_ARG(nk == 0 || ndata == 0 || (op_r && xk && out), "epb_fourier: NULL buffer");
  EPB_TRY(make_current(ctx));
  if (prec == EPB_PREC_FP64)
    return fourier_f64(ctx, (const double2*)op_r, ld_op, ndata, rset, xk, nk, (double2*)out, ndata);
  if (prec == EPB_PREC_MIXED)
    return fourier_mixed(ctx, (const double2*)op_r, ld_op, ndata, rset, xk, nk, (double2*)out, ndata);
  set_error("epb_fourier: unknown precision mode %d", prec);
  return EPB_ERR_ARG;
}

}  // extern "C"
