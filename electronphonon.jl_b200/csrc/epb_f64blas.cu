// The plain FP64 pass's dense algebra on cuBLAS: the reference's own GPU path runs its Fourier sums as
// ZGEMMs against a phase matrix (`fourier_batched!`, src/wannier/batched_fourier_core.jl:117-139, on
// CuArrays through cuBLAS), the kR->kq stage as a ZGEMM (`get_eph_kR_to_kq_batched!`,
// src/wannier_to_bloch_batched.jl:245-273) and, for nw * nm above `_FUSED_ROT_MAX_NWNM`, the two
// rotations as strided-batched ZGEMMs (`eph_apply_rotations!`, src/wannier_to_bloch_batched.jl:442-455).
// This file holds those library calls for the FP64 denominator of the mixed pass, plus the |ep|^2 / (2
// omega) fold with the per-mode reduction and the sampled blocks (a kernel of this project).
#include <cublas_v2.h>

#include <algorithm>

#include "epb_common.cuh"

namespace epb {

int launch_phase(epb_ctx* ctx, const epb_rset* rs, const double* xk, int64_t nk, double2* phase);

static const char* cublas_msg(cublasStatus_t s) {
  switch (s) {
    case CUBLAS_STATUS_NOT_INITIALIZED: return "not initialized";
    case CUBLAS_STATUS_ALLOC_FAILED: return "allocation failed";
    case CUBLAS_STATUS_INVALID_VALUE: return "invalid value";
    case CUBLAS_STATUS_ARCH_MISMATCH: return "architecture mismatch";
    case CUBLAS_STATUS_EXECUTION_FAILED: return "execution failed";
    case CUBLAS_STATUS_NOT_SUPPORTED: return "not supported";
    default: return "error";
  }
}

#define EPB_BLAS(call)                                                      \
  do {                                                                      \
    cublasStatus_t s_ = (call);                                             \
    if (s_ != CUBLAS_STATUS_SUCCESS) {                                      \
      set_error("cuBLAS %s: %s (%d)", #call, cublas_msg(s_), (int)s_);      \
      return EPB_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

// The context's handle, bound to the context's current stream.
static int blas(epb_ctx* ctx, cublasHandle_t* out) {
  if (!ctx->cublas) {
    cublasHandle_t h = nullptr;
    EPB_BLAS(cublasCreate(&h));
    ctx->cublas = h;
  }
  cublasHandle_t h = (cublasHandle_t)ctx->cublas;
  EPB_BLAS(cublasSetStream(h, ctx->stream));
  *out = h;
  return EPB_OK;
}

void cublas_release(epb_ctx* ctx) {
  if (ctx->cublas) cublasDestroy((cublasHandle_t)ctx->cublas);
  ctx->cublas = nullptr;
}

static cublasOperation_t blas_op(char t) { return t == 'C' ? CUBLAS_OP_C : t == 'T' ? CUBLAS_OP_T : CUBLAS_OP_N; }

// C = op(A) op(B), column-major, one matrix.
int zgemm_blas(epb_ctx* ctx, char ta, char tb, int64_t m, int64_t n, int64_t k, const double2* A, int64_t lda,
               const double2* B, int64_t ldb, double2* C, int64_t ldc) {
  cublasHandle_t h;
  EPB_TRY(blas(ctx, &h));
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  EPB_BLAS(cublasZgemm(h, blas_op(ta), blas_op(tb), (int)m, (int)n, (int)k, &one, (const cuDoubleComplex*)A,
                       (int)lda, (const cuDoubleComplex*)B, (int)ldb, &zero, (cuDoubleComplex*)C, (int)ldc));
  return EPB_OK;
}

// C_i = op(A_i) op(B_i) for i < batch (strides in elements; a stride of 0 reuses the operand).
int zgemm_blas_strided(epb_ctx* ctx, char ta, char tb, int64_t m, int64_t n, int64_t k, const double2* A,
                       int64_t lda, int64_t sa, const double2* B, int64_t ldb, int64_t sb, double2* C, int64_t ldc,
                       int64_t sc, int64_t batch) {
  cublasHandle_t h;
  EPB_TRY(blas(ctx, &h));
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  EPB_BLAS(cublasZgemmStridedBatched(h, blas_op(ta), blas_op(tb), (int)m, (int)n, (int)k, &one,
                                     (const cuDoubleComplex*)A, (int)lda, (long long)sa, (const cuDoubleComplex*)B,
                                     (int)ldb, (long long)sb, &zero, (cuDoubleComplex*)C, (int)ldc, (long long)sc,
                                     (int)batch));
  return EPB_OK;
}

// op(x) = sum_R op_r[:, R] exp(2 pi i R . x) for npts points as one ZGEMM: the phase matrix P (nr x npts,
// the reference's fourier_phase!) in the given scratch, then out (ndata x npts, ld ldo) = op_r P.
int fourier_zgemm(epb_ctx* ctx, const double2* op_r, int64_t ndata, int64_t ld_op, const epb_rset* rs,
                  const double* x, int64_t npts, double2* phase_scratch, double2* out, int64_t ldo) {
  if (npts == 0) return EPB_OK;
  EPB_TRY(launch_phase(ctx, rs, x, npts, phase_scratch));
  return zgemm_blas(ctx, 'N', 'N', ndata, npts, rs->nr, op_r, ld_op, phase_scratch, rs->nr, out, ldo);
}

// |ep|^2 / (2 omega) of one k over all q: ep is (nw^2, nm) per q (ld nw^2 nm between q), omega (nm, nq).
// Adds sum_{m, n, q} to g2sum[nu] and writes the sampled q's blocks (q % stride == 0) in full. One CTA
// per q at a time, threads over the nw^2 band pairs of each mode; per-mode partial sums in registers.
__global__ void __launch_bounds__(256) g2_fold_f64_kernel(const double2* __restrict__ ep, const double* __restrict__ omega,
                                                          int mn, int nm, int64_t nq, double* __restrict__ g2sum,
                                                          double* __restrict__ sample, int64_t stride) {
  __shared__ double red[32];
  for (int e = threadIdx.x; e < 32; e += blockDim.x) red[e] = 0.0;
  double part[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) part[i] = 0.0;
  const int64_t nd = (int64_t)mn * nm;
  for (int64_t q = blockIdx.x; q < nq; q += gridDim.x) {
    const double2* eq = ep + q * nd;
    const bool samp = sample && (q % stride == 0);
    double* sq = samp ? sample + (q / stride) * nd : nullptr;
#pragma unroll
    for (int nu = 0; nu < 32; ++nu) {
      if (nu < nm) {
        const double w = 1.0 / (2.0 * omega[nu + q * nm]);
        for (int e = threadIdx.x; e < mn; e += blockDim.x) {
          const double2 a = eq[e + (int64_t)nu * mn];
          const double v = (a.x * a.x + a.y * a.y) * w;
          if (samp) sq[e + (int64_t)nu * mn] = v;
          part[nu] += v;
        }
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int nu = 0; nu < 32; ++nu) {
    if (nu < nm) {
      double v = part[nu];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&red[nu], v);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nm; e += blockDim.x) atomicAdd(&g2sum[e], red[e]);
}

int g2_fold_f64(epb_ctx* ctx, const double2* ep, const double* omega, int nw, int nm, int64_t nq, double* g2sum,
                double* sample, int64_t stride) {
  if (nq == 0) return EPB_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(nq, (int64_t)ctx->sm_count * 8);
  g2_fold_f64_kernel<<<grid, 256, 0, ctx->stream>>>(ep, omega, nw * nw, nm, nq, g2sum, sample, stride < 1 ? 1 : stride);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

}  // namespace epb
