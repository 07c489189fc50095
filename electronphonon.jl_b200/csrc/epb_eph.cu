// Electron-phonon chain, FP64 path: RR->kR, kR->kq and the fused gauge rotations + |g|^2 fold.
//
//  * RR->kR (src/wannier_to_bloch_batched.jl:178-205): the Fourier over Re goes through the FP64
//    phase-on-the-fly GEMM in k chunks, then one kernel applies the k-leg rotation by uk and the
//    optional additional phase while writing the (nw, nband, nm*nr_ep, k) output.
//  * rotations (ext/ElectronPhononCUDAExt.jl:146-201, src/wannier_to_bloch_batched.jl:442-455):
//    one CTA per q stages g(q), ukq(q), uph(q) in shared memory and forms
//    T = ukq^dagger g (contract iw) and ep = T uph (contract jm), folding g2 = |ep|^2/(2 omega)
//    into the same pass. No size gate: the reference switches to two cuBLAS strided-batched
//    GEMMs above nw*nm = 24 (wannier_to_bloch_batched.jl:406); this kernel covers all sizes.
#include <algorithm>

#include "epb_common.cuh"

namespace epb {

int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                const double* xk, int64_t N, double2* out, int64_t ldo);

// ---------------------------------------------------------------------------------------------
// Generic FP64 complex GEMM C (M x N) = A (M x K, ld lda) * B (K x N, ld ldb), column-major.
constexpr int G_BM = 64, G_BN = 64, G_BK = 8, G_THREADS = 256;

__global__ void __launch_bounds__(G_THREADS, 2)
zgemm_nn_kernel(const double2* __restrict__ A, int64_t lda, const double2* __restrict__ B,
                int64_t ldb, double2* __restrict__ C, int64_t ldc, int64_t M, int64_t N, int64_t K) {
  __shared__ __align__(16) double2 As[2][G_BK][G_BM];
  __shared__ __align__(16) double2 Bs[2][G_BK][G_BN];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ty = 4 * (warp & 3) + (lane >> 3);
  const int tx = 8 * (warp >> 2) + (lane & 7);
  const int64_t m0 = (int64_t)blockIdx.y * G_BM, n0 = (int64_t)blockIdx.x * G_BN;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0, 0);
  const int64_t kt_n = (K + G_BK - 1) / G_BK;
  auto load = [&](int64_t kt, int buf) {
    int64_t k0 = kt * G_BK;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      int e = tid + t * G_THREADS;
      int mm = e % G_BM, kk = e / G_BM;
      int64_t row = m0 + mm, k = k0 + kk;
      As[buf][kk][mm] = (row < M && k < K) ? A[row + k * lda] : make_double2(0, 0);
      int kb = e % G_BK, jj = e / G_BK;
      int64_t col = n0 + jj, k2 = k0 + kb;
      Bs[buf][kb][jj] = (col < N && k2 < K) ? B[k2 + col * ldb] : make_double2(0, 0);
    }
  };
  load(0, 0);
  __syncthreads();
  for (int64_t kt = 0; kt < kt_n; ++kt) {
    int buf = kt & 1;
    if (kt + 1 < kt_n) load(kt + 1, buf ^ 1);
#pragma unroll
    for (int kk = 0; kk < G_BK; ++kk) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[buf][kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[buf][kk][tx * 4 + j];
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
    if (col >= N) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int64_t row = m0 + ty * 4 + i;
      if (row < M) C[row + col * ldc] = acc[i][j];
    }
  }
}

int zgemm_nn(epb_ctx* ctx, const double2* A, int64_t lda, const double2* B, int64_t ldb, double2* C,
             int64_t ldc, int64_t M, int64_t N, int64_t K) {
  if (M == 0 || N == 0) return EPB_OK;
  dim3 grid((unsigned)cdiv(N, G_BN), (unsigned)cdiv(M, G_BM));
  EPB_CHECK_ARG(grid.y <= 65535, "zgemm: M=%lld too large for one launch", (long long)M);
  prof_begin(ctx, EPB_PROF_ZGEMM);
  zgemm_nn_kernel<<<grid, G_THREADS, 0, ctx->stream>>>(A, lda, B, ldb, C, ldc, M, N, K);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// ---------------------------------------------------------------------------------------------
// Strided-batched FP64 complex GEMM C_b = op(A_b) op(B_b) (alpha = 1, beta = 0) with op in {N, T, C}
// (0, 1, 2), the operation of batched_gemm! (src/common/gpu_utils.jl:71-78): 32 x 32 output tiles,
// 16-deep K steps staged in shared memory with each operand read along its contiguous axis, 2 x 2
// outputs per thread, grid.z strides over the batch.
constexpr int BG_BM = 32, BG_BN = 32, BG_BK = 16, BG_THREADS = 256;

template <int OPA, int OPB>
__global__ void __launch_bounds__(BG_THREADS) zgemm_batched_kernel(
    const double2* __restrict__ A, int64_t lda, int64_t sa, const double2* __restrict__ B, int64_t ldb, int64_t sb,
    double2* __restrict__ C, int64_t ldc, int64_t sc, int64_t M, int64_t N, int64_t K, int64_t batch) {
  __shared__ double2 As[BG_BK][BG_BM + 1];
  __shared__ double2 Bs[BG_BK][BG_BN + 1];
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;  // rows 2 ty, 2 ty + 1; columns 2 tx, 2 tx + 1
  const int64_t m0 = (int64_t)blockIdx.y * BG_BM, n0 = (int64_t)blockIdx.x * BG_BN;
  for (int64_t b = blockIdx.z; b < batch; b += gridDim.z) {
    const double2* Ab = A + b * sa;
    const double2* Bb = B + b * sb;
    double2 acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) acc[i][j] = make_double2(0.0, 0.0);
    for (int64_t k0 = 0; k0 < K; k0 += BG_BK) {
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int e = tid + t * BG_THREADS;
        // A tile (m, k): read along m for 'N', along k for 'T' / 'C'
        const int am = OPA == 0 ? e % BG_BM : e / BG_BK, ak = OPA == 0 ? e / BG_BM : e % BG_BK;
        const int64_t row = m0 + am, kk = k0 + ak;
        double2 av = make_double2(0.0, 0.0);
        if (row < M && kk < K) {
          av = OPA == 0 ? Ab[row + kk * lda] : Ab[kk + row * lda];
          if (OPA == 2) av.y = -av.y;
        }
        As[ak][am] = av;
        // B tile (k, n): read along k for 'N', along n for 'T' / 'C'
        const int bk = OPB == 0 ? e % BG_BK : e / BG_BN, bn = OPB == 0 ? e / BG_BK : e % BG_BN;
        const int64_t col = n0 + bn, kb = k0 + bk;
        double2 bv = make_double2(0.0, 0.0);
        if (col < N && kb < K) {
          bv = OPB == 0 ? Bb[kb + col * ldb] : Bb[col + kb * ldb];
          if (OPB == 2) bv.y = -bv.y;
        }
        Bs[bk][bn] = bv;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BG_BK; ++kk) {
        const double2 a0 = As[kk][2 * ty], a1 = As[kk][2 * ty + 1];
        const double2 b0 = Bs[kk][2 * tx], b1 = Bs[kk][2 * tx + 1];
        cfma(acc[0][0], a0, b0);
        cfma(acc[0][1], a0, b1);
        cfma(acc[1][0], a1, b0);
        cfma(acc[1][1], a1, b1);
      }
      __syncthreads();
    }
    double2* Cb = C + b * sc;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int64_t row = m0 + 2 * ty + i, col = n0 + 2 * tx + j;
        if (row < M && col < N) Cb[row + col * ldc] = acc[i][j];
      }
  }
}

template <int OPA>
static void launch_zgemm_batched(int opb, dim3 grid, cudaStream_t s, const double2* A, int64_t lda, int64_t sa,
                                 const double2* B, int64_t ldb, int64_t sb, double2* C, int64_t ldc, int64_t sc,
                                 int64_t M, int64_t N, int64_t K, int64_t batch) {
  if (opb == 0)
    zgemm_batched_kernel<OPA, 0><<<grid, BG_THREADS, 0, s>>>(A, lda, sa, B, ldb, sb, C, ldc, sc, M, N, K, batch);
  else if (opb == 1)
    zgemm_batched_kernel<OPA, 1><<<grid, BG_THREADS, 0, s>>>(A, lda, sa, B, ldb, sb, C, ldc, sc, M, N, K, batch);
  else
    zgemm_batched_kernel<OPA, 2><<<grid, BG_THREADS, 0, s>>>(A, lda, sa, B, ldb, sb, C, ldc, sc, M, N, K, batch);
}

// ---------------------------------------------------------------------------------------------
// RR->kR rotation: out[iw, n, mp, k] = sum_jw g[iw, jw, mp, k] uk[jw, n, k] * ph[p, k]
// g: (nw, nw, M, kc) with mp in [0, M = nm*nr_ep), p = mp / nm.
__global__ void rr_rotate_kernel(const double2* __restrict__ g, const double2* __restrict__ uk,
                                 const double2* __restrict__ ph, double2* __restrict__ out,
                                 int nw, int nband, int nm, int nr_ep, int64_t kc) {
  const int64_t M = (int64_t)nm * nr_ep;
  const int64_t total = (int64_t)nw * nband * M * kc;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int iw = (int)(idx % nw);
    int64_t r = idx / nw;
    int n = (int)(r % nband);
    r /= nband;
    int64_t mp = r % M;
    int64_t k = r / M;
    const double2* gb = g + ((k * M + mp) * nw) * nw;
    const double2* ub = uk + (k * nband + n) * nw;
    double2 acc = make_double2(0, 0);
    for (int jw = 0; jw < nw; ++jw) cfma(acc, gb[iw + jw * nw], ub[jw]);
    if (ph) {
      int p = (int)(mp / nm);
      acc = cmul(acc, ph[p + k * nr_ep]);
    }
    out[idx] = acc;
  }
}

// ---------------------------------------------------------------------------------------------
// Rotations: ep[m, n, nu, q] = sum_{iw, jm} conj(ukq[iw, m, q]) g[iw, n, jm, q] uph[jm, nu, q].
// One CTA per q. Shared: g (nw*nbk*nm), T (nbkq*nbk*nm), ukq (nw*nbkq), uph (nm*nm).
__device__ __forceinline__ double2 rot_ld(double2 v) { return v; }
__device__ __forceinline__ double2 rot_ld(float2 v) { return make_double2(v.x, v.y); }

// G = double2, or float2 for a complex64 g (the tensor-core kR->kq output), widened on load.
template <typename G>
__global__ void eph_rot_kernel(const G* __restrict__ g, int64_t ldg, const double2* __restrict__ ukq,
                               const double2* __restrict__ uph, const double* __restrict__ omega,
                               double2* __restrict__ ep, double* __restrict__ g2, int nw, int nbk,
                               int nm, int nbkq, int64_t nq) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ng = nw * nbk * nm, nt = nbkq * nbk * nm;
  double2* gs = reinterpret_cast<double2*>(smem_raw);
  double2* ts = gs + ng;
  double2* us = ts + nt;
  double2* ps = us + nw * nbkq;
  for (int64_t q = blockIdx.x; q < nq; q += gridDim.x) {
    const G* gq = g + q * ldg;
    for (int e = threadIdx.x; e < ng; e += blockDim.x) gs[e] = rot_ld(gq[e]);
    for (int e = threadIdx.x; e < nw * nbkq; e += blockDim.x) us[e] = ukq[q * nw * nbkq + e];
    for (int e = threadIdx.x; e < nm * nm; e += blockDim.x) ps[e] = uph[q * nm * nm + e];
    __syncthreads();
    // T[m, n, jm] = sum_iw conj(ukq[iw, m]) g[iw, n, jm]
    for (int e = threadIdx.x; e < nt; e += blockDim.x) {
      int m = e % nbkq, r = e / nbkq;  // r = n + nbk*jm
      double2 acc = make_double2(0, 0);
      const double2* gc = gs + r * nw;
      const double2* uc = us + m * nw;
      for (int iw = 0; iw < nw; ++iw) cfma_conj(acc, uc[iw], gc[iw]);
      ts[e] = acc;
    }
    __syncthreads();
    // ep[m, n, nu] = sum_jm T[m, n, jm] uph[jm, nu]
    const int mn = nbkq * nbk;
    for (int e = threadIdx.x; e < nt; e += blockDim.x) {
      int mnidx = e % mn, nu = e / mn;
      double2 acc = make_double2(0, 0);
      for (int jm = 0; jm < nm; ++jm) cfma(acc, ts[mnidx + jm * mn], ps[jm + nu * nm]);
      int64_t o = q * nt + e;
      if (ep) ep[o] = acc;
      if (g2) g2[o] = (acc.x * acc.x + acc.y * acc.y) / (2.0 * omega[nu + q * nm]);
    }
    __syncthreads();
  }
}

template <typename G>
static int eph_rotations_t(epb_ctx* ctx, const G* g, int64_t ldg, int nw, int nbk, int nm, int64_t nq,
                           const double2* ukq, int nbkq, const double2* uph, const double* omega, double2* ep,
                           double* g2) {
  if (nq == 0) return EPB_OK;
  size_t smem = sizeof(double2) * ((size_t)nw * nbk * nm + (size_t)nbkq * nbk * nm + nw * nbkq + nm * nm);
  EPB_CHECK_ARG(smem <= 200 * 1024, "eph rotations: block (nw=%d, nbk=%d, nm=%d) exceeds shared memory",
                nw, nbk, nm);
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(eph_rot_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  int64_t blocks = nq < (int64_t)ctx->sm_count * 8 ? nq : (int64_t)ctx->sm_count * 8;
  prof_begin(ctx, EPB_PROF_ROT);
  eph_rot_kernel<G><<<(unsigned)blocks, 256, smem, ctx->stream>>>(g, ldg, ukq, uph, omega, ep, g2, nw, nbk, nm,
                                                                   nbkq, nq);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int eph_rotations_f64(epb_ctx* ctx, const double2* g, int64_t ldg, int nw, int nbk, int nm,
                      int64_t nq, const double2* ukq, int nbkq, const double2* uph,
                      const double* omega, double2* ep, double* g2) {
  return eph_rotations_t(ctx, g, ldg, nw, nbk, nm, nq, ukq, nbkq, uph, omega, ep, g2);
}

int eph_rotations_c64(epb_ctx* ctx, const float2* g, int64_t ldg, int nw, int nbk, int nm, int64_t nq,
                      const double2* ukq, int nbkq, const double2* uph, const double* omega, double2* ep,
                      double* g2) {
  return eph_rotations_t(ctx, g, ldg, nw, nbk, nm, nq, ukq, nbkq, uph, omega, ep, g2);
}

}  // namespace epb

using namespace epb;

extern "C" {

static int op_code(char t) { return t == 'N' || t == 'n' ? 0 : t == 'T' || t == 't' ? 1 : t == 'C' || t == 'c' ? 2 : -1; }

int epb_batched_zgemm(epb_ctx* ctx, char transA, char transB, int64_t m, int64_t n, int64_t k, const double* A,
                      int64_t lda, int64_t strideA, const double* B, int64_t ldb, int64_t strideB, double* C,
                      int64_t ldc, int64_t strideC, int64_t batch) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_batched_zgemm: NULL ctx");
  const int oa = op_code(transA), ob = op_code(transB);
  EPB_CHECK_ARG(oa >= 0 && ob >= 0, "epb_batched_zgemm: trans must be 'N', 'T' or 'C'");
  EPB_CHECK_ARG(m >= 0 && n >= 0 && k >= 0 && batch >= 0, "epb_batched_zgemm: negative size");
  if (m == 0 || n == 0 || batch == 0) return EPB_OK;
  EPB_CHECK_ARG(C && (k == 0 || (A && B)), "epb_batched_zgemm: NULL buffer");
  EPB_CHECK_ARG(lda >= std::max<int64_t>(1, oa == 0 ? m : k) && ldb >= std::max<int64_t>(1, ob == 0 ? k : n) &&
                    ldc >= m,
                "epb_batched_zgemm: leading dimension too small (lda=%lld ldb=%lld ldc=%lld)", (long long)lda,
                (long long)ldb, (long long)ldc);
  EPB_CHECK_ARG(cdiv(m, BG_BM) <= 65535, "epb_batched_zgemm: m=%lld too large", (long long)m);
  EPB_TRY(make_current(ctx));
  dim3 grid((unsigned)cdiv(n, BG_BN), (unsigned)cdiv(m, BG_BM),
            (unsigned)std::min<int64_t>(batch, 65535));
  const double2 *a = (const double2*)A, *b = (const double2*)B;
  double2* c = (double2*)C;
  prof_begin(ctx, EPB_PROF_ZGEMM);
  if (oa == 0)
    launch_zgemm_batched<0>(ob, grid, ctx->stream, a, lda, strideA, b, ldb, strideB, c, ldc, strideC, m, n, k, batch);
  else if (oa == 1)
    launch_zgemm_batched<1>(ob, grid, ctx->stream, a, lda, strideA, b, ldb, strideB, c, ldc, strideC, m, n, k, batch);
  else
    launch_zgemm_batched<2>(ob, grid, ctx->stream, a, lda, strideA, b, ldb, strideB, c, ldc, strideC, m, n, k, batch);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_eph_RR_to_kR(epb_ctx* ctx, const double* epmat, int64_t nw, int64_t nm, int64_t nr_ep,
                     const epb_rset* rset_el, const double* xk, int64_t nk, const double* uk,
                     int64_t nband, const double* add_phase, double* out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset_el, "epb_eph_RR_to_kR: NULL ctx or rset");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nr_ep >= 1 && nband >= 1 && nband <= nw && nk >= 0,
                "epb_eph_RR_to_kR: bad sizes");
  EPB_CHECK_ARG(nk == 0 || (epmat && xk && uk && out), "epb_eph_RR_to_kR: NULL buffer");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_RR_to_kR: bad prec");
  EPB_TRY(make_current(ctx));
  if (nk == 0) return EPB_OK;
  const int64_t ndata = nw * nw * nm * nr_ep;
  // chunk over k so that the Fourier intermediate stays below ~2 GiB
  int64_t kc = (int64_t)((2ull << 30) / (16ull * ndata));
  if (kc < 1) kc = 1;
  if (kc > nk) kc = nk;
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EPH_G, 16ull * ndata * kc, &ws));
  double2* g = (double2*)ws;
  const int64_t outk = nw * nband * nm * nr_ep;
  for (int64_t k0 = 0; k0 < nk; k0 += kc) {
    int64_t kn = nk - k0 < kc ? nk - k0 : kc;
    EPB_TRY(fourier_f64(ctx, (const double2*)epmat, ndata, ndata, rset_el, xk + 3 * k0, kn, g, ndata));
    int64_t total = outk * kn;
    int64_t blocks = cdiv(total, 256);
    if (blocks > (int64_t)ctx->sm_count * 32) blocks = (int64_t)ctx->sm_count * 32;
    prof_begin(ctx, EPB_PROF_RR_ROT);
    rr_rotate_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(
        g, (const double2*)uk + k0 * nw * nband, add_phase ? (const double2*)add_phase + k0 * nr_ep : nullptr,
        (double2*)out + k0 * outk, (int)nw, (int)nband, (int)nm, (int)nr_ep, kn);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

int epb_eph_apply_rotations(epb_ctx* ctx, const double* g, int64_t ldg, int64_t nw, int64_t nbk,
                            int64_t nm, int64_t nq, const double* ukq, int64_t nbkq,
                            const double* uph, const double* omega, double* ep_out,
                            double* g2_out) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eph_apply_rotations: NULL ctx");
  EPB_CHECK_ARG(nw >= 1 && nbk >= 1 && nm >= 1 && nbkq >= 1 && nq >= 0 && ldg >= nw * nbk * nm,
                "epb_eph_apply_rotations: bad sizes");
  EPB_CHECK_ARG(nq == 0 || (g && ukq && uph), "epb_eph_apply_rotations: NULL input");
  EPB_CHECK_ARG(!g2_out || omega, "epb_eph_apply_rotations: g2_out requires omega");
  EPB_TRY(make_current(ctx));
  return eph_rotations_f64(ctx, (const double2*)g, ldg, (int)nw, (int)nbk, (int)nm, nq,
                           (const double2*)ukq, (int)nbkq, (const double2*)uph, omega,
                           (double2*)ep_out, g2_out);
}

int epb_eph_kR_to_kq(epb_ctx* ctx, const double* ep_kR, int64_t ld, int64_t nw, int64_t nbk,
                     int64_t nm, int64_t nr_ep, const double* phase, int64_t nq,
                     const double* ukq, int64_t nbkq, const double* uph, const double* omega,
                     double* ep_out, double* g2_out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eph_kR_to_kq: NULL ctx");
  const int64_t ndata = nw * nbk * nm;
  EPB_CHECK_ARG(nw >= 1 && nbk >= 1 && nm >= 1 && nbkq >= 1 && nr_ep >= 1 && nq >= 0 && ld >= ndata,
                "epb_eph_kR_to_kq: bad sizes");
  EPB_CHECK_ARG(nq == 0 || (ep_kR && phase && ukq && uph), "epb_eph_kR_to_kq: NULL input");
  EPB_CHECK_ARG(!g2_out || omega, "epb_eph_kR_to_kq: g2_out requires omega");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_kR_to_kq: bad prec");
  EPB_TRY(make_current(ctx));
  if (nq == 0) return EPB_OK;
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EPH_T, 16ull * ndata * nq, &ws));
  double2* g = (double2*)ws;
  EPB_TRY(zgemm_nn(ctx, (const double2*)ep_kR, ld, (const double2*)phase, nr_ep, g, ndata, ndata, nq, nr_ep));
  return eph_rotations_f64(ctx, g, ndata, (int)nw, (int)nbk, (int)nm, nq, (const double2*)ukq,
                           (int)nbkq, (const double2*)uph, omega, (double2*)ep_out, g2_out);
}

}  // extern "C"
