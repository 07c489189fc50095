// Outer-q e-ph loop: g(Re, q) = sum_Rp e^{2 pi i q.Rp} g(Re, Rp) rotated into the phonon eigenmode basis
// (get_eph_RR_to_Rq!, src/wannier_to_bloch.jl:277-300), then for a list of k
// g(k, q) = sum_Re e^{2 pi i k.Re} g(Re, q) and ep[m, n, nu, k] = sum_{iw, jw} conj(ukq[iw, m, k])
// g[iw, jw, nu, k] uk[jw, n, k] (get_eph_Rq_to_kq_batched! / eph_apply_rotations_rqkq!,
// src/wannier_to_bloch_batched.jl:317-377, fused CUDA method ext/ElectronPhononCUDAExt.jl:206-258),
// plus the conversion of the e-ph matrix from the "el" layout (rows (i, j, nu, Rp), columns Re) to
// the "ph" layout (rows (i, j, nu, Re), columns Rp) (src/model.jl:80-81,293-296, src/model_new.jl:551-565).
#include <algorithm>
#include <type_traits>

#include "epb_common.cuh"

namespace epb {

int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* xk,
                int64_t N, double2* out, int64_t ldo);
int fourier_mixed(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* xk,
                  int64_t N, double2* out, int64_t ldo);
int eigh_async(epb_ctx* ctx, double2* A, int64_t n, int64_t batch, double* E, bool want_v, const double* mass,
               int prec);
int eigh_check(epb_ctx* ctx);
int split_gemm_check(epb_ctx* ctx);
int64_t oq_a_bytes(int64_t M, int64_t K);
int64_t oq_b_bytes(int64_t N, int64_t K);
int oq_pack_a(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, int64_t K, uint8_t* mem);
int oq_pack_b(epb_ctx* ctx, const epb_rset* rs, const double* x, int64_t N, uint8_t* mem);
int oq_gemm(epb_ctx* ctx, int prof_id, const uint8_t* a_mem, int64_t M, int64_t K, const uint8_t* b_mem, int64_t N,
            int64_t n0, int64_t nn, float2* C, int64_t ldc);
int window_filter(epb_ctx* ctx, const double* E, int64_t nw, int64_t nk, double wmin, double wmax, int32_t* bmin,
                  int32_t* bmax, int32_t* keep_idx, int64_t* nkeep, double* nbelow);

// FP64 Fourier sum over row blocks of at most 2^20 rows (one launch's grid limit is far above that).
static int fourier_rows(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* x,
                        int64_t N, double2* out, int64_t ldo) {
  const int64_t RB = (int64_t)1 << 20;
  for (int64_t r0 = 0; r0 < M; r0 += RB)
    EPB_TRY(fourier_f64(ctx, op + r0, ld, std::min(RB, M - r0), rs, x, N, out + r0, ldo));
  return EPB_OK;
}

static unsigned grid_oq(epb_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)ctx->sm_count * 32));
}

// out[b, ir, q] (b = (i, j) pair, ir = Re) with the mode index rotated:
// out[(ij, nu), ir, q] = sum_mu g[(ij, mu), ir, q] uph[mu, nu, q].
__device__ __forceinline__ double2 as_c128(double2 v) { return v; }
__device__ __forceinline__ double2 as_c128(float2 v) { return make_double2(v.x, v.y); }

template <typename G>
__global__ void rq_mode_rotate_kernel(const G* __restrict__ g, const double2* __restrict__ uph, int64_t nb,
                                      int64_t nm, int64_t nr, int64_t nq, double2* __restrict__ out) {
  const int64_t total = nb * nm * nr * nq;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e % nb, nu = (e / nb) % nm, rq = e / (nb * nm);  // rq = ir + nr q
    const int64_t q = rq / nr;
    const G* gp = g + rq * nb * nm + b;
    const double2* up = uph + q * nm * nm + nu * nm;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t mu = 0; mu < nm; ++mu) cfma(acc, as_c128(gp[mu * nb]), up[mu]);
    out[e] = acc;
  }
}

// One thread per (m, n, k): ep[m, n, nu, k] for all nu; g2 = |ep|^2 / (2 omega_nu) when requested.
__global__ void rqkq_rot_kernel(const double2* __restrict__ g, const double2* __restrict__ uks,
                                const double2* __restrict__ ukqs, const double* __restrict__ omega,
                                double2* __restrict__ ep, double* __restrict__ g2, int nw, int nbkq, int nbk, int nm,
                                int64_t nk) {
  const int64_t total = (int64_t)nbkq * nbk * nk;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(t % nbkq);
    const int n = (int)((t / nbkq) % nbk);
    const int64_t k = t / ((int64_t)nbkq * nbk);
    const double2* uq = ukqs + (k * nbkq + m) * nw;
    const double2* uk = uks + (k * nbk + n) * nw;
    for (int nu = 0; nu < nm; ++nu) {
      const double2* gk = g + ((k * nm + nu) * nw) * nw;
      double2 acc = make_double2(0.0, 0.0);
      for (int jw = 0; jw < nw; ++jw) {
        double2 tv = make_double2(0.0, 0.0);
        for (int iw = 0; iw < nw; ++iw) cfma_conj(tv, uq[iw], gk[iw + jw * nw]);
        cfma(acc, tv, uk[jw]);
      }
      const int64_t o = m + (int64_t)nbkq * (n + (int64_t)nbk * (nu + (int64_t)nm * k));
      if (ep) ep[o] = acc;
      if (g2) g2[o] = (acc.x * acc.x + acc.y * acc.y) / (2.0 * omega[nu]);
    }
  }
}

// "el" layout (nb nr_ep rows, nr_el columns) -> "ph" layout (nb nr_el rows, nr_ep columns), nb = nw^2 nm.
__global__ void epmat_el_to_ph_kernel(const double2* __restrict__ in, int64_t nb, int64_t nr_el, int64_t nr_ep,
                                      double2* __restrict__ out) {
  const int64_t total = nb * nr_el * nr_ep;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e % nb, re = (e / nb) % nr_el, rp = e / (nb * nr_el);  // out element (b, re, rp)
    out[e] = in[b + nb * (rp + nr_ep * re)];
  }
}


// ---- outer-q driver kernels -------------------------------------------------------------------
// Kept k (keep list from the window filter): positions, weights, energies, and eigenvectors with the
// columns outside the k window [bmin, bmax] (1-based) set to zero.
__global__ void oq_gather_k_kernel(const int32_t* __restrict__ keep, const int64_t* __restrict__ nkeep_d,
                                   const double* __restrict__ xk, const double* __restrict__ wtk,
                                   const double* __restrict__ E, const double2* __restrict__ U,
                                   const int32_t* __restrict__ bmin, const int32_t* __restrict__ bmax, int nw,
                                   double* __restrict__ xo, double* __restrict__ wo, double* __restrict__ Eo,
                                   double2* __restrict__ Uo) {
  const int64_t nkeep = *nkeep_d;
  const int64_t nw2 = (int64_t)nw * nw;
  const int64_t total = nkeep * nw2;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / nw2, r = e % nw2;
    const int64_t k = keep[j];
    const int col = (int)(r / nw) + 1;
    Uo[e] = (col >= bmin[k] && col <= bmax[k]) ? U[k * nw2 + r] : make_double2(0.0, 0.0);
    if (r < nw) Eo[j * nw + r] = E[k * nw + r];
    if (r < 3) xo[3 * j + r] = xk[3 * k + r];
    if (r == 0) wo[j] = wtk ? wtk[k] : 1.0;
  }
}

__global__ void oq_shift_kernel(const double* __restrict__ xk, int64_t nk, const double* __restrict__ xq,
                                double* __restrict__ xkq) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 3 * nk; e += (int64_t)gridDim.x * blockDim.x)
    xkq[e] = xk[e] + xq[e % 3];
}

// Zero the eigenvector columns m whose energy lies outside [wmin, wmax] (the k+q window mask of
// src/calculator/run_eph_over_q_and_k.jl:577-580).
__global__ void oq_mask_kernel(double2* __restrict__ U, const double* __restrict__ E, int nw, int64_t nk, double wmin,
                               double wmax) {
  const int64_t nw2 = (int64_t)nw * nw;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nk * nw2; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / nw2;
    const int m = (int)((e % nw2) / nw);
    const double v = E[k * nw + m];
    if (!(v >= wmin && v <= wmax)) U[e] = make_double2(0.0, 0.0);
  }
}

__global__ void oq_widen_kernel(const float2* __restrict__ in, int64_t n, double2* __restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = make_double2(in[e].x, in[e].y);
}

__global__ void oq_identity_kernel(double2* __restrict__ u, int nm, int64_t nq) {
  const int64_t nm2 = (int64_t)nm * nm;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nq * nm2; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % nm2;
    u[e] = make_double2((r % nm) == (r / nm) ? 1.0 : 0.0, 0.0);
  }
}

// One block per k: ep[m, n, nu] = sum_{iw, jw} conj(ukq[iw, m]) g[iw, jw, nu] uk[jw, n] through shared
// memory (T[m, jw] = sum_iw conj(ukq[iw, m]) g[iw, jw, nu], then T uk), and part[k] = wtk[k] sum |ep|^2.
// Shared memory: four nw x (nw + 1) complex tiles (conj(ukq)^T, uk, g_nu, T).
constexpr int OQ_ROT_THREADS = 256;
template <bool STORE>
__global__ void __launch_bounds__(OQ_ROT_THREADS) oq_rot_kernel(const double2* __restrict__ g, const double2* __restrict__ uk,
                                                              const double2* __restrict__ ukq, const double* __restrict__ wtk,
                                                              int nw, int nm, int64_t nk, double2* __restrict__ ep,
                                                              double* __restrict__ part) {
  extern __shared__ double2 oq_sm[];
  const int L = nw + 1, nw2 = nw * nw;
  double2* sq = oq_sm;         // sq[m * L + iw] = conj(ukq[iw, m])
  double2* sk = sq + nw * L;   // sk[n * L + jw] = uk[jw, n]
  double2* sg = sk + nw * L;   // sg[jw * L + iw] = g[iw, jw, nu]
  double2* st = sg + nw * L;   // st[jw * L + m] = T[m, jw]
  __shared__ double red[OQ_ROT_THREADS / 32];
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    __syncthreads();
    const double2* uq = ukq + k * nw2;
    const double2* ukk = uk + k * nw2;
    for (int e = threadIdx.x; e < nw2; e += blockDim.x) {
      const int i = e % nw, c = e / nw;
      const double2 a = uq[e];
      sq[c * L + i] = make_double2(a.x, -a.y);
      sk[c * L + i] = ukk[e];
    }
    double acc2 = 0.0;
    for (int nu = 0; nu < nm; ++nu) {
      const double2* gk = g + (k * nm + nu) * nw2;
      for (int e = threadIdx.x; e < nw2; e += blockDim.x) sg[(e / nw) * L + (e % nw)] = gk[e];
      __syncthreads();
      for (int e = threadIdx.x; e < nw2; e += blockDim.x) {
        const int m = e % nw, jw = e / nw;
        const double2* a = sq + m * L;
        const double2* b = sg + jw * L;
        double2 t = make_double2(0.0, 0.0);
        for (int iw = 0; iw < nw; ++iw) cfma(t, a[iw], b[iw]);
        st[jw * L + m] = t;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < nw2; e += blockDim.x) {
        const int m = e % nw, n = e / nw;
        const double2* b = sk + n * L;
        double2 v = make_double2(0.0, 0.0);
        for (int jw = 0; jw < nw; ++jw) cfma(v, st[jw * L + m], b[jw]);
        if (STORE) ep[(k * nm + nu) * nw2 + e] = v;
        acc2 += v.x * v.x + v.y * v.y;
      }
      __syncthreads();
    }
    if (part) {
      for (int o = 16; o > 0; o >>= 1) acc2 += __shfl_xor_sync(0xffffffffu, acc2, o);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc2;
      __syncthreads();
      if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        part[k] = wtk[k] * s;
      }
    }
  }
}

// nw <= 16: the whole g(k) block (nm x nw columns of nw, padded to nw + 1) is staged once; thread (m, jw)
// forms T[m, jw, nu] = sum_iw conj(ukq[iw, m]) g[iw, jw, nu] for OQ_NC modes at a time in registers and,
// after a barrier, writes T over the g columns it came from (only threads of the same column read them);
// then thread (m, n) forms ep[m, n, nu] = sum_jw T[m, jw, nu] uk[jw, n] for every nu. One global read of
// g(k), no per-mode round trips. Same outputs as oq_rot_kernel.
constexpr int OQ_NC = 4;
template <typename C> __device__ __forceinline__ C to_c(double2 v);
template <> __device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 to_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <typename C> __device__ __forceinline__ C to_c(float2 v);
template <> __device__ __forceinline__ double2 to_c<double2>(float2 v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ float2 to_c<float2>(float2 v) { return v; }

// C = double2: FP64 throughout; C = float2: FP32 arithmetic (the mixed mode, whose g(k, q) is FP32-level).
template <bool STORE, typename G, typename C>
__global__ void __launch_bounds__(OQ_ROT_THREADS, sizeof(C) == 8 ? 4 : 2) oq_rot_block_kernel(
    const G* __restrict__ g, const double2* __restrict__ uk, const double2* __restrict__ ukq,
    const double* __restrict__ wtk, int nw, int nm, int64_t nk, double2* __restrict__ ep, double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char oq_smb[];
  C* oq_sm = reinterpret_cast<C*>(oq_smb);
  const int L = nw + 1, nw2 = nw * nw, ncol = nm * nw;
  C* sq = oq_sm;        // sq[m * L + iw] = conj(ukq[iw, m])
  C* sk = sq + nw * L;  // sk[n * L + jw] = uk[jw, n]
  C* sg = sk + nw * L;  // sg[(nu * nw + jw) * L + iw] = g[iw, jw, nu], later T[iw := m]
  __shared__ double red[OQ_ROT_THREADS / 32];
  const int t = threadIdx.x;
  const int m = t % nw, c = t / nw;  // (m, jw) in the T stage, (m, n) in the ep stage
  const bool act = t < nw2;
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    const double2* uq = ukq + k * nw2;
    const double2* ukk = uk + k * nw2;
    const G* gk = g + k * (int64_t)nw2 * nm;
    for (int e = t; e < nw2; e += blockDim.x) {
      const int i = e % nw, j = e / nw;
      const double2 a = uq[e];
      sq[j * L + i] = to_c<C>(make_double2(a.x, -a.y));
      sk[j * L + i] = to_c<C>(ukk[e]);
    }
    for (int e = t; e < ncol * nw; e += blockDim.x) sg[(e / nw) * L + (e % nw)] = to_c<C>(gk[e]);
    __syncthreads();
    for (int nu0 = 0; nu0 < nm; nu0 += OQ_NC) {
      C tv[OQ_NC];
#pragma unroll
      for (int r = 0; r < OQ_NC; ++r) tv[r] = to_c<C>(make_double2(0.0, 0.0));
      if (act) {
        const C* a = sq + m * L;
        for (int iw = 0; iw < nw; ++iw) {
          const C av = a[iw];
#pragma unroll
          for (int r = 0; r < OQ_NC; ++r)
            if (nu0 + r < nm) cfma(tv[r], av, sg[((nu0 + r) * nw + c) * L + iw]);
        }
      }
      __syncthreads();
      if (act) {
#pragma unroll
        for (int r = 0; r < OQ_NC; ++r)
          if (nu0 + r < nm) sg[((nu0 + r) * nw + c) * L + m] = tv[r];
      }
    }
    __syncthreads();
    double acc2 = 0.0;
    if (act) {
      const C* b = sk + c * L;
      for (int nu = 0; nu < nm; ++nu) {
        const C* tc = sg + (nu * nw) * L + m;
        C v = to_c<C>(make_double2(0.0, 0.0));
        for (int jw = 0; jw < nw; ++jw) cfma(v, tc[jw * L], b[jw]);
        const double vx = v.x, vy = v.y;
        if (STORE) ep[(k * nm + nu) * nw2 + t] = make_double2(vx, vy);
        acc2 += vx * vx + vy * vy;
      }
    }
    for (int o = 16; o > 0; o >>= 1) acc2 += __shfl_xor_sync(0xffffffffu, acc2, o);
    if ((t & 31) == 0) red[t >> 5] = acc2;
    __syncthreads();
    if (t == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
      part[k] = wtk[k] * s;
    }
  }
}

// A[iq] += sum_k part[k], one block, fixed order (deterministic).
__global__ void oq_record_kernel(const double* __restrict__ part, int64_t nk, double* __restrict__ A) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t k = threadIdx.x; k < nk; k += blockDim.x) s += part[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *A += red[0];
}

static size_t oq_rot_smem(int nw) { return (size_t)4 * nw * (nw + 1) * sizeof(double2); }

// G = float2 (mixed mode): FP32 arithmetic; G = double2: FP64.
template <typename G>
static int oq_rotate(epb_ctx* ctx, const G* g, const double2* uk, const double2* ukq, const double* wtk, int nw,
                     int nm, int64_t nk, double2* ep, double* part) {
  if (nw <= 16) {
    using C = G;
    const size_t smb = (size_t)(2 + nm) * nw * (nw + 1) * sizeof(C);
    if (smb > 48 * 1024) {
      EPB_CUDA(cudaFuncSetAttribute(oq_rot_block_kernel<true, G, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb));
      EPB_CUDA(cudaFuncSetAttribute(oq_rot_block_kernel<false, G, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb));
    }
    const int per_sm = sizeof(C) == 8 ? 4 : 2;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nk, (int64_t)ctx->sm_count * per_sm));
    prof_begin(ctx, EPB_PROF_ROT);
    if (ep)
      oq_rot_block_kernel<true, G, C><<<grid, OQ_ROT_THREADS, smb, ctx->stream>>>(g, uk, ukq, wtk, nw, nm, nk, ep, part);
    else
      oq_rot_block_kernel<false, G, C><<<grid, OQ_ROT_THREADS, smb, ctx->stream>>>(g, uk, ukq, wtk, nw, nm, nk, ep, part);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
    return EPB_OK;
  }
  if constexpr (!std::is_same<G, double2>::value) {
    set_error("oq_rotate: complex64 g needs nw <= 16");
    return EPB_ERR_ARG;
  } else {
  const size_t sm = oq_rot_smem(nw);
  if (sm > 48 * 1024) {
    EPB_CUDA(cudaFuncSetAttribute(oq_rot_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    EPB_CUDA(cudaFuncSetAttribute(oq_rot_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  }
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nk, (int64_t)ctx->sm_count * 8));
  prof_begin(ctx, EPB_PROF_ROT);
  if (ep)
    oq_rot_kernel<true><<<grid, OQ_ROT_THREADS, sm, ctx->stream>>>(g, uk, ukq, wtk, nw, nm, nk, ep, part);
  else
    oq_rot_kernel<false><<<grid, OQ_ROT_THREADS, sm, ctx->stream>>>(g, uk, ukq, wtk, nw, nm, nk, ep, part);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
  }
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_epmat_el_to_ph(epb_ctx* ctx, const double* epmat_el, int64_t nw, int64_t nm, int64_t nr_el, int64_t nr_ep,
                       double* epmat_ph) {
  clear_error();
  EPB_CHECK_ARG(ctx && epmat_el && epmat_ph, "epb_epmat_el_to_ph: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nr_el >= 1 && nr_ep >= 1, "epb_epmat_el_to_ph: bad sizes");
  EPB_CHECK_ARG(epmat_el != epmat_ph, "epb_epmat_el_to_ph: in-place conversion is not supported");
  EPB_TRY(make_current(ctx));
  const int64_t nb = nw * nw * nm;
  epmat_el_to_ph_kernel<<<grid_oq(ctx, nb * nr_el * nr_ep), 256, 0, ctx->stream>>>(
      (const double2*)epmat_el, nb, nr_el, nr_ep, (double2*)epmat_ph);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_eph_RR_to_Rq(epb_ctx* ctx, const double* epmat_ph, int64_t nw, int64_t nm, int64_t nr_el,
                     const epb_rset* rset_ph, const double* xq, int64_t nq, const double* uph, double* out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset_ph, "epb_eph_RR_to_Rq: NULL ctx or rset");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nr_el >= 1 && nq >= 0, "epb_eph_RR_to_Rq: bad sizes");
  EPB_CHECK_ARG(nq == 0 || (epmat_ph && xq && uph && out), "epb_eph_RR_to_Rq: NULL buffer");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_RR_to_Rq: bad prec");
  EPB_TRY(make_current(ctx));
  if (nq == 0) return EPB_OK;
  const int64_t nb = nw * nw, ndata = nb * nm * nr_el;
  // chunk over q so that the Fourier intermediate stays below ~2 GiB
  const int64_t qc = std::max<int64_t>(1, std::min<int64_t>(nq, ((int64_t)2 << 30) / (16 * ndata)));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EPH_G, 16 * ndata * qc, &ws));
  double2* g = (double2*)ws;
  for (int64_t q0 = 0; q0 < nq; q0 += qc) {
    const int64_t qn = std::min(qc, nq - q0);
    EPB_TRY(fourier_rows(ctx, (const double2*)epmat_ph, ndata, ndata, rset_ph, xq + 3 * q0, qn, g, ndata));
    prof_begin(ctx, EPB_PROF_RR_ROT);
    rq_mode_rotate_kernel<double2><<<grid_oq(ctx, ndata * qn), 256, 0, ctx->stream>>>(
        g, (const double2*)uph + q0 * nm * nm, nb, nm, nr_el, qn, (double2*)out + q0 * ndata);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

int epb_eph_Rq_to_kq(epb_ctx* ctx, const double* g_Rq, int64_t nw, int64_t nm, const epb_rset* rset_el, const double* xk,
                     int64_t nk, const double* uks, int64_t nbk, const double* ukqs, int64_t nbkq, const double* omega,
                     double* ep_out, double* g2_out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset_el, "epb_eph_Rq_to_kq: NULL ctx or rset");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nk >= 0 && nbk >= 1 && nbk <= nw && nbkq >= 1 && nbkq <= nw,
                "epb_eph_Rq_to_kq: bad sizes");
  EPB_CHECK_ARG(nk == 0 || (g_Rq && xk && uks && ukqs && (ep_out || g2_out)), "epb_eph_Rq_to_kq: NULL buffer");
  EPB_CHECK_ARG(!g2_out || omega, "epb_eph_Rq_to_kq: g2_out requires omega");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_Rq_to_kq: bad prec");
  EPB_TRY(make_current(ctx));
  if (nk == 0) return EPB_OK;
  const int64_t ndata = nw * nw * nm;
  const int64_t kc = std::max<int64_t>(1, std::min<int64_t>(nk, ((int64_t)1 << 30) / (16 * ndata)));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EPH_T, 16 * ndata * kc, &ws));
  double2* g = (double2*)ws;
  for (int64_t k0 = 0; k0 < nk; k0 += kc) {
    const int64_t kn = std::min(kc, nk - k0);
    if (prec == EPB_PREC_MIXED)
      EPB_TRY(fourier_mixed(ctx, (const double2*)g_Rq, ndata, ndata, rset_el, xk + 3 * k0, kn, g, ndata));
    else
      EPB_TRY(fourier_f64(ctx, (const double2*)g_Rq, ndata, ndata, rset_el, xk + 3 * k0, kn, g, ndata));
    const int64_t o = nbkq * nbk * nm * k0;
    prof_begin(ctx, EPB_PROF_ROT);
    rqkq_rot_kernel<<<grid_oq(ctx, nbkq * nbk * kn), 256, 0, ctx->stream>>>(
        g, (const double2*)uks + k0 * nw * nbk, (const double2*)ukqs + k0 * nw * nbkq, omega,
        ep_out ? (double2*)ep_out + o : nullptr, g2_out ? g2_out + o : nullptr, (int)nw, (int)nbkq, (int)nbk, (int)nm, kn);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}


int epb_eph_outer_q(epb_ctx* ctx, epb_model* m, const double* xk_host, const double* wtk_host, int64_t nk,
                    const double* xq_host, int64_t nq, const epb_outer_q_params* prm, const epb_outer_q_calc* calcs,
                    int ncalc, double* A_host, int64_t* stats_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && prm, "epb_eph_outer_q: NULL ctx, model or params");
  EPB_CHECK_ARG(nk >= 0 && nq >= 0 && ncalc >= 0, "epb_eph_outer_q: bad sizes");
  EPB_CHECK_ARG((nk == 0 || xk_host) && (nq == 0 || xq_host) && (ncalc == 0 || calcs),
                "epb_eph_outer_q: NULL buffer");
  EPB_CHECK_ARG(prm->prec == EPB_PREC_FP64 || prm->prec == EPB_PREC_MIXED, "epb_eph_outer_q: bad prec");
  EPB_CHECK_ARG(prm->phonon_basis == 0 || prm->phonon_basis == 1, "epb_eph_outer_q: phonon_basis must be 0 or 1");
  for (int c = 0; c < ncalc; ++c)
    EPB_CHECK_ARG(calcs[c].run_batch, "epb_eph_outer_q: calculator %d has no run_batch", c);
  EPB_TRY(make_current(ctx));
  const int nw = (int)m->nw, nm = (int)m->nm;
  const int64_t nw2 = (int64_t)nw * nw, nd = nw2 * nm, nr_el = m->nr_el;
  const int prec = prm->prec;
  if (stats_host)
    for (int i = 0; i < 4; ++i) stats_host[i] = 0;
  if (A_host)
    for (int64_t i = 0; i < nq; ++i) A_host[i] = 0.0;
  if (nq == 0) return EPB_OK;

  // "ph"-layout epmat, made once per model
  if (!m->epmat_ph) {
    EPB_CUDA(cudaMalloc(&m->epmat_ph, (size_t)16 * nd * m->nr_ep * nr_el));
    epmat_el_to_ph_kernel<<<grid_oq(ctx, nd * nr_el * m->nr_ep), 256, 0, ctx->stream>>>(m->epmat, nd, nr_el, m->nr_ep,
                                                                                      m->epmat_ph);
    EPB_LAUNCH_CHECK();
  }

  // ---- k and q states (whole run) ----
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const int64_t nk1 = std::max<int64_t>(nk, 1);
  const size_t o_xk = take(24 * nk1), o_wk = take(8 * nk1), o_U = take(16 * nw2 * nk1), o_E = take(8 * nw * nk1),
               o_bmin = take(4 * nk1), o_bmax = take(4 * nk1), o_keep = take(4 * nk1), o_nkeep = take(64),
               o_xkk = take(24 * nk1), o_wkk = take(8 * nk1), o_Uk = take(16 * nw2 * nk1), o_Ek = take(8 * nw * nk1),
               o_xq = take(24 * nq), o_uph = take(16 * (int64_t)nm * nm * nq), o_om = take(8 * (int64_t)nm * nq),
               o_A = take(8 * nq);
  void* ws0 = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_OQ0, off + 256, &ws0));
  uint8_t* b0 = (uint8_t*)ws0;
  double* xk_d = (double*)(b0 + o_xk);
  double* wk_d = (double*)(b0 + o_wk);
  double2* U_all = (double2*)(b0 + o_U);
  double* E_all = (double*)(b0 + o_E);
  int32_t* bmin = (int32_t*)(b0 + o_bmin);
  int32_t* bmax = (int32_t*)(b0 + o_bmax);
  int32_t* keep = (int32_t*)(b0 + o_keep);
  int64_t* nkeep_d = (int64_t*)(b0 + o_nkeep);
  double* xkk = (double*)(b0 + o_xkk);
  double* wkk = (double*)(b0 + o_wkk);
  double2* Uk = (double2*)(b0 + o_Uk);
  double* Ek = (double*)(b0 + o_Ek);
  double* xq_d = (double*)(b0 + o_xq);
  double2* uph = (double2*)(b0 + o_uph);
  double* om = (double*)(b0 + o_om);
  double* A_d = (double*)(b0 + o_A);

  if (nk > 0) {
    EPB_CUDA(cudaMemcpyAsync(xk_d, xk_host, 24 * nk, cudaMemcpyHostToDevice, ctx->stream));
    if (wtk_host) EPB_CUDA(cudaMemcpyAsync(wk_d, wtk_host, 8 * nk, cudaMemcpyHostToDevice, ctx->stream));
  }
  EPB_CUDA(cudaMemcpyAsync(xq_d, xq_host, 24 * nq, cudaMemcpyHostToDevice, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(A_d, 0, 8 * nq, ctx->stream));
  const int64_t HC = 65536;
  for (int64_t k0 = 0; k0 < nk; k0 += HC) {
    const int64_t kn = std::min(HC, nk - k0);
    EPB_TRY(fourier_f64(ctx, m->ham, nw2, nw2, m->rs_el, xk_d + 3 * k0, kn, U_all + k0 * nw2, nw2));
    EPB_TRY(eigh_async(ctx, U_all + k0 * nw2, nw, kn, E_all + k0 * nw, true, nullptr, prec));
  }
  EPB_TRY(window_filter(ctx, E_all, nw, nk, prm->wmin_k, prm->wmax_k, bmin, bmax, keep, nkeep_d, nullptr));
  if (nk > 0) {
    oq_gather_k_kernel<<<grid_oq(ctx, nk * nw2), 256, 0, ctx->stream>>>(keep, nkeep_d, xk_d, wtk_host ? wk_d : nullptr,
                                                                        E_all, U_all, bmin, bmax, nw, xkk, wkk, Ek, Uk);
    EPB_LAUNCH_CHECK();
  }
  const int64_t nmm = (int64_t)nm * nm;
  for (int64_t q0 = 0; q0 < nq; q0 += HC) {
    const int64_t qn = std::min(HC, nq - q0);
    EPB_TRY(fourier_f64(ctx, m->dyn, nmm, nmm, m->rs_ph, xq_d + 3 * q0, qn, uph + q0 * nmm, nmm));
    EPB_TRY(eigh_async(ctx, uph + q0 * nmm, nm, qn, om + q0 * nm, true, m->mass, EPB_PREC_FP64));
  }
  if (prm->phonon_basis == 1) {
    oq_identity_kernel<<<grid_oq(ctx, nq * nmm), 256, 0, ctx->stream>>>(uph, nm, nq);
    EPB_LAUNCH_CHECK();
  }
  EPB_TRY(eigh_check(ctx));
  int64_t nkeep = 0;
  {
    int64_t* h = (int64_t*)ctx->pinned;
    EPB_CUDA(cudaMemcpyAsync(h, nkeep_d, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    EPB_CUDA(cudaStreamSynchronize(ctx->stream));
    nkeep = h[0];
  }

  // ---- batch sizes ----
  const int64_t KB = std::max<int64_t>(1, std::min<int64_t>(nkeep, prm->k_batch > 0 ? prm->k_batch : 4096));
  const int64_t per_q = 16 * nd * nr_el;
  const int64_t QC = std::max<int64_t>(
      1, std::min<int64_t>(nq, prm->q_chunk > 0 ? prm->q_chunk : std::max<int64_t>(1, ((int64_t)1 << 31) / per_q)));
  if (stats_host) {
    stats_host[0] = nkeep;
    stats_host[1] = (prec == EPB_PREC_MIXED && nkeep > KB) ? (KB + 127) / 128 * 128 : KB;
    stats_host[2] = QC;
  }
  const bool mixed = prec == EPB_PREC_MIXED;
  // per-run / per-q buffers: g(Re, q) of a chunk (and its mode rotation); in the mixed mode the packed
  // split-BF16 operands that live across batches: H(R) (per run), the phases of every kept k (per run),
  // g(Re, q) of the current q
  size_t off1 = 0;
  auto take1 = [&](size_t bytes) {
    size_t o = off1;
    off1 += (bytes + 1023) & ~size_t(1023);
    return o;
  };
  const size_t o_Gq = take1((size_t)per_q * QC),
               o_Grq = (prm->phonon_basis == 0 || mixed) ? take1((size_t)per_q * QC) : o_Gq,
               o_ah = mixed ? take1(oq_a_bytes(nw2, nr_el)) : 0,
               o_bk = mixed && nkeep > 0 ? take1(oq_b_bytes(nkeep, nr_el)) : 0,
               o_ag = mixed ? take1(oq_a_bytes(nd, nr_el)) : 0, o_bq = mixed ? take1(oq_b_bytes(QC, m->nr_ep)) : 0;
  void* ws1 = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_OQ1, off1 + 1024, &ws1));
  uint8_t* b1 = (uint8_t*)(((uintptr_t)ws1 + 1023) & ~uintptr_t(1023));
  double2* Gq = (double2*)(b1 + o_Gq);    // Fourier over Rp, (nd nr_el, QC)
  double2* Grq = (double2*)(b1 + o_Grq);  // after the mode rotation
  uint8_t* a_h = b1 + o_ah;
  uint8_t* b_k = b1 + o_bk;
  uint8_t* a_g = b1 + o_ag;
  uint8_t* b_q = b1 + o_bq;
  if (mixed && !m->epmat_ph_planes) {  // split-BF16 planes of the "ph"-layout epmat, once per model
    EPB_CUDA(cudaMalloc(&m->epmat_ph_planes, (size_t)oq_a_bytes(nd * nr_el, m->nr_ep)));
    EPB_TRY(oq_pack_a(ctx, m->epmat_ph, nd * nr_el, nd * nr_el, m->nr_ep, m->epmat_ph_planes));
  }
  // per-batch buffers; the mixed mode keeps a multiple of 128 k per batch (packed phase tiles)
  const int64_t KBm = (mixed && nkeep > KB) ? (KB + 127) / 128 * 128 : KB;
  size_t off2 = 0;
  auto take2 = [&](size_t bytes) {
    size_t o = off2;
    off2 += (bytes + 1023) & ~size_t(1023);
    return o;
  };
  const size_t o_xkq = take2(24 * KBm), o_H = take2(16 * nw2 * KBm), o_Ekq = take2(8 * nw * KBm),
               o_g = take2((mixed ? 8 : 16) * nd * KBm), o_ep = take2(ncalc > 0 ? 16 * nd * KBm : 0),
               o_part = take2(8 * KBm), o_bh = mixed ? take2(oq_b_bytes(KBm, nr_el)) : 0,
               o_ch = mixed ? take2(8 * nw2 * KBm) : 0, o_gw = mixed && nw > 16 ? take2(16 * nd * KBm) : 0;
  void* ws2 = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_OQ2, off2 + 1024, &ws2));
  uint8_t* b2 = (uint8_t*)(((uintptr_t)ws2 + 1023) & ~uintptr_t(1023));
  double* xkq = (double*)(b2 + o_xkq);
  double2* Hkq = (double2*)(b2 + o_H);
  double* Ekq = (double*)(b2 + o_Ekq);
  double2* gk = (double2*)(b2 + o_g);
  float2* gk32 = (float2*)(b2 + o_g);
  double2* ep = ncalc > 0 ? (double2*)(b2 + o_ep) : nullptr;
  double* part = (double*)(b2 + o_part);
  uint8_t* b_h = b2 + o_bh;
  float2* ch = (float2*)(b2 + o_ch);
  if (mixed) {
    EPB_TRY(oq_pack_a(ctx, m->ham, nw2, nw2, nr_el, a_h));
    if (nkeep > 0) EPB_TRY(oq_pack_b(ctx, m->rs_el, xkk, nkeep, b_k));
  }

  int64_t nbatches = 0;
  for (int64_t q0 = 0; q0 < nq; q0 += QC) {
    const int64_t qn = std::min(QC, nq - q0);
    // g(Re, q) = sum_Rp e^{2 pi i q.Rp} g(Re, Rp) for the chunk, then the mode rotation
    if (mixed) {  // split-BF16 tensor cores: complex64 g(Re, q), widened by the mode rotation (or a copy)
      float2* G32 = (float2*)Gq;
      EPB_TRY(oq_pack_b(ctx, m->rs_ep, xq_d + 3 * q0, qn, b_q));
      EPB_TRY(oq_gemm(ctx, EPB_PROF_UMMA_RR, m->epmat_ph_planes, nd * nr_el, m->nr_ep, b_q, qn, 0, qn, G32, nd * nr_el));
      prof_begin(ctx, EPB_PROF_RR_ROT);
      if (prm->phonon_basis == 0)
        rq_mode_rotate_kernel<float2><<<grid_oq(ctx, nd * nr_el * qn), 256, 0, ctx->stream>>>(
            G32, uph + q0 * nmm, nw2, nm, nr_el, qn, Grq);
      else
        oq_widen_kernel<<<grid_oq(ctx, nd * nr_el * qn), 256, 0, ctx->stream>>>(G32, nd * nr_el * qn, Grq);
      prof_end(ctx);
      EPB_LAUNCH_CHECK();
    } else {
      EPB_TRY(fourier_rows(ctx, m->epmat_ph, nd * nr_el, nd * nr_el, m->rs_ep, xq_d + 3 * q0, qn, Gq, nd * nr_el));
      if (prm->phonon_basis == 0) {
        prof_begin(ctx, EPB_PROF_RR_ROT);
        rq_mode_rotate_kernel<double2><<<grid_oq(ctx, nd * nr_el * qn), 256, 0, ctx->stream>>>(
            Gq, uph + q0 * nmm, nw2, nm, nr_el, qn, Grq);
        prof_end(ctx);
        EPB_LAUNCH_CHECK();
      }
    }
    for (int64_t iq = q0; iq < q0 + qn; ++iq) {
      for (int c = 0; c < ncalc; ++c)
        if (calcs[c].begin_q) {
          const int st = calcs[c].begin_q(calcs[c].user, iq, (void*)ctx->stream);
          if (st != 0) {
            set_error("epb_eph_outer_q: calculator %d begin_q returned %d at iq=%lld", c, st, (long long)iq);
            return EPB_ERR_ARG;
          }
        }
      const double2* gRq = Grq + (iq - q0) * nd * nr_el;
      if (mixed && nkeep > 0) EPB_TRY(oq_pack_a(ctx, gRq, nd, nd, nr_el, a_g));
      for (int64_t k0 = 0; k0 < nkeep; k0 += KBm) {
        const int64_t kn = std::min(KBm, nkeep - k0);
        oq_shift_kernel<<<grid_oq(ctx, 3 * kn), 256, 0, ctx->stream>>>(xkk + 3 * k0, kn, xq_d + 3 * iq, xkq);
        EPB_LAUNCH_CHECK();
        // H(k+q): split-BF16 tensor cores in the mixed mode (FP32-level H, as in the mixed outer-k pass)
        if (mixed) {
          EPB_TRY(oq_pack_b(ctx, m->rs_el, xkq, kn, b_h));
          EPB_TRY(oq_gemm(ctx, EPB_PROF_UMMA_H, a_h, nw2, nr_el, b_h, kn, 0, kn, ch, nw2));
          oq_widen_kernel<<<grid_oq(ctx, nw2 * kn), 256, 0, ctx->stream>>>(ch, nw2 * kn, Hkq);
          EPB_LAUNCH_CHECK();
        } else {
          EPB_TRY(fourier_f64(ctx, m->ham, nw2, nw2, m->rs_el, xkq, kn, Hkq, nw2));
        }
        EPB_TRY(eigh_async(ctx, Hkq, nw, kn, Ekq, true, nullptr, prec));
        oq_mask_kernel<<<grid_oq(ctx, kn * nw2), 256, 0, ctx->stream>>>(Hkq, Ekq, nw, kn, prm->wmin_kq, prm->wmax_kq);
        EPB_LAUNCH_CHECK();
        if (mixed) {
          // g(k, q) stays complex64 (the split GEMM's output precision) and is widened in the rotation
          EPB_TRY(oq_gemm(ctx, EPB_PROF_UMMA_KQ, a_g, nd, nr_el, b_k, nkeep, k0, kn, gk32, nd));
          if (nw <= 16) {
            EPB_TRY(oq_rotate(ctx, (const float2*)gk32, Uk + k0 * nw2, Hkq, wkk + k0, nw, nm, kn, ep, part));
          } else {  // nw > 16: widen to complex128 for the per-mode kernel
            double2* gw = (double2*)(b2 + o_gw);
            oq_widen_kernel<<<grid_oq(ctx, nd * kn), 256, 0, ctx->stream>>>(gk32, nd * kn, gw);
            EPB_LAUNCH_CHECK();
            EPB_TRY(oq_rotate(ctx, (const double2*)gw, Uk + k0 * nw2, Hkq, wkk + k0, nw, nm, kn, ep, part));
          }
        } else {
          EPB_TRY(fourier_f64(ctx, gRq, nd, nd, m->rs_el, xkk + 3 * k0, kn, gk, nd));
          EPB_TRY(oq_rotate(ctx, (const double2*)gk, Uk + k0 * nw2, Hkq, wkk + k0, nw, nm, kn, ep, part));
        }
        oq_record_kernel<<<1, 256, 0, ctx->stream>>>(part, kn, A_d + iq);
        EPB_LAUNCH_CHECK();
        ++nbatches;
        if (ncalc > 0) {
          epb_kbatch_payload p;
          p.iq = iq;
          p.k0 = k0;
          p.nk = kn;
          p.nw = nw;
          p.nm = nm;
          p.eps = (const double*)ep;
          p.ek = Ek + k0 * nw;
          p.ekq = Ekq;
          p.uk = (const double*)(Uk + k0 * nw2);
          p.ukq = (const double*)Hkq;
          p.wtk = wkk + k0;
          p.xk = xkk + 3 * k0;
          p.ik = keep + k0;
          p.omega = om + iq * nm;
          p.stream = (void*)ctx->stream;
          for (int c = 0; c < ncalc; ++c) {
            const int st = calcs[c].run_batch(calcs[c].user, &p);
            if (st != 0) {
              set_error("epb_eph_outer_q: calculator %d run_batch returned %d at iq=%lld", c, st, (long long)iq);
              return EPB_ERR_ARG;
            }
          }
        }
      }
      EPB_TRY(eigh_check(ctx));
      if (mixed) EPB_TRY(split_gemm_check(ctx));
      for (int c = 0; c < ncalc; ++c)
        if (calcs[c].end_q) {
          const int st = calcs[c].end_q(calcs[c].user, iq, (void*)ctx->stream);
          if (st != 0) {
            set_error("epb_eph_outer_q: calculator %d end_q returned %d at iq=%lld", c, st, (long long)iq);
            return EPB_ERR_ARG;
          }
        }
    }
  }
  if (stats_host) stats_host[3] = nbatches;
  if (A_host) {
    EPB_CUDA(cudaMemcpyAsync(A_host, A_d, 8 * nq, cudaMemcpyDeviceToHost, ctx->stream));
  }
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  return EPB_OK;
}

}  // extern "C"
