// Eigenvalue-only path for small Hermitian matrices (order <= 32): Householder reduction to a real
// symmetric tridiagonal T, then Sturm counts on T.
//
// Used where only band energies or energy-window band ranges are needed: the window test of
// src/filter.jl:19,40-72 (first = searchsortedfirst(e, wmin) = #(e < wmin) + 1, last =
// searchsortedlast(e, wmax) = #(e <= wmax)) and eigvals_batched (ext/ElectronPhononCUDAExt.jl:80-98,
// src/wannier_to_bloch_batched.jl:30-46). A window needs two Sturm counts instead of a full
// eigensolve; eigenvalues come from bisection on T.
//
// One warp per matrix; lane i holds row i of the (zero-padded) N x N matrix in registers. Step k
// (k = 0 .. N-3) reflects x = A[k+1:N, k] onto a multiple of e_1 with the Hermitian unitary
// P = I - beta u u^H, u = x + e^{i theta} ||x|| e_1 (theta = arg x_1), beta = 1 / (||x|| (||x|| + |x_1|)),
// and updates the trailing block as A <- A - u w^H - w u^H with p = beta A u,
// K = (beta / 2) u^H p (real), w = p - K u. The tridiagonal keeps d_k = A[k][k] and the squared
// off-diagonal e_k^2 = ||x||^2 (the phase of the off-diagonal does not change the eigenvalues).
// Rows and columns beyond the true order n are zero and stay decoupled; counts run over the first
// n entries only.
//
// Sturm count (number of eigenvalues below sigma): q_0 = d_0 - sigma,
// q_i = d_i - sigma - e_{i-1}^2 / q_{i-1}, count the negative q_i; |q| < pivmin is replaced by
// -pivmin (the LAPACK dstebz convention).
#include <algorithm>

#include "epb_common.cuh"

namespace epb {

constexpr int TRI_WARPS = 4;  // matrices (warps) per block

struct TriArgs {
  const float* Hp;     // Hermitian-packed FP32 input (n^2 floats per matrix: Re i<=j, then Im i<j)
  const double2* A;    // or c128 column-major input (upper triangle read)
  int n;
  int64_t batch;
  // window mode
  int nsh;             // 2 (exact) or 4 (guarded: wmin -/+ delta, wmax -/+ delta)
  double sh[4];        // shifts; counts are #(lambda < sh)
  int32_t* bmin;       // first in-window band (1-based) or 0
  int32_t* bmax;       // last in-window band or 0
  int32_t* flag;       // guarded mode: 1 if an eigenvalue may lie within delta of a window edge
  // eigenvalue mode
  double* E;           // (n, batch) ascending
  // tridiagonal mode: d and e^2 per matrix (32 doubles each)
  double* Dt;
  double* E2t;
};

template <typename T>
struct TriSmem {
  typename cplx<T>::type u[32];  // reflector u
  typename cplx<T>::type w[32];  // w = p - K u
  T d[32];      // tridiagonal
  T e2[32];
  float stage[32 * 32];  // packed FP32 input staging
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double sturm_div(double a, double b) { return a / b; }
// FP32 counts are only used with guard intervals far wider than the 2-ulp fast division error.
__device__ __forceinline__ float sturm_div(float a, float b) { return __fdividef(a, b); }

template <typename T>
__device__ __forceinline__ int sturm_count(const T* d, const T* e2, int n, T sigma, T pivmin) {
  int c = 0;
  T q = d[0] - sigma;
  if (fabs(q) < pivmin) q = -pivmin;
  c += q < T(0);
  for (int i = 1; i < n; ++i) {
    q = (d[i] - sigma) - sturm_div(e2[i - 1], q);
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < T(0);
  }
  return c;
}

// Steps k = J0 .. min(J0 + 8, N - 1) - 1 of the reduction (see the file header). The step loop is not
// unrolled (a fully unrolled 31-step reduction overflows the instruction cache); the inner loops run
// over the compile-time range j = J0 .. N - 1 with the columns j <= k masked, and column k is picked
// from registers by an 8-way select.
template <typename T, int N, int J0>
__device__ __forceinline__ void householder_phase(T (&ar)[N], T (&ai)[N], TriSmem<T>& s, int lane, T& dk, T& ek2) {
  constexpr int KEND = (J0 + 8 < N - 1) ? J0 + 8 : N - 1;
#pragma unroll 1
  for (int k = J0; k < KEND; ++k) {
    // column k below the diagonal: x_i = A[i][k], i > k (row `lane`, column k)
    T xr = 0, xi = 0;
#pragma unroll
    for (int j = J0; j < J0 + 8 && j < N; ++j)
      if (j == k) {
        xr = ar[j];
        xi = ai[j];
      }
    if (lane == k) dk = xr;
    const T xn2 = warp_sum(lane > k ? xr * xr + xi * xi : T(0));
    if (lane == k) ek2 = xn2;
    if (k == N - 2) break;      // last off-diagonal: no reflection left to apply
    if (xn2 == T(0)) continue;  // warp-uniform: column already reduced
    const T x1r = __shfl_sync(0xffffffffu, xr, k + 1), x1i = __shfl_sync(0xffffffffu, xi, k + 1);
    const T xn = sqrt(xn2), a1 = sqrt(x1r * x1r + x1i * x1i);
    const T beta = T(1) / (xn * (xn + a1));
    T ur = T(0), ui = T(0);
    if (lane > k + 1) {
      ur = xr;
      ui = xi;
    } else if (lane == k + 1) {
      // u_1 = e^{i theta} (|x_1| + ||x||)
      const T f = a1 > T(0) ? (a1 + xn) / a1 : T(1);
      ur = a1 > T(0) ? x1r * f : xn;
      ui = a1 > T(0) ? x1i * f : T(0);
    }
    s.u[lane] = mk2(ur, ui);  // zero for lanes <= k
    __syncwarp();
    // p_i = beta sum_{j>k} A[i][j] u_j (u_j = 0 for j <= k; two partial sums for ILP)
    T pr0 = 0, pi0 = 0, pr1 = 0, pi1 = 0;
#pragma unroll
    for (int j = J0 + 1; j < N; ++j) {
      const auto v = s.u[j];
      if ((j & 1) == 0) {
        pr0 = fma(ar[j], v.x, pr0);
        pr0 = fma(-ai[j], v.y, pr0);
        pi0 = fma(ar[j], v.y, pi0);
        pi0 = fma(ai[j], v.x, pi0);
      } else {
        pr1 = fma(ar[j], v.x, pr1);
        pr1 = fma(-ai[j], v.y, pr1);
        pi1 = fma(ar[j], v.y, pi1);
        pi1 = fma(ai[j], v.x, pi1);
      }
    }
    T pr = (pr0 + pr1) * beta, pi = (pi0 + pi1) * beta;
    if (lane <= k) {
      pr = T(0);
      pi = T(0);
    }
    // K = (beta / 2) Re(u^H p)
    const T kk = T(0.5) * beta * warp_sum(ur * pr + ui * pi);
    const T wr = pr - kk * ur, wi = pi - kk * ui;
    s.w[lane] = mk2(wr, wi);
    __syncwarp();
    if (lane > k) {
#pragma unroll
      for (int j = J0 + 1; j < N; ++j) {
        if (j > k) {
          const auto uj = s.u[j], wj = s.w[j];
          // A[i][j] -= u_i conj(w_j) + w_i conj(u_j)
          ar[j] -= (ur * wj.x + ui * wj.y) + (wr * uj.x + wi * uj.y);
          ai[j] -= (ui * wj.x - ur * wj.y) + (wi * uj.x - wr * uj.y);
        }
      }
    }
    __syncwarp();
  }
}

// Reduce the matrix held row-wise in (ar, ai) to tridiagonal form; writes d, e2 to shared memory.
template <typename T, int N>
__device__ __forceinline__ void householder_tridiag(T (&ar)[N], T (&ai)[N], TriSmem<T>& s, int lane) {
  static_assert(N == 32, "the reduction is laid out in four phases of eight steps");
  T dk = 0, ek2 = 0;
  householder_phase<T, N, 0>(ar, ai, s, lane, dk, ek2);
  householder_phase<T, N, 8>(ar, ai, s, lane, dk, ek2);
  householder_phase<T, N, 16>(ar, ai, s, lane, dk, ek2);
  householder_phase<T, N, 24>(ar, ai, s, lane, dk, ek2);
  if (lane == N - 1) dk = ar[N - 1];
  s.d[lane] = dk;
  s.e2[lane] = ek2;
  __syncwarp();
}

// Load row `lane` of matrix b (upper triangle as stored, Hermitian completion, zero padding).
template <typename T, int N>
__device__ __forceinline__ void load_rows(const TriArgs& a, int64_t b, int lane, T (&ar)[N], T (&ai)[N],
                                          TriSmem<T>& s) {
  const int n = a.n;
  if (a.Hp) {
    const float* src = a.Hp + b * (int64_t)n * n;
    for (int e = lane; e < n * n; e += 32) s.stage[e] = src[e];
    __syncwarp();
    const int nre = n * (n + 1) / 2;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      T re = 0, im = 0;
      if (lane < n && j < n) {
        if (lane <= j) {
          re = s.stage[j * (j + 1) / 2 + lane];
          im = lane < j ? s.stage[nre + j * (j - 1) / 2 + lane] : 0.f;
        } else {
          re = s.stage[lane * (lane + 1) / 2 + j];
          im = -s.stage[nre + lane * (lane - 1) / 2 + j];
        }
      }
      ar[j] = re;
      ai[j] = im;
    }
    __syncwarp();
  } else {
    const double2* src = a.A + b * (int64_t)n * n;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      T re = 0, im = 0;
      if (lane < n && j < n) {
        if (lane <= j) {
          const double2 v = src[lane + (int64_t)j * n];
          re = (T)v.x;
          im = lane < j ? (T)v.y : T(0);
        } else {
          const double2 v = src[j + (int64_t)lane * n];
          re = (T)v.x;
          im = (T)-v.y;
        }
      }
      ar[j] = re;
      ai[j] = im;
    }
  }
}

// MODE 0: window band ranges from Sturm counts at the shifts; MODE 1: all eigenvalues; MODE 2: the
// tridiagonal itself (d, e^2) for a later per-band bisection.
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(32 * TRI_WARPS) tridiag_kernel(TriArgs a) {
  __shared__ TriSmem<T> smem[TRI_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  TriSmem<T>& s = smem[warp];
  const int n = a.n;
  const int64_t w0 = (int64_t)blockIdx.x * TRI_WARPS + warp, nwarps = (int64_t)gridDim.x * TRI_WARPS;
  for (int64_t b = w0; b < a.batch; b += nwarps) {
    T ar[N], ai[N];
    load_rows<T, N>(a, b, lane, ar, ai, s);
    householder_tridiag<T, N>(ar, ai, s, lane);
    if (MODE == 2) {
      a.Dt[b * 32 + lane] = (double)s.d[lane];
      a.E2t[b * 32 + lane] = (double)s.e2[lane];
      __syncwarp();
      continue;
    }
    // pivmin: smallest safe pivot scaled by the largest off-diagonal (dstebz)
    T emax = 0;
    for (int i = 0; i < n; ++i) emax = fmax(emax, s.e2[i]);
    const T tiny = sizeof(T) == 8 ? T(2.2250738585072014e-308) : T(1.17549435e-38);
    const T pivmin = tiny * fmax(T(1), emax);
    if (MODE == 0) {
      int c = 0;
      const double shv = lane == 0 ? a.sh[0] : lane == 1 ? a.sh[1] : lane == 2 ? a.sh[2] : a.sh[3];
      if (lane < a.nsh) c = sturm_count<T>(s.d, s.e2, n, (T)shv, pivmin);
      const int c0 = __shfl_sync(0xffffffffu, c, 0), c1 = __shfl_sync(0xffffffffu, c, 1);
      const int c2 = __shfl_sync(0xffffffffu, c, 2), c3 = __shfl_sync(0xffffffffu, c, 3);
      if (lane == 0) {
        // exact: c0 = #(e < wmin), c1 = #(e <= wmax) (shift 1 is the successor of wmax).
        // guarded: c0/c1 bracket wmin and c2/c3 bracket wmax.
        const int below = c0, upto = a.nsh == 2 ? c1 : c3;
        const int first = below + 1, last = upto;
        const bool keep = last >= first;
        a.bmin[b] = keep ? first : 0;
        a.bmax[b] = keep ? last : 0;
        if (a.flag) a.flag[b] = a.nsh == 4 && ((c0 != c1) || (c2 != c3));
      }
    } else if (MODE == 1) {
      // Gershgorin interval of T, then bisection for eigenvalue `lane` (the (lane+1)-th smallest)
      T lo = 0, hi = 0;
      for (int i = 0; i < n; ++i) {
        const T r = (i > 0 ? sqrt(s.e2[i - 1]) : T(0)) + (i < n - 1 ? sqrt(s.e2[i]) : T(0));
        const T l = s.d[i] - r, h = s.d[i] + r;
        lo = i == 0 ? l : fmin(lo, l);
        hi = i == 0 ? h : fmax(hi, h);
      }
      const T eps = sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920929e-07);
      const T span = fmax(fabs(lo), fabs(hi));
      lo -= 2 * eps * span + 2 * pivmin;
      hi += 2 * eps * span + 2 * pivmin;
      if (lane < n) {
        for (int it = 0; it < 200; ++it) {
          const T mid = T(0.5) * (lo + hi);
          if (!(hi - lo > 2 * eps * fmax(fabs(lo), fabs(hi)) + pivmin) || mid <= lo || mid >= hi) break;
          if (sturm_count<T>(s.d, s.e2, n, mid, pivmin) > lane)
            hi = mid;
          else
            lo = mid;
        }
        a.E[b * (int64_t)n + lane] = (double)(T(0.5) * (lo + hi));
      }
    }
    __syncwarp();
  }
}

// One eigenvalue (0-based index `band`) per stored tridiagonal, one thread per matrix: bisection
// on the Gershgorin interval with Sturm counts, as in MODE 1.
__global__ void tridiag_band_kernel(const double* __restrict__ Dt, const double* __restrict__ E2t, int n, int64_t batch,
                                    int band, double* __restrict__ out) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < batch; b += (int64_t)gridDim.x * blockDim.x) {
    double d[32], e2[32];
    double emax = 0, lo = 0, hi = 0;
    for (int i = 0; i < n; ++i) {
      d[i] = Dt[b * 32 + i];
      e2[i] = E2t[b * 32 + i];
    }
    for (int i = 0; i < n; ++i) {
      emax = fmax(emax, e2[i]);
      const double r = (i > 0 ? sqrt(e2[i - 1]) : 0.0) + (i < n - 1 ? sqrt(e2[i]) : 0.0);
      lo = i == 0 ? d[i] - r : fmin(lo, d[i] - r);
      hi = i == 0 ? d[i] + r : fmax(hi, d[i] + r);
    }
    const double pivmin = 2.2250738585072014e-308 * fmax(1.0, emax), eps = 2.220446049250313e-16;
    const double span = fmax(fabs(lo), fabs(hi));
    lo -= 2 * eps * span + 2 * pivmin;
    hi += 2 * eps * span + 2 * pivmin;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (!(hi - lo > 2 * eps * fmax(fabs(lo), fabs(hi)) + pivmin) || mid <= lo || mid >= hi) break;
      if (sturm_count<double>(d, e2, n, mid, pivmin) > band)
        hi = mid;
      else
        lo = mid;
    }
    out[b] = 0.5 * (lo + hi);
  }
}

template <typename T, int MODE>
static int launch_tridiag(epb_ctx* ctx, const TriArgs& a) {
  auto kern = tridiag_kernel<T, 32, MODE>;
  int per_sm = 0;
  EPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * TRI_WARPS, 0));
  if (per_sm < 1) per_sm = 1;
  int64_t blocks = std::min<int64_t>(cdiv(a.batch, TRI_WARPS), (int64_t)per_sm * ctx->sm_count * 4);
  if (blocks < 1) blocks = 1;
  prof_begin(ctx, EPB_PROF_TRIDIAG);
  kern<<<(unsigned)blocks, 32 * TRI_WARPS, 0, ctx->stream>>>(a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Window band ranges of a batch of order-n Hermitian matrices (packed FP32 `Hp` or c128 `A`).
// delta == 0: exact counts at wmin and the successor of wmax (FP64 solve). delta > 0: FP32 solve
// with guard shifts wmin -/+ delta and wmax -/+ delta; `flag` marks the matrices whose counts
// differ across a guard interval (an eigenvalue may lie within delta of an edge).
int tridiag_window(epb_ctx* ctx, const float* Hp, const double2* A, int n, int64_t batch, double wmin, double wmax,
                   double delta, int32_t* bmin, int32_t* bmax, int32_t* flag) {
  if (batch == 0) return EPB_OK;
  EPB_CHECK_ARG(n >= 1 && n <= 32, "window counts: order %d outside 1..32", n);
  TriArgs a{};
  a.Hp = Hp;
  a.A = A;
  a.n = n;
  a.batch = batch;
  a.bmin = bmin;
  a.bmax = bmax;
  a.flag = flag;
  if (delta > 0) {
    EPB_CHECK_ARG(flag, "window counts: guarded mode needs a flag array");
    a.nsh = 4;
    a.sh[0] = wmin - delta;
    a.sh[1] = wmin + delta;
    a.sh[2] = wmax - delta;
    a.sh[3] = wmax + delta;
    return launch_tridiag<float, 0>(ctx, a);
  }
  a.nsh = 2;
  a.sh[0] = wmin;
  a.sh[1] = nextafter(wmax, INFINITY);
  return launch_tridiag<double, 0>(ctx, a);
}

// Energy of band `band` (0-based) of each matrix: FP64 reduction stored to Dt/E2t (batch x 32
// doubles each, caller workspace), then one bisection per matrix.
int tridiag_band(epb_ctx* ctx, const float* Hp, const double2* A, int n, int64_t batch, int band, double* Dt,
                 double* E2t, double* out) {
  if (batch == 0) return EPB_OK;
  EPB_CHECK_ARG(n >= 1 && n <= 32 && band >= 0 && band < n, "band energy: order %d / band %d", n, band);
  TriArgs a{};
  a.Hp = Hp;
  a.A = A;
  a.n = n;
  a.batch = batch;
  a.Dt = Dt;
  a.E2t = E2t;
  EPB_TRY((launch_tridiag<double, 2>(ctx, a)));
  const int64_t blocks = std::min<int64_t>(cdiv(batch, 128), (int64_t)ctx->sm_count * 16);
  prof_begin(ctx, EPB_PROF_TRIDIAG);
  tridiag_band_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), 128, 0, ctx->stream>>>(Dt, E2t, n, batch, band, out);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Ascending eigenvalues (FP64 reduction and bisection) of a batch of order-n Hermitian matrices.
int tridiag_eigvals(epb_ctx* ctx, const float* Hp, const double2* A, int n, int64_t batch, double* E) {
  if (batch == 0) return EPB_OK;
  EPB_CHECK_ARG(n >= 1 && n <= 32, "tridiagonal eigenvalues: order %d outside 1..32", n);
  TriArgs a{};
  a.Hp = Hp;
  a.A = A;
  a.n = n;
  a.batch = batch;
  a.E = E;
  return launch_tridiag<double, 1>(ctx, a);
}

}  // namespace epb
