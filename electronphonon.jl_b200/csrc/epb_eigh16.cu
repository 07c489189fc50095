// Batched Hermitian eigensolver for n <= 16, register resident: one-sided (Hestenes) Jacobi.
//
// Replaces eigvals_batched / eigen_batched (ext/ElectronPhononCUDAExt.jl:80-115, cuSOLVER
// heevjBatched) for the small matrices of the e-ph pass (nw = 16 electrons, nm = 12 modes).
//
// A 16-lane half-warp owns one matrix; lane l holds column l of A = H + sigma I in registers
// (sigma = 1.1 ||H||_F makes A positive definite, so its right singular vectors are the
// eigenvectors of H and the column norms after orthogonalisation are lambda + sigma). Each round
// pairs the lanes by the circle method (lane 15 fixed); partners swap columns with shuffles,
// form the 2x2 Gram matrix [[a, g], [g*, b]] and both apply the same plane rotation
//     t = sign(tau) / (|tau| + sqrt(1 + tau^2)), tau = (b - a) / (2 |g|), e = g / |g|,
//     a_p <- c a_p - s conj(e) a_q,   a_q <- s e a_p + c a_q,
// (the same J as the two-sided solver, applied to columns only). A pair is skipped when
// |g| <= tol sqrt(a b); a sweep with no rotation ends the solve. Lanes >= n carry sigma e_l,
// orthogonal to every live column, so they never rotate.
//
// Mixed precision (EPB_PREC_MIXED): the sweeps run in FP32 to tol = 1e-6, then one FP64
// refinement on the same registers: Lowdin re-orthonormalisation V(I - F/2), F = V^H V - I
// (this re-orthogonalises near-degenerate clusters, whose FP32 vectors are defined only up to a
// rotation inside the cluster), and a first-order Rayleigh-Ritz update from S = V^H H V:
//     S'_kl = S_kl - F_kl (S_kk + S_ll) / 2,   E_kl = S'_kl / (S'_ll - S'_kk),
//     v_l <- v_l + sum_k v_k (E_kl - F_kl / 2),  lambda_l = S'_ll + sum_k |S'_kl|^2 / (S'_ll - S'_kk).
// Pairs whose first-order coupling is not small (|S'_kl| > 0.1 |S'_ll - S'_kk|) are left to the
// orthonormalisation (their vectors are accurate as a subspace, which is what gauge-invariant
// quantities use). EPB_PREC_FP64 runs the sweeps in FP64 to tol = 1e-15 and skips the refinement.
#include <type_traits>

#include "epb_common.cuh"

namespace epb {

constexpr int E16 = 16;

__device__ __forceinline__ int circle_partner(int l, int r) {
  // 16 players, player 15 fixed, 15 rounds
  if (l == 15) return r;
  if (l == r) return 15;
  int p = (2 * r - l) % 15;
  return p < 0 ? p + 15 : p;
}

template <typename T>
__device__ __forceinline__ T shfl(T v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}
__device__ __forceinline__ float2 shfl2(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// Sweeps of the one-sided Jacobi on the register column a[16] (of this lane). All 32 lanes of the
// warp take part (two matrices); returns the number of sweeps.
template <typename T>
__device__ int onesided_sweeps(typename cplx<T>::type (&a)[E16], T tol, int max_sweeps) {
  using C = typename cplx<T>::type;
  const int lane = threadIdx.x & 31;
  const int l = lane & 15, base = lane & 16;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    T nrm = 0;
#pragma unroll
    for (int i = 0; i < E16; ++i) nrm += a[i].x * a[i].x + a[i].y * a[i].y;
    int rotated = 0;
#pragma unroll 1
    for (int r = 0; r < 15; ++r) {
      const int pl = circle_partner(l, r);
      const int src = base + pl;
      C b[E16];
#pragma unroll
      for (int i = 0; i < E16; ++i) b[i] = shfl2(a[i], src);
      const T nb = shfl(nrm, src);
      const bool isP = l < pl;
      C g = mk2(T(0), T(0));
#pragma unroll
      for (int i = 0; i < E16; ++i) {
        if (isP)
          cfma_conj(g, a[i], b[i]);
        else
          cfma_conj(g, b[i], a[i]);
      }
      const T ap = isP ? nrm : nb, aq = isP ? nb : nrm;
      const T ag = sqrt(g.x * g.x + g.y * g.y);
      if (ag > tol * sqrt(ap * aq) && ag > T(0)) {
        rotated = 1;
        const T tau = (aq - ap) / (T(2) * ag);
        const T t = (tau >= T(0) ? T(1) : T(-1)) / (fabs(tau) + sqrt(T(1) + tau * tau));
        const T c = T(1) / sqrt(T(1) + t * t), s = t * c;
        const C e = mk2(g.x / ag, g.y / ag);
        if (isP) {
          const C ec = mk2(e.x, -e.y);
#pragma unroll
          for (int i = 0; i < E16; ++i) {
            C u = cmul(ec, b[i]);
            a[i] = mk2(c * a[i].x - s * u.x, c * a[i].y - s * u.y);
          }
          nrm = ap - t * ag;
        } else {
#pragma unroll
          for (int i = 0; i < E16; ++i) {
            C u = cmul(e, b[i]);
            a[i] = mk2(s * u.x + c * a[i].x, s * u.y + c * a[i].y);
          }
          nrm = aq + t * ag;
        }
      }
    }
    if (!__any_sync(0xffffffffu, rotated)) break;
  }
  return sweep;
}

struct Eigh16Args {
  const double2* A;   // c128 input (n x n per matrix, upper triangle), or null
  const float* Hp;    // packed FP32 Hermitian input (n*n per matrix), or null
  double2* U64;       // c128 eigenvector output (may alias A), or null
  float2* U32;        // c64 eigenvector output, or null
  double* E;          // eigenvalues (n per matrix), or null
  const double* mass; // phonon mode: scale by 1/sqrt(m_i m_j), omega = sign sqrt, u /= sqrt(m)
  int n;
  int64_t batch;
  int max_sweeps;
  int* nonconv;
  int refine;         // FP64 refinement iterations (mixed only)
  int64_t* flag_list; // if non-null: matrices with a near-degenerate pair are listed, not written
  int* flag_count;
};

template <bool MIXED>
__global__ void __launch_bounds__(128) eigh16_kernel(Eigh16Args a) {
  using T = typename std::conditional<MIXED, float, double>::type;
  using C = typename cplx<T>::type;
  // per matrix: H (FP64, 16 x 16) and V (FP64, 16 x 16) for the refinement; 8 matrices per block
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto Hs = reinterpret_cast<double2(*)[E16 * E16]>(smem_raw);
  auto Vs = reinterpret_cast<double2(*)[E16 * E16]>(smem_raw + 8 * E16 * E16 * sizeof(double2));
  const int lane = threadIdx.x & 31;
  const int l = lane & 15;
  const int slot = (threadIdx.x >> 4);  // matrix slot within the block (0..7)
  const int n = a.n;
  const int64_t per_block = blockDim.x / 16;
  for (int64_t b0 = (int64_t)blockIdx.x * per_block; b0 < a.batch; b0 += (int64_t)gridDim.x * per_block) {
    const int64_t b = b0 + slot;
    const bool live = b < a.batch;
    // ---- load column l of H (FP64), Frobenius norm ----
    double2 h[E16];
#pragma unroll
    for (int i = 0; i < E16; ++i) {
      double2 v = make_double2(0.0, 0.0);
      if (live && l < n && i < n) {
        if (a.Hp) {
          const float* hp = a.Hp + b * (int64_t)n * n;
          const int nre = n * (n + 1) / 2;
          int ii = i <= l ? i : l, jj = i <= l ? l : i;
          double re = hp[jj * (jj + 1) / 2 + ii];
          double im = ii < jj ? hp[nre + jj * (jj - 1) / 2 + ii] : 0.0;
          v = make_double2(re, i <= l ? im : -im);
        } else {
          const double2* ab = a.A + b * (int64_t)n * n;
          if (i <= l) {
            v = ab[i + (int64_t)l * n];
          } else {
            double2 u = ab[l + (int64_t)i * n];
            v = make_double2(u.x, -u.y);
          }
        }
        if (i == l) v.y = 0.0;
        if (a.mass) {
          double s = 1.0 / (sqrt(a.mass[i]) * sqrt(a.mass[l]));
          v.x *= s;
          v.y *= s;
        }
      }
      h[i] = v;
    }
    double f2 = 0.0;
#pragma unroll
    for (int i = 0; i < E16; ++i) f2 += h[i].x * h[i].x + h[i].y * h[i].y;
    for (int o = 8; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);  // within the half-warp
    const double sigma = f2 > 0.0 ? 1.1 * sqrt(f2) : 1.0;  // zero (or padding) matrices: shift 1
    // ---- one-sided Jacobi on A = H + sigma I ----
    C col[E16];
#pragma unroll
    for (int i = 0; i < E16; ++i) {
      double2 v = h[i];
      if (i == l) v.x += sigma;  // lanes >= n: sigma e_l
      col[i] = mk2((T)v.x, (T)v.y);
    }
    if (MIXED) {
#pragma unroll
      for (int i = 0; i < E16; ++i) Hs[slot][i + E16 * l] = h[i];
    }
    const T tol = MIXED ? T(1e-6) : T(1e-15);
    int sw = onesided_sweeps<T>(col, tol, a.max_sweeps);
    if (sw >= a.max_sweeps && lane == 0) atomicAdd(a.nonconv, 1);
    // eigenvector = normalised column, eigenvalue = |column| - sigma
    double nr2 = 0.0;
#pragma unroll
    for (int i = 0; i < E16; ++i) nr2 += (double)col[i].x * col[i].x + (double)col[i].y * col[i].y;
    const double inv = 1.0 / sqrt(nr2);
    double2 v[E16];
#pragma unroll
    for (int i = 0; i < E16; ++i) v[i] = make_double2(col[i].x * inv, col[i].y * inv);
    double lam = sqrt(nr2) - sigma;
    bool cluster = false;  // some pair stayed outside first-order validity (near-degenerate)
    if (MIXED) {
      // ---- FP64 refinement (a.refine iterations) ----
      for (int it = 0; it < a.refine; ++it) {
#pragma unroll
        for (int i = 0; i < E16; ++i) Vs[slot][i + E16 * l] = v[i];
        __syncwarp();
        double2 w[E16];  // w = H v
#pragma unroll
        for (int i = 0; i < E16; ++i) w[i] = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < E16; ++k) {
          double2 vk = v[k];
#pragma unroll
          for (int i = 0; i < E16; ++i) cfma(w[i], Hs[slot][i + E16 * k], vk);
        }
        double d = 0.0, fll = 0.0;
#pragma unroll
        for (int i = 0; i < E16; ++i) {
          d += v[i].x * w[i].x + v[i].y * w[i].y;   // Re v^H H v
          fll += v[i].x * v[i].x + v[i].y * v[i].y;
        }
        fll -= 1.0;
        const double dp = d * (1.0 - fll);          // S'_ll
        double2 tcol[E16];                          // column l of (E - F/2)
        double lam_corr = 0.0;
        cluster = false;
#pragma unroll
        for (int k = 0; k < E16; ++k) {
          const double dk = __shfl_sync(0xffffffffu, d, (lane & 16) + k);
          const double dpk = __shfl_sync(0xffffffffu, dp, (lane & 16) + k);
          double2 s = make_double2(0.0, 0.0), g = make_double2(0.0, 0.0);
#pragma unroll
          for (int i = 0; i < E16; ++i) {
            double2 vik = Vs[slot][i + E16 * k];
            cfma_conj(s, vik, w[i]);
            cfma_conj(g, vik, v[i]);
          }
          double2 t;
          if (k == l) {
            t = make_double2(-0.5 * fll, 0.0);
          } else {
            double2 sp = make_double2(s.x - 0.5 * g.x * (dk + d), s.y - 0.5 * g.y * (dk + d));
            double gap = dp - dpk;
            double asp = sqrt(sp.x * sp.x + sp.y * sp.y);
            t = make_double2(-0.5 * g.x, -0.5 * g.y);
            if (k < n && l < n) {
              if (asp < 0.1 * fabs(gap)) {
                t.x += sp.x / gap;
                t.y += sp.y / gap;
                lam_corr += asp * asp / gap;
              } else if (asp > 1e-13 * sigma) {
                cluster = true;
              }
            }
          }
          tcol[k] = t;
        }
        double2 vn[E16];
#pragma unroll
        for (int i = 0; i < E16; ++i) vn[i] = v[i];
#pragma unroll
        for (int k = 0; k < E16; ++k) {
          double2 t = tcol[k];
#pragma unroll
          for (int i = 0; i < E16; ++i) cfma(vn[i], Vs[slot][i + E16 * k], t);
        }
#pragma unroll
        for (int i = 0; i < E16; ++i) v[i] = vn[i];
        lam = dp + lam_corr;
        __syncwarp();
      }
    }
    // a matrix with a near-degenerate pair is re-solved by the FP64 slow path when requested
    const bool flagged = __any_sync(0xffffffffu, cluster && live) &&
                         (__ballot_sync(0xffffffffu, cluster && live) & (0xFFFFu << (lane & 16)));
    if (a.flag_list && flagged && l == 0) {
      int pos = atomicAdd(a.flag_count, 1);
      a.flag_list[pos] = b;
    }
    // ---- sort (rank among live lanes) and write ----
    int rank = 0;
#pragma unroll
    for (int k = 0; k < E16; ++k) {
      double lk = __shfl_sync(0xffffffffu, lam, (lane & 16) + k);
      rank += (k < n) && (lk < lam || (lk == lam && k < l));
    }
    if (live && l < n && !(a.flag_list && flagged)) {
      double ev = lam;
      if (a.mass) ev = ev >= 0 ? sqrt(ev) : -sqrt(-ev);
      if (a.E) a.E[b * n + rank] = ev;
#pragma unroll
      for (int i = 0; i < E16; ++i) {
        if (i < n) {
          double2 o = v[i];
          if (a.mass) {
            double s = 1.0 / sqrt(a.mass[i]);
            o.x *= s;
            o.y *= s;
          }
          if (a.U32) a.U32[b * (int64_t)n * n + i + (int64_t)rank * n] = make_float2((float)o.x, (float)o.y);
          if (a.U64) a.U64[b * (int64_t)n * n + i + (int64_t)rank * n] = o;
        }
      }
    }
  }
}

int eigh16_launch(epb_ctx* ctx, Eigh16Args& a, bool mixed) {
  if (a.batch == 0) return EPB_OK;
  const int threads = 128;  // 8 matrices per block
  int64_t blocks_needed = cdiv(a.batch, threads / 16);
  int64_t cap = (int64_t)ctx->sm_count * (mixed ? 8 : 8);
  unsigned grid = (unsigned)(blocks_needed < cap ? blocks_needed : cap);
  const size_t smem = mixed ? 2 * 8 * E16 * E16 * sizeof(double2) : 0;
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(eigh16_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * 8 * E16 * E16 * sizeof(double2))));
    attr = true;
  }
  prof_begin(ctx, EPB_PROF_EIGH);
  if (mixed)
    eigh16_kernel<true><<<grid, threads, smem, ctx->stream>>>(a);
  else
    eigh16_kernel<false><<<grid, threads, 0, ctx->stream>>>(a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

}  // namespace epb
