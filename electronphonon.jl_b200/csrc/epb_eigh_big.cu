// Batched Hermitian eigensolver for orders 65 .. 96: FP32 two-sided Jacobi in shared memory, then
// FP64 Rayleigh-Ritz refinement with exact FP64 treatment of near-degenerate clusters.
//
// Replaces eigen_batched / eigvals_batched (ext/ElectronPhononCUDAExt.jl:80-115; CPU reference
// src/wannier_to_bloch_batched.jl:30-65, LAPACK ZHEEV) for the orders whose FP64 Jacobi state
// (A and V, 2 n^2 complex doubles) does not fit in shared memory.
//
// One CTA (512 threads) per matrix, persistent, matrices taken from a device work counter so that
// uneven orders balance. Per matrix:
//  1. A (Hermitian completion of the upper triangle) in FP32 in shared memory, cyclic two-sided
//     Jacobi with round-robin pairs (jacobi_team) accumulating V in FP32.
//  2. FP64 refinement, `refine` iterations, each on the CTA's global scratch (L2-resident):
//       G = V^H V,  V <- V (3/2 I - 1/2 G)               (Loewdin re-orthonormalisation)
//       S = V^H (H V), lambda_i = Re S_ii, tau = max(100 max_{i != j} |S_ij|, 1e-6 max |lambda|)
//       clusters: runs of the sorted lambda with consecutive gaps < tau
//       M_ij = S_ij / (lambda_j - lambda_i) between clusters (first-order Rayleigh-Ritz),
//       Q_c = the FP64 Jacobi eigenvectors of the cluster block S_cc (re-orthogonalisation of the
//             cluster inside its invariant subspace; clusters of up to 32 members)
//       V <- V (I + X) blockdiag(Q_c), X the first-order coefficients (zero inside clusters)
//  3. A last Loewdin step and S; eigenvalues = Re S_ii (Rayleigh quotients) ascending, eigenvectors
//     written over the input in ascending order.
// The FP32 solve leaves |S_ij| ~ 1e-7 ||H||; each refinement squares the relative error, so two
// iterations reach FP64 accuracy. EPB_PREC_FP64 runs three.
#include <algorithm>

#include "epb_jacobi.cuh"

namespace epb {

constexpr int BIG_NMAX = 96;

struct BigArgs {
  double2* A;
  const int64_t* a_off;
  const int32_t* nvec;
  int n_uniform;
  int64_t batch;
  double* E;
  const int64_t* e_off;
  int want_v;
  int max_sweeps;
  int refine;
  int n_lo;                        // orders <= n_lo belong to other kernels (skipped silently)
  int n_hi;                        // > 0: orders above n_hi belong to other kernels (skipped silently)
  int* nonconv;
  int* badsize;
  unsigned long long* counter;     // work counter (zeroed before launch)
  double2* scratch;                // 3 NMAX^2 per CTA
};

// Complex FP64 n x n GEMM, C = op(A) B, operands in global memory (L2-resident scratch or the input),
// 32 x 32 output tiles staged through shared memory. OPA: 0 = A, 1 = A^H, 2 = Hermitian completion of
// the upper triangle of A (diagonal imaginary part dropped).
template <int OPA, int NT>
__device__ void big_gemm(int n, const double2* __restrict__ A, int lda, const double2* __restrict__ B, int ldb,
                         double2* __restrict__ C, int ldc, double2* As, double2* Bs) {
  constexpr int NWB = NT / 32, RPT = 32 / NWB;  // warps; output rows per thread (ty + NWB r)
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int nt = (n + 31) / 32;
  for (int t = 0; t < nt * nt; ++t) {
    const int i0 = (t % nt) * 32, j0 = (t / nt) * 32;
    double2 acc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) acc[r] = make_double2(0.0, 0.0);
    for (int k0 = 0; k0 < n; k0 += 32) {
      __syncthreads();
      for (int e = tid; e < 1024; e += NT) {
        const int r = e & 31, c = e >> 5;  // As[r][c] = op(A)(i0 + r, k0 + c); Bs[c][r] = B(k0 + c, j0 + r)
        const int i = i0 + r, k = k0 + c;
        double2 v = make_double2(0.0, 0.0);
        if (i < n && k < n) {
          if (OPA == 0) {
            v = A[i + (int64_t)k * lda];
          } else if (OPA == 1) {
            const double2 u = A[k + (int64_t)i * lda];
            v = make_double2(u.x, -u.y);
          } else {
            if (i <= k) {
              v = A[i + (int64_t)k * lda];
              if (i == k) v.y = 0.0;
            } else {
              const double2 u = A[k + (int64_t)i * lda];
              v = make_double2(u.x, -u.y);
            }
          }
        }
        As[r * 33 + c] = v;
        const int kb = k0 + r, j = j0 + c;
        Bs[r * 33 + c] = (kb < n && j < n) ? B[kb + (int64_t)j * ldb] : make_double2(0.0, 0.0);
      }
      __syncthreads();
#pragma unroll 8
      for (int kk = 0; kk < 32; ++kk) {
        const double2 b = Bs[kk * 33 + tx];
#pragma unroll
        for (int r = 0; r < RPT; ++r) cfma(acc[r], As[(ty + NWB * r) * 33 + kk], b);
      }
    }
    // C(i0 + ty + NWB r, j0 + tx)
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = i0 + ty + NWB * r, j = j0 + tx;
      if (i < n && j < n) C[i + (int64_t)j * ldc] = acc[r];
    }
  }
  __syncthreads();
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = 0.0;
  for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

// Shared memory: FP32 Jacobi state (A32 NMAX x (NMAX+1), V32 NMAX x NMAX, rotation parameters),
// reused by the refinement for GEMM tiles and the cluster solve.
template <int NMAX>
struct BigSmem {
  static constexpr int A32 = NMAX * (NMAX + 1) * 8;
  static constexpr int V32 = NMAX * NMAX * 8;
  static constexpr int PRM = (NMAX / 2 + 1) * 64;
  static constexpr int JAC = A32 + V32 + PRM + 64;
  static constexpr int TILES = 2 * 32 * 33 * 16;
  static constexpr int CLU = 32 * 33 * 16 + 32 * 32 * 16 + 17 * 64 + 64;
  static constexpr int REF = TILES > CLU ? TILES : CLU;
  static constexpr int TOTAL = (JAC > REF ? JAC : REF) + 4 * NMAX * 8 + 64 * 8;
};

template <int NMAX, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) eigh_big_kernel(BigArgs a) {
  using SM = BigSmem<NMAX>;
  extern __shared__ __align__(16) unsigned char sm[];
  // per-matrix vectors after the union region
  constexpr int U = SM::TOTAL - 4 * NMAX * 8 - 64 * 8;
  double* lam = reinterpret_cast<double*>(sm + U);           // NMAX
  int* rank = reinterpret_cast<int*>(lam + NMAX);         // NMAX
  int* perm = rank + NMAX;                                // NMAX
  int* cid = perm + NMAX;                                 // NMAX
  int* csize = cid + NMAX;                                // NMAX (cluster sizes by first sorted index)
  double* red = reinterpret_cast<double*>(sm + SM::TOTAL - 64 * 8);  // reductions, flags
  __shared__ long long s_b;
  __shared__ int s_flag;
  double2* slab = a.scratch + (int64_t)blockIdx.x * 3 * NMAX * NMAX;
  double2* V = slab;
  double2* W = slab + NMAX * NMAX;
  double2* G = slab + 2 * NMAX * NMAX;
  const int tid = threadIdx.x;

  for (;;) {
    if (tid == 0) s_b = (long long)atomicAdd(a.counter, 1ull);
    __syncthreads();
    const int64_t b = s_b;
    __syncthreads();
    if (b >= a.batch) break;
    const int n = a.nvec ? a.nvec[b] : a.n_uniform;
    if (n <= a.n_lo || (a.n_hi > 0 && n > a.n_hi)) continue;
    if (n > NMAX) {
      if (tid == 0 && a.n_lo == 0) atomicAdd(a.badsize, 1);  // varlen batches count bad orders on the host
      continue;
    }
    const int64_t aoff = a.a_off ? a.a_off[b] : b * (int64_t)n * n;
    const int64_t eoff = a.e_off ? a.e_off[b] : b * (int64_t)n;
    double2* H = a.A + aoff;

    // ---- 1. FP32 Jacobi ----
    float2* A32 = reinterpret_cast<float2*>(sm);
    float2* V32 = reinterpret_cast<float2*>(sm + SM::A32);
    void* prm = sm + SM::A32 + SM::V32;
    int* flag = reinterpret_cast<int*>(sm + SM::A32 + SM::V32 + SM::PRM);
    const int lda = n + 1;
    double fro2 = 0.0;
    for (int e = tid; e < n * n; e += NT) {
      const int i = e % n, j = e / n;
      double2 v;
      if (i <= j) {
        v = H[i + (int64_t)j * n];
        if (i == j) v.y = 0.0;
      } else {
        const double2 u = H[j + (int64_t)i * n];
        v = make_double2(u.x, -u.y);
      }
      A32[i + j * lda] = make_float2((float)v.x, (float)v.y);
      V32[i + j * n] = make_float2(i == j ? 1.f : 0.f, 0.f);
      fro2 += v.x * v.x + v.y * v.y;
    }
    for (int o = 16; o > 0; o >>= 1) fro2 += __shfl_xor_sync(0xffffffffu, fro2, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = fro2;
    __syncthreads();
    double fro = 0.0;
    for (int w = 0; w < NT / 32; ++w) fro += red[w];
    fro = sqrt(fro);
    __syncthreads();
    // stop at 8 eps32 x the RMS eigenvalue: below that, FP32 rounding of (near-)degenerate pairs would
    // re-trigger 45-degree rotations forever; the FP64 refinement supplies the remaining accuracy
    const int sw = jacobi_team<float, NT>(A32, lda, V32, n, n, true, reinterpret_cast<RotParam<float>*>(prm), flag,
                                             8.f * 1.1920929e-07f * (float)(fro / sqrt((double)n)), a.max_sweeps);
    if (sw >= a.max_sweeps && tid == 0) atomicAdd(a.nonconv, 1);
    for (int e = tid; e < n * n; e += NT) {
      const float2 v = V32[e];
      V[e] = make_double2(v.x, v.y);
    }
    __syncthreads();

    // ---- 2./3. FP64 refinement ----
    double2* As = reinterpret_cast<double2*>(sm);
    double2* Bs = As + 32 * 33;
    for (int it = 0; it <= a.refine; ++it) {
      // Loewdin: G = V^H V; W = V (3/2 I - 1/2 G); swap
      big_gemm<1, NT>(n, V, n, V, n, G, n, As, Bs);
      for (int e = tid; e < n * n; e += NT) {
        const int i = e % n, j = e / n;
        double2 g = G[e];
        G[e] = make_double2((i == j ? 1.5 : 0.0) - 0.5 * g.x, -0.5 * g.y);
      }
      __syncthreads();
      big_gemm<0, NT>(n, V, n, G, n, W, n, As, Bs);
      {
        double2* t = V;
        V = W;
        W = t;
      }
      // S = V^H (H V)
      big_gemm<2, NT>(n, H, n, V, n, W, n, As, Bs);
      big_gemm<1, NT>(n, V, n, W, n, G, n, As, Bs);
      double off = 0.0, dmax = 0.0;
      for (int e = tid; e < n * n; e += NT) {
        const int i = e % n, j = e / n;
        const double2 s = G[e];
        if (i == j) {
          lam[i] = s.x;
          dmax = fmax(dmax, fabs(s.x));
        } else {
          off = fmax(off, sqrt(s.x * s.x + s.y * s.y));
        }
      }
      __syncthreads();
      off = block_max<NT>(off, red);
      dmax = block_max<NT>(dmax, red);
      // ascending order (ties by index)
      for (int i = tid; i < n; i += NT) {
        int r = 0;
        for (int j = 0; j < n; ++j) r += (lam[j] < lam[i]) || (lam[j] == lam[i] && j < i);
        rank[i] = r;
        perm[r] = i;
      }
      __syncthreads();
      if (it == a.refine) break;  // final pass: Loewdin + Rayleigh quotients only
      // clusters: consecutive sorted gaps below tau
      // Below a relative gap of 1e-6 the first-order update is never used: the FP64 noise of S
      // (~n eps ||H||) would otherwise rotate near-degenerate vectors by noise / gap.
      const double tau = fmax(100.0 * off, 1e-6 * fmax(dmax, fro / n));
      if (tid == 0) {
        int c = 0, start = 0;
        s_flag = 0;
        cid[perm[0]] = 0;
        for (int r = 1; r < n; ++r) {
          if (lam[perm[r]] - lam[perm[r - 1]] >= tau) {
            csize[start] = r - start;
            if (r - start > 32) s_flag = 1;
            start = r;
            ++c;
          }
          cid[perm[r]] = c;
        }
        csize[start] = n - start;
        if (n - start > 32) s_flag = 1;
      }
      __syncthreads();
      if (s_flag && tid == 0) atomicAdd(a.nonconv, 1);  // oversize cluster: first-order only within it
      // M (in W): first-order Rayleigh-Ritz between clusters, identity inside clusters for now
      for (int e = tid; e < n * n; e += NT) {
        const int i = e % n, j = e / n;
        double2 m = make_double2(i == j ? 1.0 : 0.0, 0.0);
        if (i != j && cid[i] != cid[j]) {
          const double2 s = G[e];
          const double d = lam[j] - lam[i];
          m = make_double2(s.x / d, s.y / d);
        }
        W[e] = m;
      }
      __syncthreads();
      // clusters of 2..32 members: FP64 Jacobi of the block S_cc by warp 0, Q_c into M
      if (tid < 32) {
        double2* Ac = reinterpret_cast<double2*>(sm);       // 32 x 33
        double2* Qc = Ac + 32 * 33;                           // 32 x 32
        void* prmc = Qc + 32 * 32;
        int* flc = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(prmc) + 17 * 64);
        for (int r0 = 0; r0 < n;) {
          const int k = csize[r0];  // r0 is always the first sorted index of a cluster
          if (k >= 2 && k <= 32) {
            for (int e = tid; e < k * k; e += 32) {
              const int p = e % k, q = e / k;
              Ac[p + q * 33] = G[perm[r0 + p] + (int64_t)perm[r0 + q] * n];
              Qc[p + q * k] = make_double2(p == q ? 1.0 : 0.0, 0.0);
            }
            __syncwarp();
            jacobi_team<double, 32>(Ac, 33, Qc, k, k, true, reinterpret_cast<RotParam<double>*>(prmc), flc,
                                    2.220446049250313e-16 * fmax(dmax, 1e-300), 30);
            // M[:, c] <- M[:, c] Q_c: the cluster columns of (I + X) rotated into the cluster's eigenbasis
            for (int i = tid; i < n; i += 32) {
              double2 row[32];
              for (int p = 0; p < k; ++p) row[p] = W[i + (int64_t)perm[r0 + p] * n];
              for (int q = 0; q < k; ++q) {
                double2 acc = make_double2(0.0, 0.0);
                for (int p = 0; p < k; ++p) cfma(acc, row[p], Qc[p + q * k]);
                W[i + (int64_t)perm[r0 + q] * n] = acc;
              }
            }
            __syncwarp();
          }
          r0 += k;
        }
      }
      __syncthreads();
      // V <- V M
      big_gemm<0, NT>(n, V, n, W, n, G, n, As, Bs);
      {
        double2* t = V;
        V = G;
        G = t;
      }
    }
    // outputs: eigenvalues ascending, eigenvectors over the input (column rank[i] = V[:, i])
    if (a.E)
      for (int i = tid; i < n; i += NT) a.E[eoff + rank[i]] = lam[i];
    if (a.want_v)
      for (int e = tid; e < n * n; e += NT) {
        const int row = e % n, col = e / n;
        H[row + (int64_t)rank[col] * n] = V[e];
      }
    __syncthreads();
    // restore the slab order for the next matrix
    V = slab;
    W = slab + NMAX * NMAX;
    G = slab + 2 * NMAX * NMAX;
  }
}

}  // namespace epb

namespace epb {

// One instance of the persistent solver over a (uniform or varlen) batch: orders in (n_lo, NMAX] are solved,
// the others left to the other kernels. The L2 scratch slab (3 NMAX^2 complex doubles per CTA) shares the
// workspace slot of every instance; its size is that of the largest instance, so that the slot is not
// reallocated between the launches of one varlen batch (which may be captured in a graph).
template <int NMAX, int NT, int MINB>
static int launch_big(epb_ctx* ctx, BigArgs a, int64_t batch) {
  using SM = BigSmem<NMAX>;
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(eigh_big_kernel<NMAX, NT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  SM::TOTAL));
    attr = true;
  }
  const int64_t grid = std::min<int64_t>((int64_t)ctx->sm_count * MINB, batch);
  // largest slab of the instances below: <96, 512, 1>, <80, 256, 2>, <64, 256, 2>, <48, 256, 2>, <32, 128, 4>
  const size_t per_sm = std::max<size_t>({(size_t)3 * 96 * 96, (size_t)3 * 80 * 80 * 2, (size_t)3 * 64 * 64 * 2,
                                          (size_t)3 * 48 * 48 * 2, (size_t)3 * 32 * 32 * 4});
  const size_t slab_max = per_sm * sizeof(double2) * (size_t)ctx->sm_count;
  const size_t slab = (size_t)3 * NMAX * NMAX * sizeof(double2) * (size_t)grid;
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EIGH_BIG, (slab > slab_max ? slab : slab_max) + 256, &ws));
  a.scratch = (double2*)((uint8_t*)ws + 256);
  a.counter = (unsigned long long*)ws;
  EPB_CUDA(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), ctx->stream));
  prof_begin(ctx, EPB_PROF_EIGH);
  eigh_big_kernel<NMAX, NT, MINB><<<(unsigned)grid, NT, SM::TOTAL, ctx->stream>>>(a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Launch the order-65..96 solver over a (uniform or varlen) batch; matrices of order <= n_lo are
// left to the other kernels. Status words as in the other eigensolvers.
int eigh_big_launch(epb_ctx* ctx, double2* A, const int64_t* a_off, const int32_t* nvec, int n_uniform, int64_t batch,
                    double* E, const int64_t* e_off, bool want_v, int n_lo, int prec, int* nonconv, int* badsize) {
  if (batch == 0) return EPB_OK;
  BigArgs a{};
  a.A = A;
  a.a_off = a_off;
  a.nvec = nvec;
  a.n_uniform = n_uniform;
  a.batch = batch;
  a.E = E;
  a.e_off = e_off;
  a.want_v = want_v ? 1 : 0;
  a.max_sweeps = 20;
  a.refine = prec == EPB_PREC_FP64 ? 3 : 2;
  a.n_lo = n_lo;
  a.nonconv = nonconv;
  a.badsize = badsize;
  // orders up to 80 on a two-CTA-per-SM instance (106 KB of shared memory each), 81..96 on one 512-thread
  // CTA per SM; a uniform batch takes the one instance that covers its order
  if (nvec == nullptr) {
    if (n_uniform <= 80) return launch_big<80, 256, 2>(ctx, a, batch);
    return launch_big<BIG_NMAX, 512, 1>(ctx, a, batch);
  }
  const int st = launch_big<80, 256, 2>(ctx, a, batch);
  if (st != EPB_OK) return st;
  a.n_lo = std::max(n_lo, 80);
  return launch_big<BIG_NMAX, 512, 1>(ctx, a, batch);
}

// The same solver for the mixed-precision classes below 65 (c128 in and out): orders (n_lo, n_hi] with
// n_hi = 32, 48 or 64 on instances sized for them -- 18, 40 and 69 KB of shared memory, four 128-thread,
// two 256-thread and two 256-thread CTAs per SM. (The shared-memory FP64 Rayleigh-Ritz solver of
// epb_eigh.cu keeps H, V and S in FP64 in shared memory: 51 KB per matrix at order 32, 111 KB at 48,
// 200 KB at 64, i.e. 4, 2 and 1 matrices per SM.)
int eigh_mid_launch(epb_ctx* ctx, double2* A, const int64_t* a_off, const int32_t* nvec, int n_uniform, int64_t batch,
                    double* E, const int64_t* e_off, bool want_v, int n_lo, int n_hi, int* nonconv, int* badsize) {
  if (batch == 0) return EPB_OK;
  BigArgs a{};
  a.A = A;
  a.a_off = a_off;
  a.nvec = nvec;
  a.n_uniform = n_uniform;
  a.batch = batch;
  a.E = E;
  a.e_off = e_off;
  a.want_v = want_v ? 1 : 0;
  a.max_sweeps = 20;
  a.refine = 2;
  a.n_lo = n_lo;
  a.nonconv = nonconv;
  a.badsize = badsize;
  if (n_hi <= 32) return launch_big<32, 128, 4>(ctx, a, batch);
  if (n_hi <= 48) return launch_big<48, 256, 2>(ctx, a, batch);
  return launch_big<64, 256, 2>(ctx, a, batch);
}

// Any instance of the solver for the orders (n_lo, n_hi] of a (uniform or varlen) batch: inst = 32, 48, 64,
// 80 or 96 picks the instance (the largest order it holds), refine the FP64 refinement iterations (2 mixed, 3
// FP64). Used by the varlen size classes and their autotuner.
int eigh_l2_launch(epb_ctx* ctx, double2* A, const int64_t* a_off, const int32_t* nvec, int n_uniform, int64_t batch,
                   double* E, const int64_t* e_off, bool want_v, int n_lo, int n_hi, int inst, int refine,
                   int* nonconv, int* badsize) {
  if (batch == 0) return EPB_OK;
  BigArgs a{};
  a.A = A;
  a.a_off = a_off;
  a.nvec = nvec;
  a.n_uniform = n_uniform;
  a.batch = batch;
  a.E = E;
  a.e_off = e_off;
  a.want_v = want_v ? 1 : 0;
  a.max_sweeps = 20;
  a.refine = refine;
  a.n_lo = n_lo;
  a.n_hi = n_hi;
  a.nonconv = nonconv;
  a.badsize = badsize;
  switch (inst) {
    case 32: return launch_big<32, 128, 4>(ctx, a, batch);
    case 48: return launch_big<48, 256, 2>(ctx, a, batch);
    case 64: return launch_big<64, 256, 2>(ctx, a, batch);
    case 80: return launch_big<80, 256, 2>(ctx, a, batch);
    default: return launch_big<BIG_NMAX, 512, 1>(ctx, a, batch);
  }
}

}  // namespace epb
