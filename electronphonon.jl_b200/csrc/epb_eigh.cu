// Batched Hermitian eigensolver: cyclic two-sided Jacobi with round-robin parallel ordering.
//
// Replaces eigvals_batched / eigen_batched (ext/ElectronPhononCUDAExt.jl:80-115, which calls
// cuSOLVER heevjBatched; CPU method src/wannier_to_bloch_batched.jl:30-65). One "team" (a warp for
// n <= 32, four warps for n <= 64) owns one matrix in shared memory at a time and loops over the
// batch. Each round rotates n/2 disjoint (p, q) pairs at once:
//     t = sign(tau) / (|tau| + sqrt(1 + tau^2)),  tau = (a_qq - a_pp) / (2 |a_pq|),
//     J = [[c, s e^{i phi}], [-s e^{-i phi}, c]] on (p, q),  a_pq = |a_pq| e^{i phi},
// applied as A <- A J (columns), A <- J^H A (rows), V <- V J.
// A rotation is skipped when |a_pq| <= eps * ||A||_F / n; a sweep with no rotation ends the solve.
//
// Precision modes:
//   EPB_PREC_FP64  : the whole solve in FP64.
//   EPB_PREC_MIXED : the solve in FP32, then one FP64 refinement per matrix: modified Gram-Schmidt
//                    of the FP32 vectors, S = V^H H V in FP64 (H re-read in FP64), a thresholded
//                    FP64 Jacobi on the nearly diagonal S (this re-orthogonalises near-degenerate
//                    clusters, whose FP32 vectors are only defined up to a rotation), V <- V Q.
#include <algorithm>
#include <cstring>

#include "epb_eigh16.cuh"
#include "epb_jacobi.cuh"

namespace epb {

struct EighArgs {
  double2* A;
  const int64_t* a_off;  // nullptr: uniform, offset b*n*n
  const int32_t* nvec;   // nullptr: uniform n
  int n_uniform;
  int64_t batch;
  double* E;
  const int64_t* e_off;  // nullptr: b*n
  int want_v;
  int max_sweeps;
  int* nonconv;          // device counter of matrices that hit the sweep limit
  int* badsize;          // device counter of matrices whose order exceeds the kernel's maximum
  const double* mass;    // phonon mode: non-null => mass scaling + omega = sign sqrt
  const float* Hp;       // mixed kernel only: packed FP32 Hermitian input (n*n floats per matrix:
                         // Re H_ij for i <= j then Im H_ij for i < j, both column by column)
  float2* U32;           // mixed kernel only: eigenvectors as complex64 (n x n per matrix)
  int n_lo;              // varlen size classes: orders <= n_lo belong to other kernels (skipped silently);
  int skip_hi;           // nonzero: orders above NMAX are skipped silently too (the caller counts bad orders)
};

// Matrix order outside this kernel's class: skip; count only orders that no kernel handles.
__device__ __forceinline__ bool eigh_skip(const EighArgs& a, int n, int nmax, int tid) {
  if (n >= 1 && n <= nmax && n > a.n_lo) return false;
  const bool bad = a.skip_hi == 0 && (n < 0 || n > nmax);
  if (bad && tid == 0) atomicAdd(a.badsize, 1);
  return true;
}

// Shared memory layout per team (elements of the solve type T):
//   A: n x (n+1) [padded], V: n x n, plus RotParam[npair] and a flag.
template <typename T, int TEAM, int NMAX>
__global__ void eigh_kernel(EighArgs a) {
  using C = typename cplx<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TEAMS = (TEAM == 32) ? 4 : 1;  // teams per block
  const int team = threadIdx.x / TEAM;
  const int tid = threadIdx.x % TEAM;
  constexpr int LDA = NMAX + 1;
  // per-team region
  size_t per_team = sizeof(C) * (NMAX * LDA + NMAX * NMAX) + sizeof(RotParam<T>) * (NMAX / 2 + 1) + 16;
  per_team = (per_team + 15) & ~size_t(15);
  unsigned char* base = smem_raw + team * per_team;
  C* As = reinterpret_cast<C*>(base);
  C* Vs = As + NMAX * LDA;
  RotParam<T>* prm = reinterpret_cast<RotParam<T>*>(Vs + NMAX * NMAX);
  int* flag = reinterpret_cast<int*>(prm + NMAX / 2 + 1);

  const int64_t team_global = (int64_t)blockIdx.x * TEAMS + team;
  const int64_t nteams = (int64_t)gridDim.x * TEAMS;
  for (int64_t b = team_global; b < a.batch; b += nteams) {
    const int n = a.nvec ? a.nvec[b] : a.n_uniform;
    if (eigh_skip(a, n, NMAX, tid)) continue;
    const int64_t aoff = a.a_off ? a.a_off[b] : b * (int64_t)n * n;
    const int64_t eoff = a.e_off ? a.e_off[b] : b * (int64_t)n;
    double2* Ag = a.A + aoff;
    const int lda = n + 1;
    // load upper triangle, mirror to the lower (Hermitian from 'U'), optional mass scaling
    T fro2 = 0;
    for (int e = tid; e < n * n; e += TEAM) {
      int i = e % n, j = e / n;
      double2 v;
      if (i <= j) {
        v = Ag[i + (int64_t)j * n];
      } else {
        double2 u = Ag[j + (int64_t)i * n];
        v = make_double2(u.x, -u.y);
      }
      if (i == j) v.y = 0.0;
      if (a.mass) {
        double s = 1.0 / (sqrt(a.mass[i]) * sqrt(a.mass[j]));
        v.x *= s;
        v.y *= s;
      }
      As[i + j * lda] = mk2((T)v.x, (T)v.y);
      Vs[i + j * n] = mk2(T(i == j ? 1 : 0), T(0));
      fro2 += (T)(v.x * v.x + v.y * v.y);
    }
    // team reduction of ||A||_F^2 through the flag slot area (use warp shuffles per warp)
    for (int o = 16; o > 0; o >>= 1) fro2 += __shfl_xor_sync(0xffffffffu, fro2, o);
    __shared__ T red[TEAMS * (TEAM / 32)];
    if ((tid & 31) == 0) red[team * (TEAM / 32) + tid / 32] = fro2;
    team_sync<TEAM>();
    T tot = 0;
    for (int w = 0; w < TEAM / 32; ++w) tot += red[team * (TEAM / 32) + w];
    team_sync<TEAM>();
    const T eps = sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920929e-07);
    const T thr = eps * sqrt(tot) / T(n > 0 ? n : 1);
    int sweeps = jacobi_team<T, TEAM>(As, lda, Vs, n, n, a.want_v != 0, prm, flag, thr, a.max_sweeps);
    if (sweeps >= a.max_sweeps && tid == 0) atomicAdd(a.nonconv, 1);
    // sort eigenvalues ascending (rank by value, ties by index) and write out
    for (int i = tid; i < n; i += TEAM) {
      T ei = As[i + i * lda].x;
      int rank = 0;
      for (int j = 0; j < n; ++j) {
        T ej = As[j + j * lda].x;
        rank += (ej < ei) || (ej == ei && j < i);
      }
      double ev = (double)ei;
      if (a.mass) ev = ev >= 0 ? sqrt(ev) : -sqrt(-ev);
      if (a.E) a.E[eoff + rank] = ev;
      // stash rank in the (now unused) imaginary part of the diagonal
      As[i + i * lda].y = (T)rank;
    }
    team_sync<TEAM>();
    if (a.want_v) {
      for (int e = tid; e < n * n; e += TEAM) {
        int row = e % n, col = e / n;
        int rank = (int)As[col + col * lda].y;
        C v = Vs[row + col * n];
        double2 o = make_double2((double)v.x, (double)v.y);
        if (a.mass) {
          double s = 1.0 / sqrt(a.mass[row]);
          o.x *= s;
          o.y *= s;
        }
        Ag[row + (int64_t)rank * n] = o;
      }
    }
    team_sync<TEAM>();
  }
}

// ---------------------------------------------------------------------------------------------
// Mixed precision: FP32 solve, FP64 refinement (see file header).
template <int TEAM, int NMAX>
__global__ void eigh_mixed_kernel(EighArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TEAMS = (TEAM == 32) ? 4 : 1;
  const int team = threadIdx.x / TEAM;
  const int tid = threadIdx.x % TEAM;
  constexpr int LDA = NMAX + 1;
  // per team: H64 (NMAX x LDA double2) | V64 (NMAX x LDA double2) | region R (max of FP32 solve
  // buffers and S64) | params
  constexpr size_t h64 = sizeof(double2) * NMAX * LDA;
  constexpr size_t f32 = sizeof(float2) * (NMAX * LDA + NMAX * NMAX);
  constexpr size_t regR = (h64 > f32 ? h64 : f32);
  constexpr size_t prmb = sizeof(RotParam<double>) * (NMAX / 2 + 1) + 16;
  constexpr size_t per_team = ((2 * h64 + regR + prmb) + 15) & ~size_t(15);
  unsigned char* base = smem_raw + team * per_team;
  double2* H = reinterpret_cast<double2*>(base);
  double2* V = reinterpret_cast<double2*>(base + h64);
  unsigned char* R = base + 2 * h64;
  float2* A32 = reinterpret_cast<float2*>(R);
  float2* V32 = A32 + NMAX * LDA;
  double2* S = reinterpret_cast<double2*>(R);
  RotParam<double>* prm64 = reinterpret_cast<RotParam<double>*>(base + 2 * h64 + regR);
  RotParam<float>* prm32 = reinterpret_cast<RotParam<float>*>(prm64);
  int* flag = reinterpret_cast<int*>(prm64 + NMAX / 2 + 1);
  __shared__ double red[TEAMS * (TEAM / 32)];

  const int64_t team_global = (int64_t)blockIdx.x * TEAMS + team;
  const int64_t nteams = (int64_t)gridDim.x * TEAMS;
  for (int64_t b = team_global; b < a.batch; b += nteams) {
    const int n = a.nvec ? a.nvec[b] : a.n_uniform;
    if (eigh_skip(a, n, NMAX, tid)) continue;
    const int64_t aoff = a.a_off ? a.a_off[b] : b * (int64_t)n * n;
    const int64_t eoff = a.e_off ? a.e_off[b] : b * (int64_t)n;
    double2* Ag = a.A ? a.A + aoff : nullptr;
    const float* Hp = a.Hp ? a.Hp + b * (int64_t)n * n : nullptr;
    const int lda = n + 1;
    const int nre = n * (n + 1) / 2;
    double fro2 = 0;
    for (int e = tid; e < n * n; e += TEAM) {
      int i = e % n, j = e / n;
      double2 v;
      if (Hp) {
        int ii = i <= j ? i : j, jj = i <= j ? j : i;
        double re = Hp[jj * (jj + 1) / 2 + ii];
        double im = ii < jj ? Hp[nre + jj * (jj - 1) / 2 + ii] : 0.0;
        v = make_double2(re, i <= j ? im : -im);
      } else if (i <= j) {
        v = Ag[i + (int64_t)j * n];
      } else {
        double2 u = Ag[j + (int64_t)i * n];
        v = make_double2(u.x, -u.y);
      }
      if (i == j) v.y = 0.0;
      if (a.mass) {
        double s = 1.0 / (sqrt(a.mass[i]) * sqrt(a.mass[j]));
        v.x *= s;
        v.y *= s;
      }
      H[i + j * lda] = v;
      A32[i + j * lda] = make_float2((float)v.x, (float)v.y);
      V32[i + j * n] = make_float2(i == j ? 1.f : 0.f, 0.f);
      fro2 += v.x * v.x + v.y * v.y;
    }
    for (int o = 16; o > 0; o >>= 1) fro2 += __shfl_xor_sync(0xffffffffu, fro2, o);
    if ((tid & 31) == 0) red[team * (TEAM / 32) + tid / 32] = fro2;
    team_sync<TEAM>();
    double tot = 0;
    for (int w = 0; w < TEAM / 32; ++w) tot += red[team * (TEAM / 32) + w];
    team_sync<TEAM>();
    const double fro = sqrt(tot);
    // FP32 stop at 8 eps32 x the RMS eigenvalue (rounding of degenerate pairs stays below it); the FP64
    // stage below supplies the accuracy
    int sw = jacobi_team<float, TEAM>(A32, lda, V32, n, n, true, prm32, flag,
                                      8.f * 1.1920929e-07f * (float)(fro / sqrt((double)n)), a.max_sweeps);
    if (sw >= a.max_sweeps && tid == 0) atomicAdd(a.nonconv, 1);
    // V64 <- V32, then modified Gram-Schmidt (column by column)
    for (int e = tid; e < n * n; e += TEAM) {
      int i = e % n, j = e / n;
      float2 v = V32[i + j * n];
      V[i + j * lda] = make_double2(v.x, v.y);
    }
    team_sync<TEAM>();
    // Modified Gram-Schmidt, one barrier per column: every warp forms the norm of column j itself (lanes
    // over the rows, butterfly sum, the same order in every warp), the projections use the unnormalised
    // column j with 1 / |v_j|^2, and column j is scaled in the next column's phase, where nobody reads it.
    {
      const int lane = tid & 31;
      double inv_prev = 1.0;
      for (int j = 0; j < n; ++j) {
        double s2 = 0.0;
        for (int i = lane; i < n; i += 32) s2 += V[i + j * lda].x * V[i + j * lda].x + V[i + j * lda].y * V[i + j * lda].y;
        for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        const double inv2 = 1.0 / s2;
        if (j > 0)
          for (int i = tid; i < n; i += TEAM) {
            V[i + (j - 1) * lda].x *= inv_prev;
            V[i + (j - 1) * lda].y *= inv_prev;
          }
        // project column j out of columns > j
        for (int c = j + 1 + tid; c < n; c += TEAM) {
          double2 d = make_double2(0, 0);
          for (int i = 0; i < n; ++i) cfma_conj(d, V[i + j * lda], V[i + c * lda]);
          d.x *= inv2;
          d.y *= inv2;
          for (int i = 0; i < n; ++i) {
            double2 vj = V[i + j * lda];
            V[i + c * lda].x -= d.x * vj.x - d.y * vj.y;
            V[i + c * lda].y -= d.x * vj.y + d.y * vj.x;
          }
        }
        inv_prev = sqrt(inv2);
        team_sync<TEAM>();
      }
      for (int i = tid; i < n; i += TEAM) {
        V[i + (n - 1) * lda].x *= inv_prev;
        V[i + (n - 1) * lda].y *= inv_prev;
      }
      team_sync<TEAM>();
    }
    // S = V^H (H V): compute W = H V into S's region first column-wise? Use S as W then overwrite.
    // W column c (thread per (row, col))
    for (int e = tid; e < n * n; e += TEAM) {
      int i = e % n, c = e / n;
      double2 w = make_double2(0, 0);
      for (int k = 0; k < n; ++k) cfma(w, H[i + k * lda], V[k + c * lda]);
      S[i + c * lda] = w;
    }
    team_sync<TEAM>();
    // H is no longer needed: compute S = V^H W into H's region
    for (int e = tid; e < n * n; e += TEAM) {
      int i = e % n, c = e / n;
      double2 s = make_double2(0, 0);
      for (int k = 0; k < n; ++k) cfma_conj(s, V[k + i * lda], S[k + c * lda]);
      H[i + c * lda] = s;
    }
    team_sync<TEAM>();
    // symmetrise S and reset the rotation accumulator Q (in S's region, ld = n)
    for (int e = tid; e < n * n; e += TEAM) {
      int i = e % n, c = e / n;
      if (i < c) {
        double2 u = H[i + c * lda], l = H[c + i * lda];
        double2 m2 = make_double2(0.5 * (u.x + l.x), 0.5 * (u.y - l.y));
        H[i + c * lda] = m2;
        H[c + i * lda] = make_double2(m2.x, -m2.y);
      } else if (i == c) {
        H[i + i * lda].y = 0.0;
      }
      S[i + c * n] = make_double2(i == c ? 1.0 : 0.0, 0.0);
    }
    team_sync<TEAM>();
    jacobi_team<double, TEAM>(H, lda, S, n, n, true, prm64, flag, 2.220446049250313e-16 * fro / n, 8);
    // eigenvalue ranks, then the eigenvectors V Q straight into their sorted output columns (one thread per
    // output entry; Q is the rotation accumulated in S)
    for (int i = tid; i < n; i += TEAM) {
      double ei = H[i + i * lda].x;
      int rank = 0;
      for (int j = 0; j < n; ++j) {
        double ej = H[j + j * lda].x;
        rank += (ej < ei) || (ej == ei && j < i);
      }
      double ev = ei;
      if (a.mass) ev = ev >= 0 ? sqrt(ev) : -sqrt(-ev);
      if (a.E) a.E[eoff + rank] = ev;
      H[i + i * lda].y = (double)rank;
    }
    team_sync<TEAM>();
    if (a.want_v) {
      for (int e = tid; e < n * n; e += TEAM) {
        const int row = e % n, col = e / n;
        const int rank = (int)H[col + col * lda].y;
        double2 o = make_double2(0, 0);
        for (int k = 0; k < n; ++k) cfma(o, V[row + k * lda], S[k + col * n]);
        if (a.mass) {
          double sc = 1.0 / sqrt(a.mass[row]);
          o.x *= sc;
          o.y *= sc;
        }
        if (a.U32)
          a.U32[b * (int64_t)n * n + row + (int64_t)rank * n] = make_float2((float)o.x, (float)o.y);
        else
          Ag[row + (int64_t)rank * n] = o;
      }
    }
    team_sync<TEAM>();
  }
}

template <typename T, int TEAM, int NMAX>
static size_t eigh_smem() {
  using C = typename cplx<T>::type;
  size_t per_team = sizeof(C) * (NMAX * (NMAX + 1) + NMAX * NMAX) + sizeof(RotParam<T>) * (NMAX / 2 + 1) + 16;
  per_team = (per_team + 15) & ~size_t(15);
  return per_team * ((TEAM == 32) ? 4 : 1);
}

template <int TEAM, int NMAX>
static size_t eigh_mixed_smem() {
  constexpr int LDA = NMAX + 1;
  size_t h64 = sizeof(double2) * NMAX * LDA;
  size_t f32 = sizeof(float2) * (NMAX * LDA + NMAX * NMAX);
  size_t regR = h64 > f32 ? h64 : f32;
  size_t prmb = sizeof(RotParam<double>) * (NMAX / 2 + 1) + 16;
  size_t per_team = ((2 * h64 + regR + prmb) + 15) & ~size_t(15);
  return per_team * ((TEAM == 32) ? 4 : 1);
}

template <typename Kern>
static int launch_eigh(epb_ctx* ctx, Kern kern, size_t smem, int threads, EighArgs& a) {
  EPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int teams_per_block = threads == 32 * 4 ? 4 : 1;
  int per_sm = 0;
  EPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
  if (per_sm < 1) {
    set_error("eigensolver: shared memory request %zu bytes does not fit", smem);
    return EPB_ERR_UNSUPPORTED;
  }
  int64_t blocks_needed = cdiv(a.batch, teams_per_block);
  int64_t blocks = (int64_t)per_sm * ctx->sm_count;
  if (blocks > blocks_needed) blocks = blocks_needed;
  if (blocks < 1) blocks = 1;
  prof_begin(ctx, EPB_PROF_EIGH);
  kern<<<(unsigned)blocks, threads, smem, ctx->stream>>>(a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Dispatch on max order and precision. The mixed solver of orders 33..48 has its own instance: its shared
// memory (111 KB per team) lets two teams share an SM, against one at orders up to 64.
int eigh_dispatch(epb_ctx* ctx, EighArgs& a, int nmax, int prec) {
  if (prec == EPB_PREC_FP64) {
    if (nmax <= 16)
      return launch_eigh(ctx, eigh_kernel<double, 32, 16>, eigh_smem<double, 32, 16>(), 128, a);
    if (nmax <= 32)
      return launch_eigh(ctx, eigh_kernel<double, 32, 32>, eigh_smem<double, 32, 32>(), 128, a);
    if (nmax <= 64)
      return launch_eigh(ctx, eigh_kernel<double, 128, 64>, eigh_smem<double, 128, 64>(), 128, a);
  } else if (prec == EPB_PREC_MIXED) {
    if (nmax <= 16)
      return launch_eigh(ctx, eigh_mixed_kernel<32, 16>, eigh_mixed_smem<32, 16>(), 128, a);
    if (nmax <= 32)
      return launch_eigh(ctx, eigh_mixed_kernel<32, 32>, eigh_mixed_smem<32, 32>(), 128, a);
    if (nmax <= 48)
      return launch_eigh(ctx, eigh_mixed_kernel<128, 48>, eigh_mixed_smem<128, 48>(), 128, a);
    if (nmax <= 64)
      return launch_eigh(ctx, eigh_mixed_kernel<128, 64>, eigh_mixed_smem<128, 64>(), 128, a);
  } else {
    set_error("eigensolver: unknown precision mode %d", prec);
    return EPB_ERR_ARG;
  }
  set_error("eigensolver: matrix order %d > 64 not supported here (orders up to 64 on this path)", nmax);
  return EPB_ERR_ARG;
}

int eigh_check(epb_ctx* ctx);

// Offsets of the listed matrices for the FP64 slow path.
__global__ void flag_offsets_kernel(const int64_t* __restrict__ list, const int* __restrict__ count, int64_t n,
                                    int64_t* __restrict__ a_off, int64_t* __restrict__ e_off, int32_t* __restrict__ nvec,
                                    int64_t cap) {
  int64_t c = *count;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < c) {
      a_off[i] = list[i] * n * n;
      e_off[i] = list[i] * n;
      nvec[i] = (int32_t)n;
    } else {
      nvec[i] = 0;  // unused slots: order 0 is skipped by the kernel without being reported
    }
  }
}

// Uniform batches of order <= 16 go to the register-resident one-sided Jacobi (epb_eigh16.cu).
// With c128 in/out (the public API) the FP64 refinement runs twice, and matrices with a
// near-degenerate pair outside first-order validity (planted clusters) are re-solved by the FP64
// two-sided Jacobi, which reads the untouched input.
static int eigh_small(epb_ctx* ctx, const EighArgs& a, int prec) {
  Eigh16Args b{};
  b.A = a.A;
  b.Hp = a.Hp;
  b.U64 = a.want_v && !a.U32 ? a.A : nullptr;
  b.U32 = a.U32;
  b.E = a.E;
  b.mass = a.mass;
  b.n = a.n_uniform;
  b.batch = a.batch;
  b.max_sweeps = prec == EPB_PREC_FP64 ? 30 : 20;
  b.nonconv = ctx->dstat + 0;
  b.refine = a.U32 ? 1 : 2;
  b.angle_stop = a.U32 ? 1e-2f : 1e-4f;  // the pass's packed path (complex64 output) as in eigh16_mixed_jacobi
  const bool slow_path = prec == EPB_PREC_MIXED && !a.Hp && a.A;
  int64_t* list = nullptr;
  if (prec == EPB_PREC_MIXED) {
    // workspace: FP32 eigenvectors (16 x 16 per matrix), then the slow-path list and offsets
    const size_t v32 = (size_t)a.batch * 16 * 16 * sizeof(float2);
    void* ws = nullptr;
    EPB_TRY(ws_get(ctx, EPB_WS_EIGH, v32 + (slow_path ? (size_t)a.batch * 32 : 0) + 256, &ws));
    b.V32 = (float2*)ws;
    if (slow_path) {
      list = (int64_t*)((char*)ws + ((v32 + 255) & ~size_t(255)));
      b.flag_list = list;
      b.flag_count = ctx->dstat + 4;
      EPB_CUDA(cudaMemsetAsync(b.flag_count, 0, sizeof(int), ctx->stream));
    }
  }
  EPB_TRY(eigh16_launch(ctx, b, prec == EPB_PREC_MIXED));
  if (!slow_path) return EPB_OK;
  // slow path on the (rare) flagged matrices: capacity = batch, count read on the device
  int64_t* a_off = list + a.batch;
  int64_t* e_off = a_off + a.batch;
  int32_t* nvec = (int32_t*)(e_off + a.batch);
  flag_offsets_kernel<<<(unsigned)cdiv(a.batch, 256), 256, 0, ctx->stream>>>(list, b.flag_count, a.n_uniform,
                                                                            a_off, e_off, nvec, a.batch);
  EPB_LAUNCH_CHECK();
  int* h = (int*)ctx->pinned;
  EPB_CUDA(cudaMemcpyAsync(h, b.flag_count, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*h == 0) return EPB_OK;
  EighArgs s{};
  s.A = a.A;
  s.a_off = a_off;
  s.nvec = nvec;
  s.batch = *h;
  s.E = a.E;
  s.e_off = e_off;
  s.want_v = a.want_v;
  s.mass = a.mass;
  s.nonconv = ctx->dstat + 0;
  s.badsize = ctx->dstat + 1;
  s.max_sweeps = 30;
  return eigh_dispatch(ctx, s, 16, EPB_PREC_FP64);
}

int eigh_big_launch(epb_ctx* ctx, double2* A, const int64_t* a_off, const int32_t* nvec, int n_uniform, int64_t batch,
                    double* E, const int64_t* e_off, bool want_v, int n_lo, int prec, int* nonconv, int* badsize);
int eigh_mid_launch(epb_ctx* ctx, double2* A, const int64_t* a_off, const int32_t* nvec, int n_uniform, int64_t batch,
                    double* E, const int64_t* e_off, bool want_v, int n_lo, int n_hi, int* nonconv, int* badsize);
int eigh_l2_launch(epb_ctx* ctx, double2* A, const int64_t* a_off, const int32_t* nvec, int n_uniform, int64_t batch,
                   double* E, const int64_t* e_off, bool want_v, int n_lo, int n_hi, int inst, int refine,
                   int* nonconv, int* badsize);
bool tune_lookup(const std::vector<std::pair<std::string, int64_t>>& kv, const std::string& key, int64_t* value);
void tune_store(std::vector<std::pair<std::string, int64_t>>& kv, const std::string& key, int64_t value);

// Orders of a varlen batch outside 0..96 (no kernel handles them; order 0 is an empty matrix).
__global__ void eigh_badorder_kernel(const int32_t* __restrict__ nvec, int64_t batch, int* __restrict__ badsize) {
  int c = 0;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < batch; b += (int64_t)gridDim.x * blockDim.x) {
    const int n = nvec[b];
    c += n < 0 || n > 96;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(badsize, c);
}

// Size classes of a mixed-precision varlen batch with two candidate kernels each, (lo, hi]: candidate 0 is
// the shared-memory FP64 Rayleigh-Ritz solver (orders <= 64) or, for 65..80, the 512-thread instance of the
// L2-scratch solver; candidate 1 the L2-scratch instance sized for the class.
constexpr int VL_NCLS = 4;
constexpr int VL_LO[VL_NCLS] = {16, 32, 48, 64}, VL_HI[VL_NCLS] = {32, 48, 64, 80};

static std::string varlen_key(int c) {
  char key[64];
  snprintf(key, sizeof(key), "eigh_varlen/%d/%d/%d", VL_LO[c], VL_HI[c], (int)EPB_PREC_MIXED);
  return key;
}

// Candidate `v` of mixed class c over the whole batch (the kernel takes the matrices of its class only).
static int varlen_class(epb_ctx* ctx, const EighArgs& a, int c, int v) {
  if (v == 0 && VL_HI[c] <= 64) {
    EighArgs s = a;
    s.n_lo = VL_LO[c];
    s.skip_hi = 1;
    return eigh_dispatch(ctx, s, VL_HI[c], EPB_PREC_MIXED);
  }
  const int inst = v == 0 ? 96 : VL_HI[c];
  return eigh_l2_launch(ctx, a.A, a.a_off, a.nvec, 0, a.batch, a.E, a.e_off, a.want_v != 0, VL_LO[c], VL_HI[c], inst, 2,
                        a.nonconv, a.badsize);
}

// The varlen batch without any host read-back (capturable in a CUDA graph): every size class kernel runs
// over the whole batch, taking the matrices of its class and skipping the others -- FP64: orders 1..16,
// 17..32, 33..64 on the shared-memory Jacobi, 65..96 on the persistent L2-scratch solver; mixed: 1..16 on
// the register Jacobi, then for 17..32, 33..48, 49..64, 65..80 the candidate in the context's tuning table
// (epb_eigh_varlen times them on the first batch; default the L2-scratch instance), 81..96 on the
// L2-scratch solver. Orders outside 0..96 are counted into the status words that eigh_check reads.
int eigh_varlen_async(epb_ctx* ctx, EighArgs& a, int prec) {
  if (a.batch == 0) return EPB_OK;
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "eigensolver: unknown precision mode %d", prec);
  EPB_CHECK_ARG(!a.mass, "eigensolver: varlen batches take no masses");
  a.nonconv = ctx->dstat + 0;
  a.badsize = ctx->dstat + 1;
  a.max_sweeps = prec == EPB_PREC_FP64 ? 30 : 20;
  eigh_badorder_kernel<<<(unsigned)std::min<int64_t>(cdiv(a.batch, 256), (int64_t)ctx->sm_count * 8), 256, 0,
                         ctx->stream>>>(a.nvec, a.batch, a.badsize);
  EPB_LAUNCH_CHECK();
  if (prec == EPB_PREC_FP64) {
    const int lo[3] = {0, 16, 32}, hi[3] = {16, 32, 64};
    for (int c = 0; c < 3; ++c) {
      EighArgs s = a;
      s.n_lo = lo[c];
      s.skip_hi = 1;
      EPB_TRY(eigh_dispatch(ctx, s, hi[c], prec));
    }
    return eigh_big_launch(ctx, a.A, a.a_off, a.nvec, 0, a.batch, a.E, a.e_off, a.want_v != 0, 64, prec, a.nonconv,
                           a.badsize);
  }
  {
    EighArgs s = a;
    s.n_lo = 0;
    s.skip_hi = 1;
    EPB_TRY(eigh_dispatch(ctx, s, 16, prec));
  }
  for (int c = 0; c < VL_NCLS; ++c) {
    int64_t v = 1;
    tune_lookup(ctx->tuned, varlen_key(c), &v);
    EPB_TRY(varlen_class(ctx, a, c, (int)v));
  }
  return eigh_l2_launch(ctx, a.A, a.a_off, a.nvec, 0, a.batch, a.E, a.e_off, a.want_v != 0, 80, 96, 96, 2, a.nonconv,
                        a.badsize);
}

// max over the batch of a_off[b] + n_b^2 and e_off[b] + n_b: the extents of A (complex entries) and E
__global__ void varlen_extent_kernel(const int64_t* __restrict__ a_off, const int64_t* __restrict__ e_off,
                                     const int32_t* __restrict__ nvec, int64_t batch, unsigned long long* ext) {
  unsigned long long ea = 0, ee = 0;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < batch; b += (int64_t)gridDim.x * blockDim.x) {
    const int n = nvec[b];
    if (n < 1 || n > 96) continue;
    ea = max(ea, (unsigned long long)(a_off[b] + (int64_t)n * n));
    ee = max(ee, (unsigned long long)(e_off[b] + n));
  }
  for (int o = 16; o > 0; o >>= 1) {
    ea = max(ea, __shfl_xor_sync(0xffffffffu, ea, o));
    ee = max(ee, __shfl_xor_sync(0xffffffffu, ee, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(ext, ea);
    atomicMax(ext + 1, ee);
  }
}

// Autotuner of the mixed varlen classes (synchronous calls only): for every class whose choice is not in
// the context's table, both candidates solve a copy of the first (at most 32768) matrices of the caller's
// batch (the copy restored before each), timed with CUDA events; the faster goes into the table under
// eigh_varlen/<lo>/<hi>/<prec>. Costs two copies of that sample in a workspace and twice its solve time,
// once per context (or never, with an imported table).
static int varlen_tune(epb_ctx* ctx, const EighArgs& a_in) {
  bool need = false;
  int64_t v;
  for (int c = 0; c < VL_NCLS; ++c) need = need || !tune_lookup(ctx->tuned, varlen_key(c), &v);
  if (!need || a_in.batch == 0) return EPB_OK;
  EighArgs a = a_in;
  a.batch = std::min<int64_t>(a.batch, 32768);
  unsigned long long* ext = (unsigned long long*)(ctx->dstat + 20);  // status words 20..23
  EPB_CUDA(cudaMemsetAsync(ext, 0, 2 * sizeof(unsigned long long), ctx->stream));
  varlen_extent_kernel<<<(unsigned)std::min<int64_t>(cdiv(a.batch, 256), (int64_t)ctx->sm_count * 8), 256, 0,
                         ctx->stream>>>(a.a_off, a.e_off, a.nvec, a.batch, ext);
  EPB_LAUNCH_CHECK();
  unsigned long long h[2] = {0, 0};
  EPB_CUDA(cudaMemcpyAsync(h, ext, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  const size_t abytes = (size_t)h[0] * sizeof(double2), ebytes = (size_t)h[1] * sizeof(double);
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS5, 2 * abytes + ebytes + 512, &ws));
  double2* orig = (double2*)ws;
  double2* work = (double2*)((char*)ws + ((abytes + 255) & ~size_t(255)));
  double* ework = (double*)((char*)work + ((abytes + 255) & ~size_t(255)));
  EPB_CUDA(cudaMemcpyAsync(orig, a.A, abytes, cudaMemcpyDeviceToDevice, ctx->stream));
  EighArgs t = a;
  t.A = work;
  t.E = ework;
  t.nonconv = ctx->dstat + 24;  // trial counters, not reported
  t.badsize = ctx->dstat + 25;
  t.max_sweeps = 20;
  cudaEvent_t e0, e1;
  EPB_CUDA(cudaEventCreate(&e0));
  EPB_CUDA(cudaEventCreate(&e1));
  int st = EPB_OK;
  for (int c = 0; c < VL_NCLS && st == EPB_OK; ++c) {
    if (tune_lookup(ctx->tuned, varlen_key(c), &v)) continue;
    float ms[2] = {0.f, 0.f};
    for (int cand = 0; cand < 2 && st == EPB_OK; ++cand) {
      if (cudaMemcpyAsync(work, orig, abytes, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess) st = EPB_ERR_CUDA;
      if (st == EPB_OK) st = cudaEventRecord(e0, ctx->stream) == cudaSuccess ? EPB_OK : EPB_ERR_CUDA;
      if (st == EPB_OK) st = varlen_class(ctx, t, c, cand);
      if (st == EPB_OK) st = cudaEventRecord(e1, ctx->stream) == cudaSuccess ? EPB_OK : EPB_ERR_CUDA;
      if (st == EPB_OK) st = cudaEventSynchronize(e1) == cudaSuccess ? EPB_OK : EPB_ERR_CUDA;
      if (st == EPB_OK) cudaEventElapsedTime(&ms[cand], e0, e1);
    }
    if (st == EPB_OK) tune_store(ctx->tuned, varlen_key(c), ms[1] <= ms[0] ? 1 : 0);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == EPB_ERR_CUDA) set_error("eigensolver autotuner: a copy, launch or event failed");
  return st;
}

int eigh_run(epb_ctx* ctx, EighArgs& a, int nmax, int prec) {
  if (a.batch == 0) return EPB_OK;
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "eigensolver: unknown precision mode %d", prec);
  a.nonconv = ctx->dstat + 0;
  a.badsize = ctx->dstat + 1;
  EPB_CUDA(cudaMemsetAsync(ctx->dstat, 0, 2 * sizeof(int), ctx->stream));
  a.max_sweeps = prec == EPB_PREC_FP64 ? 30 : 20;
  if (!a.nvec) {
    const int n = a.n_uniform;
    if (n <= 16)
      EPB_TRY(eigh_small(ctx, a, prec));
    else if (n <= 64 && prec == EPB_PREC_MIXED && !a.mass && !a.Hp && !a.U32)
      EPB_TRY(eigh_mid_launch(ctx, a.A, nullptr, nullptr, n, a.batch, a.E, nullptr, a.want_v != 0, 0,
                              n <= 32 ? 32 : n <= 48 ? 48 : 64, a.nonconv, a.badsize));
    else if (n <= 64)
      EPB_TRY(eigh_dispatch(ctx, a, n, prec));
    else if (n <= 96) {
      EPB_CHECK_ARG(!a.mass, "eigensolver: phonon (mass-scaled) batches are limited to order 64");
      EPB_TRY(eigh_big_launch(ctx, a.A, nullptr, nullptr, n, a.batch, a.E, nullptr, a.want_v != 0, 0, prec, a.nonconv,
                              a.badsize));
    } else {
      set_error("eigensolver: matrix order %d not supported (orders 1 to 96)", n);
      return EPB_ERR_ARG;
    }
    return eigh_check(ctx);
  }
  // varlen: the class autotuner (first mixed batch of the context), every size class without read-back,
  // then the status words
  (void)nmax;
  if (prec == EPB_PREC_MIXED && !a.mass) EPB_TRY(varlen_tune(ctx, a));
  EPB_CUDA(cudaMemsetAsync(ctx->dstat, 0, 2 * sizeof(int), ctx->stream));
  EPB_TRY(eigh_varlen_async(ctx, a, prec));
  return eigh_check(ctx);
}

// Stream-ordered variant for the pass pipeline: counters accumulate in a context slot until
// eigh_check() reads them back (one sync per pass instead of one per call).
int eigh_async(epb_ctx* ctx, double2* A, int64_t n, int64_t batch, double* E, bool want_v,
               const double* mass, int prec) {
  if (batch == 0) return EPB_OK;
  EighArgs a{};
  a.A = A;
  a.n_uniform = (int)n;
  a.batch = batch;
  a.E = E;
  a.want_v = want_v;
  a.mass = mass;
  a.nonconv = ctx->dstat + 0;
  a.badsize = ctx->dstat + 1;
  a.max_sweeps = prec == EPB_PREC_FP64 ? 30 : 20;
  if (n <= 16) return eigh_small(ctx, a, prec);
  return eigh_dispatch(ctx, a, (int)n, prec);
}

// Mixed-precision eigensolve of packed FP32 Hermitian matrices (the tensor-core H(k+q) output),
// eigenvectors written as complex64, eigenvalues (optional) as FP64. Stream-ordered.
int eigh_mixed_packed(epb_ctx* ctx, const float* Hp, int64_t n, int64_t batch, float2* U, double* E) {
  if (batch == 0) return EPB_OK;
  EighArgs a{};
  a.Hp = Hp;
  a.U32 = U;
  a.n_uniform = (int)n;
  a.batch = batch;
  a.E = E;
  a.want_v = 1;
  a.nonconv = ctx->dstat + 0;
  a.badsize = ctx->dstat + 1;
  a.max_sweeps = 20;
  if (n <= 16) return eigh_small(ctx, a, EPB_PREC_MIXED);
  return eigh_dispatch(ctx, a, (int)n, EPB_PREC_MIXED);
}

// Read back (one sync) and clear the eigensolver status words accumulated since the last check.
int eigh_check(epb_ctx* ctx) {
  int* h = (int*)ctx->pinned;
  EPB_CUDA(cudaMemcpyAsync(h, ctx->dstat, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(ctx->dstat, 0, 2 * sizeof(int), ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h[1] > 0) {
    set_error("eigensolver: %d matrices have an order outside the supported range (skipped)", h[1]);
    return EPB_ERR_ARG;
  }
  if (h[0] > 0) {
    set_error("eigensolver: %d matrices reached the sweep limit", h[0]);
    return EPB_ERR_NOCONVERGE;
  }
  return EPB_OK;
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_eigh_batched(epb_ctx* ctx, double* A, int64_t n, int64_t batch, double* E, char jobz,
                     int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eigh_batched: NULL ctx");
  EPB_CHECK_ARG(n >= 1 && batch >= 0, "epb_eigh_batched: bad n=%lld batch=%lld", (long long)n,
                (long long)batch);
  EPB_CHECK_ARG(jobz == 'N' || jobz == 'V', "epb_eigh_batched: jobz must be 'N' or 'V'");
  EPB_CHECK_ARG(batch == 0 || (A && E), "epb_eigh_batched: NULL buffer");
  EPB_TRY(make_current(ctx));
  EighArgs a{};
  a.A = (double2*)A;
  a.n_uniform = (int)n;
  a.batch = batch;
  a.E = E;
  a.want_v = jobz == 'V';
  return eigh_run(ctx, a, (int)n, prec);
}

int epb_eigh_varlen(epb_ctx* ctx, double* A, const int64_t* a_offset, const int32_t* n,
                    int64_t batch, double* E, const int64_t* e_offset, char jobz, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eigh_varlen: NULL ctx");
  EPB_CHECK_ARG(batch >= 0, "epb_eigh_varlen: batch < 0");
  EPB_CHECK_ARG(batch == 0 || (A && a_offset && n && E && e_offset), "epb_eigh_varlen: NULL buffer");
  EPB_CHECK_ARG(jobz == 'N' || jobz == 'V', "epb_eigh_varlen: jobz must be 'N' or 'V'");
  EPB_TRY(make_current(ctx));
  EighArgs a{};
  a.A = (double2*)A;
  a.a_off = a_offset;
  a.nvec = n;
  a.batch = batch;
  a.E = E;
  a.e_off = e_offset;
  a.want_v = jobz == 'V';
  return eigh_run(ctx, a, 64, prec);
}

int epb_eigh_varlen_async(epb_ctx* ctx, double* A, const int64_t* a_offset, const int32_t* n, int64_t batch, double* E,
                          const int64_t* e_offset, char jobz, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eigh_varlen_async: NULL ctx");
  EPB_CHECK_ARG(batch >= 0, "epb_eigh_varlen_async: batch < 0");
  EPB_CHECK_ARG(batch == 0 || (A && a_offset && n && E && e_offset), "epb_eigh_varlen_async: NULL buffer");
  EPB_CHECK_ARG(jobz == 'N' || jobz == 'V', "epb_eigh_varlen_async: jobz must be 'N' or 'V'");
  EPB_TRY(make_current(ctx));
  EighArgs a{};
  a.A = (double2*)A;
  a.a_off = a_offset;
  a.nvec = n;
  a.batch = batch;
  a.E = E;
  a.e_off = e_offset;
  a.want_v = jobz == 'V';
  return eigh_varlen_async(ctx, a, prec);
}

int epb_eigh_status(epb_ctx* ctx) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eigh_status: NULL ctx");
  EPB_TRY(make_current(ctx));
  return eigh_check(ctx);
}

int epb_ph_eigen_batched(epb_ctx* ctx, double* D, const double* mass, int64_t nm, int64_t nq,
                         double* omega, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && mass, "epb_ph_eigen_batched: NULL argument");
  EPB_CHECK_ARG(nm >= 1 && nq >= 0, "epb_ph_eigen_batched: bad sizes");
  EPB_CHECK_ARG(nq == 0 || (D && omega), "epb_ph_eigen_batched: NULL buffer");
  EPB_TRY(make_current(ctx));
  EighArgs a{};
  a.A = (double2*)D;
  a.n_uniform = (int)nm;
  a.batch = nq;
  a.E = omega;
  a.want_v = 1;
  a.mass = mass;
  return eigh_run(ctx, a, (int)nm, prec);
}

}  // extern "C"
