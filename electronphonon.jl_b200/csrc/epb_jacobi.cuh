// Cyclic two-sided Jacobi for one Hermitian matrix held by a thread team in shared memory (used by
// the batched eigensolvers of epb_eigh.cu and epb_eigh_big.cu).
#pragma once

#include "epb_common.cuh"

namespace epb {

template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if (TEAM == 32)
    __syncwarp();
  else
    __syncthreads();
}

// Round-robin (circle method) pair i of round r for m players (m even); player m-1 is fixed.
__device__ __forceinline__ void rr_pair(int m, int r, int i, int& p, int& q) {
  int a, b;
  if (i == 0) {
    a = m - 1;
    b = r;
  } else {
    a = (r + i) % (m - 1);
    b = (r - i + (m - 1)) % (m - 1);
  }
  p = a < b ? a : b;
  q = a < b ? b : a;
}

template <typename T>
struct RotParam {
  T c, s;
  typename cplx<T>::type e;  // e^{i phi}
  int p, q;                  // p < 0: skip
};

// One full Jacobi solve of the n x n Hermitian matrix in A (column-major, leading dim lda) with
// eigenvectors accumulated into V (leading dim ldv; must hold identity on entry if want_v).
// Returns the number of sweeps used (max_sweeps + 1 if not converged).
template <typename T, int TEAM>
__device__ int jacobi_team(typename cplx<T>::type* A, int lda, typename cplx<T>::type* V, int ldv,
                           int n, bool want_v, RotParam<T>* prm, int* flag, T thr,
                           int max_sweeps) {
  using C = typename cplx<T>::type;
  const int tid = threadIdx.x % TEAM;
  const int m = (n + 1) & ~1;
  const int npair = m / 2;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0) *flag = 0;
    team_sync<TEAM>();
    for (int r = 0; r < m - 1; ++r) {
      for (int i = tid; i < npair; i += TEAM) {
        int p, q;
        rr_pair(m, r, i, p, q);
        RotParam<T> P;
        P.p = -1;
        P.q = q;
        if (q < n) {
          C b = A[p + q * lda];
          T ab = sqrt(b.x * b.x + b.y * b.y);
          if (ab > thr) {
            T a = A[p + p * lda].x, d = A[q + q * lda].x;
            T tau = (d - a) / (T(2) * ab);
            T t;
            if (fabs(tau) > T(1e15))
              t = T(0.5) / tau;
            else
              t = (tau >= T(0) ? T(1) : T(-1)) / (fabs(tau) + sqrt(T(1) + tau * tau));
            T c = T(1) / sqrt(T(1) + t * t);
            P.c = c;
            P.s = t * c;
            P.e = mk2(b.x / ab, b.y / ab);
            P.p = p;
            *flag = 1;
          }
        }
        prm[i] = P;
      }
      team_sync<TEAM>();
      // columns: A <- A J, V <- V J
      for (int task = tid; task < npair * n; task += TEAM) {
        int i = task / n, row = task % n;
        RotParam<T> P = prm[i];
        if (P.p < 0) continue;
        C ap = A[row + P.p * lda], aq = A[row + P.q * lda];
        C ec = mk2(P.e.x, -P.e.y);
        C sp = cmul(ec, aq);
        C sq = cmul(P.e, ap);
        A[row + P.p * lda] = mk2(P.c * ap.x - P.s * sp.x, P.c * ap.y - P.s * sp.y);
        A[row + P.q * lda] = mk2(P.s * sq.x + P.c * aq.x, P.s * sq.y + P.c * aq.y);
        if (want_v) {
          C vp = V[row + P.p * ldv], vq = V[row + P.q * ldv];
          C tp = cmul(ec, vq), tq = cmul(P.e, vp);
          V[row + P.p * ldv] = mk2(P.c * vp.x - P.s * tp.x, P.c * vp.y - P.s * tp.y);
          V[row + P.q * ldv] = mk2(P.s * tq.x + P.c * vq.x, P.s * tq.y + P.c * vq.y);
        }
      }
      team_sync<TEAM>();
      // rows: A <- J^H A
      for (int task = tid; task < npair * n; task += TEAM) {
        int i = task / n, col = task % n;
        RotParam<T> P = prm[i];
        if (P.p < 0) continue;
        C ap = A[P.p + col * lda], aq = A[P.q + col * lda];
        C ec = mk2(P.e.x, -P.e.y);
        C sp = cmul(P.e, aq), sq = cmul(ec, ap);
        A[P.p + col * lda] = mk2(P.c * ap.x - P.s * sp.x, P.c * ap.y - P.s * sp.y);
        A[P.q + col * lda] = mk2(P.s * sq.x + P.c * aq.x, P.s * sq.y + P.c * aq.y);
      }
      team_sync<TEAM>();
    }
    int any = *flag;
    team_sync<TEAM>();
    if (!any) break;
  }
  return sweep;
}

}  // namespace epb
