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
// Returns the number of sweeps used (max_sweeps + 1 if not converged, or if n > 64 TEAM / 32).
template <typename T, int TEAM>
__device__ int jacobi_team(typename cplx<T>::type* A, int lda, typename cplx<T>::type* V, int ldv,
                           int n, bool want_v, RotParam<T>* prm, int* flag, T thr, int max_sweeps) {
  using C = typename cplx<T>::type;
  static_assert(TEAM % 32 == 0, "jacobi_team: the team is whole warps");
  constexpr int NWT = TEAM / 32;  // warps of the team
  const int tid = threadIdx.x % TEAM;
  const int m = (n + 1) & ~1;
  const int npair = m / 2;
  const int lane = tid & 31, wt = tid >> 5;
  const int mine = npair > wt ? (npair - wt + NWT - 1) / NWT : 0;  // pairs of this warp: wt, wt + NWT, ...
  if (npair > 32 * NWT) return max_sweeps + 1;  // a lane per pair of the warp: n <= 64 TEAM / 32
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0) *flag = 0;
    team_sync<TEAM>();
    for (int r = 0; r < m - 1; ++r) {
      // A warp owns the pairs wt + j NWT (j < mine <= 32): lane j forms pair j's rotation (in parallel)
      // into the team's parameter slots, then the warp applies each pair with the lanes over the rows
      // (a broadcast read of the slot). Columns p, q of a pair are touched by its warp only, so the
      // parameters need no barrier before the column update; every element gets the same operations as
      // in a flat (pair, row) task loop.
      if (lane < mine) {
        const int i = wt + lane * NWT;
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
      __syncwarp();
      // columns: A <- A J, V <- V J
      for (int i = wt; i < npair; i += NWT) {
        const RotParam<T> P = prm[i];
        if (P.p < 0) continue;
        const C ec = mk2(P.e.x, -P.e.y);
        C* Ap = A + P.p * lda;
        C* Aq = A + P.q * lda;
        for (int row = lane; row < n; row += 32) {
          const C ap = Ap[row], aq = Aq[row];
          const C sp = cmul(ec, aq), sq = cmul(P.e, ap);
          Ap[row] = mk2(P.c * ap.x - P.s * sp.x, P.c * ap.y - P.s * sp.y);
          Aq[row] = mk2(P.s * sq.x + P.c * aq.x, P.s * sq.y + P.c * aq.y);
        }
        if (want_v) {
          C* Vp = V + P.p * ldv;
          C* Vq = V + P.q * ldv;
          for (int row = lane; row < n; row += 32) {
            const C vp = Vp[row], vq = Vq[row];
            const C tp = cmul(ec, vq), tq = cmul(P.e, vp);
            Vp[row] = mk2(P.c * vp.x - P.s * tp.x, P.c * vp.y - P.s * tp.y);
            Vq[row] = mk2(P.s * tq.x + P.c * vq.x, P.s * tq.y + P.c * vq.y);
          }
        }
      }
      team_sync<TEAM>();
      // rows: A <- J^H A (the same pairs and parameters, lanes over the columns)
      for (int i = wt; i < npair; i += NWT) {
        const RotParam<T> P = prm[i];
        if (P.p < 0) continue;
        const C ec = mk2(P.e.x, -P.e.y);
        for (int col = lane; col < n; col += 32) {
          C* Ac = A + col * lda;
          const C ap = Ac[P.p], aq = Ac[P.q];
          const C sp = cmul(P.e, aq), sq = cmul(ec, ap);
          Ac[P.p] = mk2(P.c * ap.x - P.s * sp.x, P.c * ap.y - P.s * sp.y);
          Ac[P.q] = mk2(P.s * sq.x + P.c * aq.x, P.s * sq.y + P.c * aq.y);
        }
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
