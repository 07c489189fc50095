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
                           int n, bool want_v, int* flag, T thr, int max_sweeps) {
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
      // A warp owns the pairs wt + j NWT (j < mine <= 32): lane j forms pair j's rotation (in parallel),
      // then the warp applies each pair with the lanes over the rows, taking the parameters by shuffle.
      // Columns p, q of a pair are touched by its warp only, so no barrier separates the parameters
      // from the column update; every element gets the same operations as in a flat task loop.
      T Pc = T(1), Ps = T(0), Pex = T(1), Pey = T(0);
      int Pp = -1, Pq = 0;
      if (lane < mine) {
        int p, q;
        rr_pair(m, r, wt + lane * NWT, p, q);
        Pq = q;
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
            Pc = c;
            Ps = t * c;
            Pex = b.x / ab;
            Pey = b.y / ab;
            Pp = p;
            *flag = 1;
          }
        }
      }
      __syncwarp();
      // columns: A <- A J, V <- V J
      for (int j = 0; j < mine; ++j) {
        const int pp = __shfl_sync(0xffffffffu, Pp, j);
        if (pp < 0) continue;
        const int pq = __shfl_sync(0xffffffffu, Pq, j);
        const T c = __shfl_sync(0xffffffffu, Pc, j), sn = __shfl_sync(0xffffffffu, Ps, j);
        const C e = mk2(__shfl_sync(0xffffffffu, Pex, j), __shfl_sync(0xffffffffu, Pey, j));
        const C ec = mk2(e.x, -e.y);
        C* Ap = A + pp * lda;
        C* Aq = A + pq * lda;
        for (int row = lane; row < n; row += 32) {
          const C ap = Ap[row], aq = Aq[row];
          const C sp = cmul(ec, aq), sq = cmul(e, ap);
          Ap[row] = mk2(c * ap.x - sn * sp.x, c * ap.y - sn * sp.y);
          Aq[row] = mk2(sn * sq.x + c * aq.x, sn * sq.y + c * aq.y);
        }
        if (want_v) {
          C* Vp = V + pp * ldv;
          C* Vq = V + pq * ldv;
          for (int row = lane; row < n; row += 32) {
            const C vp = Vp[row], vq = Vq[row];
            const C tp = cmul(ec, vq), tq = cmul(e, vp);
            Vp[row] = mk2(c * vp.x - sn * tp.x, c * vp.y - sn * tp.y);
            Vq[row] = mk2(sn * tq.x + c * vq.x, sn * tq.y + c * vq.y);
          }
        }
      }
      team_sync<TEAM>();
      // rows: A <- J^H A (the same pairs and parameters, lanes over the columns)
      for (int j = 0; j < mine; ++j) {
        const int pp = __shfl_sync(0xffffffffu, Pp, j);
        if (pp < 0) continue;
        const int pq = __shfl_sync(0xffffffffu, Pq, j);
        const T c = __shfl_sync(0xffffffffu, Pc, j), sn = __shfl_sync(0xffffffffu, Ps, j);
        const C e = mk2(__shfl_sync(0xffffffffu, Pex, j), __shfl_sync(0xffffffffu, Pey, j));
        const C ec = mk2(e.x, -e.y);
        for (int col = lane; col < n; col += 32) {
          C* Ac = A + col * lda;
          const C ap = Ac[pp], aq = Ac[pq];
          const C sp = cmul(e, aq), sq = cmul(ec, ap);
          Ac[pp] = mk2(c * ap.x - sn * sp.x, c * ap.y - sn * sp.y);
          Ac[pq] = mk2(sn * sq.x + c * aq.x, sn * sq.y + c * aq.y);
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
