// Batched Hermitian eigensolver for n <= 16, register resident: one-sided (Hestenes) Jacobi.
//
// Replaces eigvals_batched / eigen_batched (ext/ElectronPhononCUDAExt.jl:80-115, cuSOLVER
// heevjBatched) for the small matrices of the e-ph pass (nw = 16 electrons, nm = 12 modes).
//
// FP64 sweeps: a 16-lane half-warp owns one matrix; lane l holds column l of A = H + sigma I in
// registers (sigma = 1.1 ||H||_F makes A positive definite, so its right singular vectors are the
// eigenvectors of H and the column norms after orthogonalisation are lambda + sigma). Each round
// pairs the lanes by the circle method (lane 15 fixed); partners swap columns with shuffles,
// form the 2x2 Gram matrix [[a, g], [g*, b]] and both apply the same plane rotation
//     t = sign(tau) / (|tau| + sqrt(1 + tau^2)), tau = (b - a) / (2 |g|), e = g / |g|,
//     a_p <- c a_p - s conj(e) a_q,   a_q <- s e a_p + c a_q,
// (the same J as the two-sided solver, applied to columns only). A pair is skipped when
// |g| <= tol sqrt(a b); a sweep with no rotation ends the solve. Lanes >= n carry sigma e_l,
// orthogonal to every live column, so they never rotate. FP32 sweeps (mixed precision) hold two
// columns per lane, 8 lanes per matrix (eigh16_jacobi2c_kernel; the pair order is described there).
//
// Mixed precision (EPB_PREC_MIXED): the sweeps run in FP32 to tol = 1e-6 (or until a sweep whose
// rotation angles were all below 1e-4 -- 1e-2 for the pass, see PASS_ANGLE_STOP -- after which the columns
// are orthogonal to the FP32 floor, resp. to 1e-4), then one FP64
// refinement on the same registers: Lowdin re-orthonormalisation V(I - F/2), F = V^H V - I
// (this re-orthogonalises near-degenerate clusters, whose FP32 vectors are defined only up to a
// rotation inside the cluster), and a first-order Rayleigh-Ritz update from S = V^H H V:
//     S'_kl = S_kl - F_kl (S_kk + S_ll) / 2,   E_kl = S'_kl / (S'_ll - S'_kk),
//     v_l <- v_l + sum_k v_k (E_kl - F_kl / 2),  lambda_l = S'_ll + sum_k |S'_kl|^2 / (S'_ll - S'_kk).
// Pairs whose first-order coupling is not small (|S'_kl| > 0.1 |S'_ll - S'_kk|) are left to the
// orthonormalisation (their vectors are accurate as a subspace, which is what gauge-invariant
// quantities use). EPB_PREC_FP64 runs the sweeps in FP64 to tol = 1e-15 and skips the refinement.
#include <algorithm>

#include "epb_common.cuh"
#include "epb_eigh16.cuh"

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
      // the p lane (l < partner) forms g = a_p^H a_q, decides and builds both columns' coefficients; the q
      // lane takes its coefficients and new norm by shuffle (one decision per pair, no divergent update)
      C g0 = mk2(T(0), T(0)), g1 = mk2(T(0), T(0));  // two chains: shorter dependency
#pragma unroll
      for (int i = 0; i < E16; i += 2) {
        cfma_conj(g0, a[i], b[i]);
        cfma_conj(g1, a[i + 1], b[i + 1]);
      }
      const C g = mk2(g0.x + g1.x, g0.y + g1.y);
      const T ag = sqrt(g.x * g.x + g.y * g.y);
      T c = T(1), fx = T(0), fy = T(0), qx = T(0), qy = T(0), np_ = nrm, nq_ = nb;
      int rot = 0;
      if (isP && ag > tol * sqrt(nrm * nb) && ag > T(0)) {
        rot = 1;
        const T tau = (nb - nrm) / (T(2) * ag);
        const T t = (tau >= T(0) ? T(1) : T(-1)) / (fabs(tau) + sqrt(T(1) + tau * tau));
        c = T(1) / sqrt(T(1) + t * t);
        const T s = t * c, ex = g.x / ag, ey = g.y / ag;
        fx = -s * ex;  // p: a_p <- c a_p - s conj(e) a_q
        fy = s * ey;
        qx = s * ex;   // q: a_q <- c a_q + s e a_p
        qy = s * ey;
        np_ = nrm - t * ag;
        nq_ = nb + t * ag;
      }
      const T c_r = shfl(c, src), qx_r = shfl(qx, src), qy_r = shfl(qy, src), nq_r = shfl(nq_, src);
      const int rot_r = __shfl_sync(0xffffffffu, rot, src);
      if (!isP) {
        rot = rot_r;
        c = c_r;
        fx = qx_r;
        fy = qy_r;
        np_ = nq_r;
      }
      if (rot) {
        rotated = 1;
        const C f = mk2(fx, fy);
#pragma unroll
        for (int i = 0; i < E16; ++i) {
          const C u = cmul(f, b[i]);
          a[i] = mk2(c * a[i].x + u.x, c * a[i].y + u.y);
        }
        nrm = np_;
      }
    }
    if (!__any_sync(0xffffffffu, rotated)) break;
  }
  return sweep;
}

// Load column l of matrix b (FP64), optionally mass-scaled; zero outside the live n x n block.
__device__ __forceinline__ double2 load_h(const Eigh16Args& a, int64_t b, int i, int l, int n) {
  double2 v = make_double2(0.0, 0.0);
  if (l < n && i < n) {
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
  return v;
}

// Rank of this lane's eigenvalue among the live lanes of its half-warp, then the outputs.
__device__ __forceinline__ void write_sorted(const Eigh16Args& a, int64_t b, bool live, int lane, int l, int n,
                                             double lam, const double2 (&v)[E16]) {
  int rank = 0;
#pragma unroll
  for (int k = 0; k < E16; ++k) {
    double lk = __shfl_sync(0xffffffffu, lam, (lane & 16) + k);
    rank += (k < n) && (lk < lam || (lk == lam && k < l));
  }
  if (live && l < n) {
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

// ---- FP32 sweeps, two columns per lane (8 lanes per matrix, 4 matrices per warp) ------------------------
// Lane l of a matrix's 8-lane group keeps columns l ("a") and l + 8 ("b") of H + sigma I for the whole solve,
// as packed f32x2 pairs (real / imaginary parts of entries 2i, 2i+1). A sweep is 15 steps of 8 disjoint
// pairs, in the same order every sweep:
//   steps 0..7: lane l rotates its own pair (a_l, b_{(l+s) mod 8}); between steps the b columns move one lane
//     down the ring (after the eighth move they are home again). These are the 64 pairs between the two
//     halves, each formed by one lane alone: no duplicated Gram product, one column shuffle per pair.
//   steps 8..14: the round-robin over the 8 lanes, lane l rotating a_l with the partner's a and b_l with the
//     partner's b; both lanes of such a pair form the same Gram entry bit for bit (the 16-lane rule below).
// Against one column per lane this drops a quarter of the Gram products and of the column shuffles per sweep
// and holds two matrices per 16 lanes. An FP32 emulation of the sweeps (GUE matrices, stop at 1e-2) gives
// 5.07 sweeps per warp of four matrices, 5.2-5.3 for the 16-lane round-robin per warp of two, and 5.6-6.0 for
// two-column orders whose pair sequence changes from sweep to sweep.

__device__ __forceinline__ int circle8_partner(int l, int r) {
  // 8 players, player 7 fixed, 7 rounds
  if (l == 7) return r;
  if (l == r) return 7;
  const int p = (2 * r - l) % 7;
  return p < 0 ? p + 7 : p;
}

// Rotation of the pair (p, q) with g = a_p^H a_q and squared norms A, B: c, and w with s e = w g and
// t |g| = tg (signed); see the 16-lane form. Returns false below the tolerance.
__device__ __forceinline__ bool pair_rotation(float gx, float gy, float A, float B, float tol2, float as2, float& c,
                                              float& w, float& tg, int& big) {
  const float ag2 = gx * gx + gy * gy;
  if (!(ag2 > tol2 * (A * B) && ag2 > 0.f)) return false;
  const float d = B - A;
  const float rr = rsqrtf(fmaf(d, d, 4.f * ag2));
  const float c2 = fmaf(0.5f * fabsf(d), rr, 0.5f);
  const float ic = rsqrtf(c2);
  c = c2 * ic;
  w = copysignf(rr * ic, d);
  const float tq = rr * ic * ic;
  big |= ag2 * (tq * tq) > as2;
  tg = w * ic * ag2;
  return true;
}

// Squared norm of a packed column.
__device__ __forceinline__ float col_norm2(const f32x2 (&X)[8], const f32x2 (&Y)[8]) {
  f32x2 n0 = pk(0.f, 0.f), n1 = pk(0.f, 0.f);
#pragma unroll
  for (int i = 0; i < 8; i += 2) {
    n0 = pfma(Y[i], Y[i], pfma(X[i], X[i], n0));
    n1 = pfma(Y[i + 1], Y[i + 1], pfma(X[i + 1], X[i + 1], n1));
  }
  return hsum(padd(n0, n1));
}

// One round-robin pair between lanes: rotate this lane's column (X, Y; squared norm nrm) against the partner
// lane's column of the same half. Both lanes derive the same rotation (bitwise-identical Gram sums).
__device__ __forceinline__ void robin_pair(f32x2 (&X)[8], f32x2 (&Y)[8], float& nrm, int src, bool isP, float tol2,
                                           float as2, int& big) {
  const f32x2 Z = pk(0.f, 0.f);
  f32x2 PX[8], PY[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    PX[i] = __shfl_sync(0xffffffffu, X[i], src);
    PY[i] = __shfl_sync(0xffffffffu, Y[i], src);
  }
  const float nb = __shfl_sync(0xffffffffu, nrm, src);
  f32x2 gx0 = Z, gx1 = Z, gy0 = Z, gy1 = Z, gi0 = Z, gi1 = Z, gj0 = Z, gj1 = Z;
#pragma unroll
  for (int i = 0; i < 8; i += 2) {
    gx0 = pfma(X[i], PX[i], gx0);
    gx1 = pfma(X[i + 1], PX[i + 1], gx1);
    gy0 = pfma(Y[i], PY[i], gy0);
    gy1 = pfma(Y[i + 1], PY[i + 1], gy1);
    gi0 = pfma(X[i], PY[i], gi0);
    gi1 = pfma(X[i + 1], PY[i + 1], gi1);
    gj0 = pfma(Y[i], PX[i], gj0);
    gj1 = pfma(Y[i + 1], PX[i + 1], gj1);
  }
  const float hi = hsum(padd(gi0, gi1)), hj = hsum(padd(gj0, gj1));
  const float gx = hsum(padd(padd(gx0, gx1), padd(gy0, gy1))), gy = isP ? hi - hj : hj - hi;
  const float A = isP ? nrm : nb, B = isP ? nb : nrm;
  float c, w, tg;
  if (pair_rotation(gx, gy, A, B, tol2, as2, c, w, tg, big)) {
    // p: a_p <- c a_p - w conj(g) a_q;  q: a_q <- c a_q + w g a_p
    const float fx = isP ? -w * gx : w * gx, fy = w * gy;
    nrm = isP ? A - tg : B + tg;
    const f32x2 C2 = pk(c, c), FX = pk(fx, fx), FY = pk(fy, fy), FYN = pk(-fy, -fy);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const f32x2 xr = pfma(C2, X[i], pfma(FX, PX[i], pmul(FYN, PY[i])));
      const f32x2 yr = pfma(C2, Y[i], pfma(FX, PY[i], pmul(FY, PX[i])));
      X[i] = xr;
      Y[i] = yr;
    }
  }
}

__device__ int onesided_sweeps_2col(f32x2 (&XA)[8], f32x2 (&YA)[8], f32x2 (&XB)[8], f32x2 (&YB)[8], float tol,
                                    int max_sweeps, float angle_stop) {
  const int lane = threadIdx.x & 31;
  const int l = lane & 7, base = lane & 24;
  const f32x2 Z = pk(0.f, 0.f);
  const float tol2 = tol * tol, as2 = angle_stop * angle_stop;
  const int down = base + ((l + 1) & 7);
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    float nA = col_norm2(XA, YA), nB = col_norm2(XB, YB);
    int big = 0;
    // steps 0..7: the lane's own pair (a, b), then b moves one lane down the ring
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
      f32x2 gx0 = Z, gx1 = Z, gi0 = Z, gi1 = Z, gj0 = Z, gj1 = Z;
#pragma unroll
      for (int i = 0; i < 8; i += 2) {
        gx0 = pfma(YA[i], YB[i], pfma(XA[i], XB[i], gx0));
        gx1 = pfma(YA[i + 1], YB[i + 1], pfma(XA[i + 1], XB[i + 1], gx1));
        gi0 = pfma(XA[i], YB[i], gi0);
        gi1 = pfma(XA[i + 1], YB[i + 1], gi1);
        gj0 = pfma(YA[i], XB[i], gj0);
        gj1 = pfma(YA[i + 1], XB[i + 1], gj1);
      }
      // g = a^H b
      const float gx = hsum(padd(gx0, gx1)), gy = hsum(padd(gi0, gi1)) - hsum(padd(gj0, gj1));
      float c, w, tg;
      if (pair_rotation(gx, gy, nA, nB, tol2, as2, c, w, tg, big)) {
        // a <- c a - w conj(g) b;  b <- c b + w g a
        const float fx = w * gx, fy = w * gy;
        nA -= tg;
        nB += tg;
        const f32x2 C2 = pk(c, c), FX = pk(fx, fx), FY = pk(fy, fy), FXN = pk(-fx, -fx), FYN = pk(-fy, -fy);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const f32x2 xa = pfma(C2, XA[i], pfma(FXN, XB[i], pmul(FYN, YB[i])));
          const f32x2 ya = pfma(C2, YA[i], pfma(FXN, YB[i], pmul(FY, XB[i])));
          const f32x2 xb = pfma(C2, XB[i], pfma(FX, XA[i], pmul(FYN, YA[i])));
          const f32x2 yb = pfma(C2, YB[i], pfma(FX, YA[i], pmul(FY, XA[i])));
          XA[i] = xa;
          YA[i] = ya;
          XB[i] = xb;
          YB[i] = yb;
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        XB[i] = __shfl_sync(0xffffffffu, XB[i], down);
        YB[i] = __shfl_sync(0xffffffffu, YB[i], down);
      }
      nB = __shfl_sync(0xffffffffu, nB, down);
    }
    // steps 8..14: round-robin over the 8 lanes within each half
#pragma unroll 1
    for (int r = 0; r < 7; ++r) {
      const int p = circle8_partner(l, r);
      const int src = base + p;
      robin_pair(XA, YA, nA, src, l < p, tol2, as2, big);
      robin_pair(XB, YB, nB, src, l < p, tol2, as2, big);
    }
    if (!__any_sync(0xffffffffu, big)) break;
  }
  return sweep;
}

// Mixed precision, first half: FP32 sweeps with two columns per lane; writes the normalised, unsorted FP32
// columns to a.V32 (16 x 16 per matrix, column j = the rotated column j of H + sigma I) for the refinement.
__global__ void __launch_bounds__(128, 4) eigh16_jacobi2c_kernel(Eigh16Args a) {
  const int lane = threadIdx.x & 31;
  const int l = lane & 7;
  const int slot = threadIdx.x >> 3;
  const int n = a.n;
  const int64_t per_block = blockDim.x / 8;
  for (int64_t b0 = (int64_t)blockIdx.x * per_block; b0 < a.batch; b0 += (int64_t)gridDim.x * per_block) {
    const int64_t b = b0 + slot;
    const bool live = b < a.batch;
    float ar[E16], ai[E16], br[E16], bi[E16];
    double f2 = 0.0;
#pragma unroll
    for (int i = 0; i < E16; ++i) {
      const double2 u = live ? load_h(a, b, i, l, n) : make_double2(0.0, 0.0);
      const double2 v = live ? load_h(a, b, i, l + 8, n) : make_double2(0.0, 0.0);
      f2 += (u.x * u.x + u.y * u.y) + (v.x * v.x + v.y * v.y);
      ar[i] = (float)u.x;
      ai[i] = (float)u.y;
      br[i] = (float)v.x;
      bi[i] = (float)v.y;
    }
    for (int o = 4; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);  // within the 8-lane group
    const double sigma = f2 > 0.0 ? 1.1 * sqrt(f2) : 1.0;                       // zero (or padding): shift 1
#pragma unroll
    for (int i = 0; i < E16; ++i) {
      if (i == l) ar[i] += (float)sigma;  // columns >= n: sigma e_j
      if (i == l + 8) br[i] += (float)sigma;
    }
    f32x2 XA[8], YA[8], XB[8], YB[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      XA[i] = pk(ar[2 * i], ar[2 * i + 1]);
      YA[i] = pk(ai[2 * i], ai[2 * i + 1]);
      XB[i] = pk(br[2 * i], br[2 * i + 1]);
      YB[i] = pk(bi[2 * i], bi[2 * i + 1]);
    }
    const int sw = onesided_sweeps_2col(XA, YA, XB, YB, 1e-6f, a.max_sweeps, a.angle_stop > 0.f ? a.angle_stop : 1e-4f);
    if (sw >= a.max_sweeps && lane == 0) atomicAdd(a.nonconv, 1);
    if (live) {
      float2* vo = a.V32 + b * (int64_t)E16 * E16;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const f32x2(&X)[8] = h ? XB : XA;
        const f32x2(&Y)[8] = h ? YB : YA;
        double nr2 = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float2 x = upk(X[i]), y = upk(Y[i]);
          nr2 += (double)x.x * x.x + (double)y.x * y.x;
          nr2 += (double)x.y * x.y + (double)y.y * y.y;
        }
        const double inv = 1.0 / sqrt(nr2);
        float2* vc = vo + (int64_t)E16 * (l + 8 * h);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float2 x = upk(X[i]), y = upk(Y[i]);
          vc[2 * i] = make_float2((float)(x.x * inv), (float)(y.x * inv));
          vc[2 * i + 1] = make_float2((float)(x.y * inv), (float)(y.y * inv));
        }
      }
    }
  }
}

// Whole solve in FP64 (sorted output): a 16-lane half-warp per matrix, lane l holding column l.
__global__ void __launch_bounds__(128, 1) eigh16_jacobi_kernel(Eigh16Args a) {
  const int lane = threadIdx.x & 31;
  const int l = lane & 15;
  const int slot = threadIdx.x >> 4;
  const int n = a.n;
  const int64_t per_block = blockDim.x / 16;
  for (int64_t b0 = (int64_t)blockIdx.x * per_block; b0 < a.batch; b0 += (int64_t)gridDim.x * per_block) {
    const int64_t b = b0 + slot;
    const bool live = b < a.batch;
    double2 col[E16];
    double f2 = 0.0;
#pragma unroll
    for (int i = 0; i < E16; ++i) {
      col[i] = live ? load_h(a, b, i, l, n) : make_double2(0.0, 0.0);
      f2 += col[i].x * col[i].x + col[i].y * col[i].y;
    }
    for (int o = 8; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);  // within the half-warp
    const double sigma = f2 > 0.0 ? 1.1 * sqrt(f2) : 1.0;  // zero (or padding) matrices: shift 1
#pragma unroll
    for (int i = 0; i < E16; ++i)
      if (i == l) col[i].x += sigma;  // lanes >= n: sigma e_l
    const int sw = onesided_sweeps<double>(col, 1e-15, a.max_sweeps);
    if (sw >= a.max_sweeps && lane == 0) atomicAdd(a.nonconv, 1);
    double nr2 = 0.0;
#pragma unroll
    for (int i = 0; i < E16; ++i) nr2 += col[i].x * col[i].x + col[i].y * col[i].y;
    const double inv = 1.0 / sqrt(nr2);
    double2 v[E16];
#pragma unroll
    for (int i = 0; i < E16; ++i) v[i] = make_double2(col[i].x * inv, col[i].y * inv);
    write_sorted(a, b, live, lane, l, n, sqrt(nr2) - sigma, v);
  }
}

// MODE 2: FP64 refinement of FP32 eigenvectors (see the file header), sorted output.
__global__ void __launch_bounds__(128) eigh16_refine_kernel(Eigh16Args a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto Hs = reinterpret_cast<double2(*)[E16 * E16]>(smem_raw);
  auto Vs = reinterpret_cast<double2(*)[E16 * E16]>(smem_raw + 8 * E16 * E16 * sizeof(double2));
  const int lane = threadIdx.x & 31;
  const int l = lane & 15;
  const int slot = threadIdx.x >> 4;
  const int n = a.n;
  const int64_t per_block = blockDim.x / 16;
  for (int64_t b0 = (int64_t)blockIdx.x * per_block; b0 < a.batch; b0 += (int64_t)gridDim.x * per_block) {
    const int64_t b = b0 + slot;
    const bool live = b < a.batch;
    double f2 = 0.0;
#pragma unroll
    for (int i = 0; i < E16; ++i) {
      double2 hv = live ? load_h(a, b, i, l, n) : make_double2(0.0, 0.0);
      f2 += hv.x * hv.x + hv.y * hv.y;
      Hs[slot][i + E16 * l] = hv;
    }
    for (int o = 8; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    const double sigma = f2 > 0.0 ? 1.1 * sqrt(f2) : 1.0;
    double2 v[E16];
    {
      const float2* vi = a.V32 + (live ? b : 0) * (int64_t)E16 * E16 + (int64_t)E16 * l;
#pragma unroll
      for (int i = 0; i < E16; ++i) {
        float2 x = live ? vi[i] : make_float2(i == l ? 1.f : 0.f, 0.f);
        v[i] = make_double2(x.x, x.y);
      }
    }
    double lam = 0.0;
    bool cluster = false;
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
        d += v[i].x * w[i].x + v[i].y * w[i].y;
        fll += v[i].x * v[i].x + v[i].y * v[i].y;
      }
      fll -= 1.0;
      const double dp = d * (1.0 - fll);
      double2 tcol[E16];
      double lam_corr = 0.0;
      cluster = false;
#pragma unroll
      for (int k = 0; k < E16; ++k) {
        const double dk = __shfl_sync(0xffffffffu, d, (lane & 16) + k);
        const double dpk = __shfl_sync(0xffffffffu, dp, (lane & 16) + k);
        double2 s0 = make_double2(0.0, 0.0), s1 = s0, g0 = s0, g1 = s0;
#pragma unroll
        for (int i = 0; i < E16; i += 2) {
          double2 v0 = Vs[slot][i + E16 * k], v1 = Vs[slot][i + 1 + E16 * k];
          cfma_conj(s0, v0, w[i]);
          cfma_conj(s1, v1, w[i + 1]);
          cfma_conj(g0, v0, v[i]);
          cfma_conj(g1, v1, v[i + 1]);
        }
        const double2 s = make_double2(s0.x + s1.x, s0.y + s1.y), g = make_double2(g0.x + g1.x, g0.y + g1.y);
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
      // v <- v + V t  (w is dead after the S / G sums: reuse it for V t)
#pragma unroll
      for (int i = 0; i < E16; ++i) w[i] = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < E16; ++k) {
        double2 t = tcol[k];
#pragma unroll
        for (int i = 0; i < E16; ++i) cfma(w[i], Vs[slot][i + E16 * k], t);
      }
#pragma unroll
      for (int i = 0; i < E16; ++i) v[i] = make_double2(v[i].x + w[i].x, v[i].y + w[i].y);
      lam = dp + lam_corr;
      __syncwarp();
    }
    const bool flagged = (__ballot_sync(0xffffffffu, cluster && live) & (0xFFFFu << (lane & 16))) != 0;
    if (a.flag_list && flagged && l == 0) {
      int pos = atomicAdd(a.flag_count, 1);
      a.flag_list[pos] = b;
    }
    if (!(a.flag_list && flagged)) write_sorted(a, b, live, lane, l, n, lam, v);
    __syncwarp();
  }
}

// MODE 2, two lanes per column: the same refinement as eigh16_refine_kernel, one matrix per warp;
// lane (l, h) holds rows 8h .. 8h + 7 of column l, partial column sums are combined with one shuffle
// across the halves. Half the per-lane state of the one-lane-per-column form (fits in ~128
// registers, twice the resident warps) and half the unrolled code.
constexpr int RLD = E16 + 1;  // padded leading dimension of the shared H and V tiles

__global__ void __launch_bounds__(128, 3) eigh16_refine2_kernel(Eigh16Args a) {
  __shared__ double2 Hs[4][E16 * RLD];  // H[i][k] at i * RLD + k
  __shared__ double2 Vs[4][E16 * RLD];  // V[i][k] at i * RLD + k
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane & 15, h = lane >> 4, r0 = 8 * h;
  const int n = a.n;
  double2* H = Hs[warp];
  double2* V = Vs[warp];
  for (int64_t b = (int64_t)blockIdx.x * 4 + warp; b - warp < a.batch; b += (int64_t)gridDim.x * 4) {
    const bool live = b < a.batch;
    double f2 = 0.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const double2 hv = live ? load_h(a, b, r0 + r, l, n) : make_double2(0.0, 0.0);
      f2 += hv.x * hv.x + hv.y * hv.y;
      H[(r0 + r) * RLD + l] = hv;
    }
    for (int o = 16; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    const double sigma = f2 > 0.0 ? 1.1 * sqrt(f2) : 1.0;
    double2 v[8];
    {
      const float2* vi = a.V32 + (live ? b : 0) * (int64_t)E16 * E16 + (int64_t)E16 * l + r0;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const float2 x = live ? vi[r] : make_float2(r0 + r == l ? 1.f : 0.f, 0.f);
        v[r] = make_double2(x.x, x.y);
      }
    }
    double lam = 0.0;
    bool cluster = false;  // sticky over the iterations: once a pair is out of first-order range, the matrix is flagged
    // first-order range |S'_kl| < theta |gap|: the update leaves O(theta^2) mixing per iteration. With an exact
    // slow path for flagged matrices (public API) theta = 1e-3 (two iterations: O(1e-12)); without one (the
    // pass's eigenvectors) theta = 0.1, correcting as much as first order can.
    const double th2 = a.flag_list ? 1e-6 : 1e-2;
    for (int it = 0; it < a.refine; ++it) {
#pragma unroll
      for (int r = 0; r < 8; ++r) V[(r0 + r) * RLD + l] = v[r];
      __syncwarp();
      // w = H v on this lane's rows; d = Re v^H w, fll = |v|^2 - 1 (whole column)
      double2 w[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) w[r] = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < E16; ++k) {
        const double2 vk = V[k * RLD + l];
#pragma unroll
        for (int r = 0; r < 8; ++r) cfma(w[r], H[(r0 + r) * RLD + k], vk);
      }
      double d = 0.0, fll = 0.0;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        d += v[r].x * w[r].x + v[r].y * w[r].y;
        fll += v[r].x * v[r].x + v[r].y * v[r].y;
      }
      d += __shfl_xor_sync(0xffffffffu, d, 16);
      fll += __shfl_xor_sync(0xffffffffu, fll, 16);
      fll -= 1.0;
      const double dp = d * (1.0 - fll);
      double lam_corr = 0.0;
      double2 u[8];  // V t accumulated over k
#pragma unroll
      for (int r = 0; r < 8; ++r) u[r] = make_double2(0.0, 0.0);
      // S and G columns for KB values of k at a time: 4 KB independent FP64 accumulation chains (KB = 2
      // keeps the kernel inside 168 registers, three CTAs per SM)
      constexpr int KB = 2;
#pragma unroll 1
      for (int k0 = 0; k0 < E16; k0 += KB) {
        double2 sb[KB], gb[KB];
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) sb[kk] = gb[kk] = make_double2(0.0, 0.0);
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
          for (int kk = 0; kk < KB; ++kk) {
            const double2 vik = V[(r0 + r) * RLD + k0 + kk];
            cfma_conj(sb[kk], vik, w[r]);
            cfma_conj(gb[kk], vik, v[r]);
          }
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) {
          sb[kk].x += __shfl_xor_sync(0xffffffffu, sb[kk].x, 16);
          sb[kk].y += __shfl_xor_sync(0xffffffffu, sb[kk].y, 16);
          gb[kk].x += __shfl_xor_sync(0xffffffffu, gb[kk].x, 16);
          gb[kk].y += __shfl_xor_sync(0xffffffffu, gb[kk].y, 16);
        }
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) {
        const int k = k0 + kk;
        const double dk = __shfl_sync(0xffffffffu, d, k);
        const double dpk = __shfl_sync(0xffffffffu, dp, k);
        const double2 s = sb[kk], g = gb[kk];
        double2 t;
        if (k == l) {
          t = make_double2(-0.5 * fll, 0.0);
        } else {
          const double2 sp = make_double2(s.x - 0.5 * g.x * (dk + d), s.y - 0.5 * g.y * (dk + d));
          const double gap = dp - dpk;
          const double asp2 = sp.x * sp.x + sp.y * sp.y;
          t = make_double2(-0.5 * g.x, -0.5 * g.y);
          if (k < n && l < n) {
            if (asp2 < th2 * gap * gap) {
              // 1 / gap: FP32 reciprocal + one FP64 Newton step (~1e-14 relative; t itself is O(1e-6))
              const double ag = fabs(gap);
              double rg;
              if (ag > 1e-30 && ag < 1e30) {
                rg = (double)__frcp_rn((float)gap);
                rg = rg * (2.0 - gap * rg);
              } else {
                rg = 1.0 / gap;
              }
              t.x += sp.x * rg;
              t.y += sp.y * rg;
              lam_corr += asp2 * rg;
            } else if (asp2 > 1e-26 * sigma * sigma) {
              cluster = true;
            }
          }
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) cfma(u[r], V[(r0 + r) * RLD + k], t);
        }
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = make_double2(v[r].x + u[r].x, v[r].y + u[r].y);
      lam = dp + lam_corr;
      __syncwarp();
    }
    // both halves agree on lam and on the flag (each half saw the whole column sums)
    const bool flagged = __ballot_sync(0xffffffffu, cluster && live) != 0;
    if (a.flag_list && flagged && lane == 0) {
      const int pos = atomicAdd(a.flag_count, 1);
      a.flag_list[pos] = b;
    }
    if (!(a.flag_list && flagged)) {
      int rank = 0;
#pragma unroll
      for (int k = 0; k < E16; ++k) {
        const double lk = __shfl_sync(0xffffffffu, lam, k);
        rank += (k < n) && (lk < lam || (lk == lam && k < l));
      }
      if (live && l < n) {
        double ev = lam;
        if (a.mass) ev = ev >= 0 ? sqrt(ev) : -sqrt(-ev);
        if (a.E && h == 0) a.E[b * n + rank] = ev;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const int i = r0 + r;
          if (i < n) {
            double2 o = v[r];
            if (a.mass) {
              const double sc = 1.0 / sqrt(a.mass[i]);
              o.x *= sc;
              o.y *= sc;
            }
            if (a.U32) a.U32[b * (int64_t)n * n + i + (int64_t)rank * n] = make_float2((float)o.x, (float)o.y);
            if (a.U64) a.U64[b * (int64_t)n * n + i + (int64_t)rank * n] = o;
          }
        }
      }
    }
    __syncwarp();
  }
}

// MODE 2 for complex64 output (the e-ph pass): the same first-order update as eigh16_refine2_kernel with
// the residual in FP64 and the correction in FP32. With R = H V - V diag(d), d_l = Re v_l^H H v_l (FP64,
// the products of FP32 data are exact), the coupling of the update is
//     S'_kl = S_kl - G_kl (d_k + d_l) / 2 = v_k^H r_l + G_kl (d_l - d_k) / 2        (k != l),
// where every term is small: r_l = O(off-diagonal coupling) is rounded to FP32 (relative 6e-8 of a small
// number) and v_k^H r_l, G_kl = v_k^H v_l and the update V t run in FP32. The FP32 rounding of G_kl
// (a few 1e-8, from a sum of O(1) products) enters t at the size of the FP32 rounding of the output
// columns, so the stored complex64 vectors are as accurate as with the all-FP64 update; |v_l|^2 - 1 and
// the Rayleigh quotients (the eigenvalues, used for the order) stay FP64. FP64 work: W = H V (128 complex
// FMAs per lane); FP32: S, G and V t (384 complex FMAs per lane), against 512 FP64 complex FMAs per lane
// for the all-FP64 update. Pass only: no mass scaling, no flag list, one iteration.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__global__ void __launch_bounds__(128, 4) eigh16_refine_c64_kernel(Eigh16Args a) {
  __shared__ double2 Hs[4][E16 * RLD];  // H[i][k] at i * RLD + k
  __shared__ float2 Vs[4][E16 * RLD];   // V[i][k] (FP32 Jacobi vectors)
  __shared__ float2 Rs[4][E16 * RLD];   // R[i][l] = (H V - V d)[i][l], rounded to FP32
  // packed FP32 H (n = 16) and FP32 vectors of the warp's next matrix, fetched with cp.async while the
  // current one is refined (the solve is latency-bound at 16 warps per SM)
  __shared__ __align__(16) float HpS[4][E16 * E16];
  __shared__ __align__(16) float2 VpS[4][E16 * E16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane & 15, h = lane >> 4, r0 = 8 * h;
  const int n = a.n;
  double2* H = Hs[warp];
  float2* V = Vs[warp];
  float2* R = Rs[warp];
  constexpr double th2 = 1e-2;  // first-order range |S'_kl| < 0.1 |gap| (no slow path in the pass)
  const int64_t step = (int64_t)gridDim.x * 4;
  const bool staged = a.Hp != nullptr && n == E16 &&
                      ((reinterpret_cast<uintptr_t>(a.Hp) | reinterpret_cast<uintptr_t>(a.V32)) & 15) == 0;
  auto prefetch = [&](int64_t bn) {
    if (bn < a.batch) {
      const float4* hs = reinterpret_cast<const float4*>(a.Hp + bn * (E16 * E16));     // 64 x 16 bytes
      const float4* vs = reinterpret_cast<const float4*>(a.V32 + bn * (E16 * E16));    // 128 x 16 bytes
      for (int c = lane; c < 64; c += 32) cp_async16(&HpS[warp][4 * c], hs + c);
      for (int c = lane; c < 128; c += 32) cp_async16(&VpS[warp][2 * c], vs + c);
    }
    cp_async_commit();
  };
  if (staged) prefetch((int64_t)blockIdx.x * 4 + warp);
  for (int64_t b = (int64_t)blockIdx.x * 4 + warp; b - warp < a.batch; b += step) {
    const bool live = b < a.batch;
    float2 v[8];
    if (staged) {
      cp_async_wait0();
      __syncwarp();
      const float* hp = HpS[warp];
      constexpr int NRE = E16 * (E16 + 1) / 2;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = r0 + r, ii = i <= l ? i : l, jj = i <= l ? l : i;
        const float re = hp[jj * (jj + 1) / 2 + ii];
        const float im = ii < jj ? hp[NRE + jj * (jj - 1) / 2 + ii] : 0.f;
        H[i * RLD + l] = live ? make_double2(re, i <= l ? im : -im) : make_double2(0.0, 0.0);
        v[r] = live ? VpS[warp][E16 * l + i] : make_float2(i == l ? 1.f : 0.f, 0.f);
        V[i * RLD + l] = v[r];
      }
      __syncwarp();  // every lane has read the staging buffers
      prefetch(b + step);
    } else {
#pragma unroll
      for (int r = 0; r < 8; ++r) H[(r0 + r) * RLD + l] = live ? load_h(a, b, r0 + r, l, n) : make_double2(0.0, 0.0);
      const float2* vi = a.V32 + (live ? b : 0) * (int64_t)E16 * E16 + (int64_t)E16 * l + r0;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        v[r] = live ? vi[r] : make_float2(r0 + r == l ? 1.f : 0.f, 0.f);
        V[(r0 + r) * RLD + l] = v[r];
      }
    }
    __syncwarp();
    // w = H v on this lane's rows (FP64)
    double2 w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) w[r] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < E16; ++k) {
      const float2 vk32 = V[k * RLD + l];
      const double2 vk = make_double2(vk32.x, vk32.y);
#pragma unroll
      for (int r = 0; r < 8; ++r) cfma(w[r], H[(r0 + r) * RLD + k], vk);
    }
    // d = Re v^H w, fll = |v|^2 - 1 (whole column, FP64)
    double d = 0.0, fll = 0.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const double vx = v[r].x, vy = v[r].y;
      d = fma(vx, w[r].x, fma(vy, w[r].y, d));
      fll = fma(vx, vx, fma(vy, vy, fll));
    }
    d += __shfl_xor_sync(0xffffffffu, d, 16);
    fll += __shfl_xor_sync(0xffffffffu, fll, 16);
    fll -= 1.0;
    const double dp = d * (1.0 - fll);
#pragma unroll
    for (int r = 0; r < 8; ++r)
      R[(r0 + r) * RLD + l] = make_float2((float)(w[r].x - (double)v[r].x * d), (float)(w[r].y - (double)v[r].y * d));
    __syncwarp();
    float2 u[8];  // V t accumulated over k (FP32)
#pragma unroll
    for (int r = 0; r < 8; ++r) u[r] = make_float2(0.f, 0.f);
    float2 rl[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) rl[r] = R[(r0 + r) * RLD + l];
    float lam_corr = 0.f;
    constexpr int KB = 4;
#pragma unroll 1
    for (int k0 = 0; k0 < E16; k0 += KB) {
      float2 sb[KB], gb[KB];
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) sb[kk] = gb[kk] = make_float2(0.f, 0.f);
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) {
          const float2 vik = V[(r0 + r) * RLD + k0 + kk];
          cfma_conj(sb[kk], vik, rl[r]);
          cfma_conj(gb[kk], vik, v[r]);
        }
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) {
        sb[kk].x += __shfl_xor_sync(0xffffffffu, sb[kk].x, 16);
        sb[kk].y += __shfl_xor_sync(0xffffffffu, sb[kk].y, 16);
        gb[kk].x += __shfl_xor_sync(0xffffffffu, gb[kk].x, 16);
        gb[kk].y += __shfl_xor_sync(0xffffffffu, gb[kk].y, 16);
      }
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) {
        const int k = k0 + kk;
        const double dk = __shfl_sync(0xffffffffu, d, k);
        const double dpk = __shfl_sync(0xffffffffu, dp, k);
        const float2 g = gb[kk];
        float2 t;
        if (k == l) {
          t = make_float2((float)(-0.5 * fll), 0.f);
        } else {
          const float hd = (float)(0.5 * (d - dk));
          const float2 sp = make_float2(fmaf(g.x, hd, sb[kk].x), fmaf(g.y, hd, sb[kk].y));
          const double gap = dp - dpk;
          const float asp2 = fmaf(sp.x, sp.x, sp.y * sp.y);
          t = make_float2(-0.5f * g.x, -0.5f * g.y);
          if (k < n && l < n && (double)asp2 < th2 * gap * gap) {
            const double ag = fabs(gap);
            const float rg = (ag > 1e-30 && ag < 1e30) ? __frcp_rn((float)gap) : (float)(1.0 / gap);
            t.x = fmaf(sp.x, rg, t.x);
            t.y = fmaf(sp.y, rg, t.y);
            lam_corr = fmaf(asp2, rg, lam_corr);
          }
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) cfma(u[r], V[(r0 + r) * RLD + k], t);
      }
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = make_float2(v[r].x + u[r].x, v[r].y + u[r].y);
    const double lam = dp + (double)lam_corr;
    int rank = 0;
    double gmin = 1e300, amax = 0.0;  // smallest gap to another eigenvalue, largest |eigenvalue|
#pragma unroll
    for (int k = 0; k < E16; ++k) {
      const double lk = __shfl_sync(0xffffffffu, lam, k);
      rank += (k < n) && (lk < lam || (lk == lam && k < l));
      if (k < n) {
        amax = fmax(amax, fabs(lk));
        if (k != l) gmin = fmin(gmin, fabs(lk - lam));
      }
    }
    if (a.gap_count) {
      // a near-degenerate pair: its eigenvectors turn by the FP32-level error of H over the gap, so the
      // matrix is listed for the FP64 re-solve. Gaps under 1e-6 of max |lambda| are degenerate at the
      // precision of the data (symmetry-enforced pairs, e.g. Kramers): there the split of |g|^2 between the
      // pair's bands is a gauge choice in any precision, and such matrices are not listed
      for (int o = 8; o > 0; o >>= 1) gmin = fmin(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
      if (live && lane == 0 && gmin < (double)a.gap_rel * amax && gmin >= 1e-6 * amax) {
        const int pos = atomicAdd(a.gap_count, 1);
        if (pos < a.gap_cap) a.gap_list[pos] = b;
      }
    }
    if (live && l < n) {
      if (a.E && h == 0) a.E[b * n + rank] = lam;
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r0 + r < n) a.U32[b * (int64_t)n * n + r0 + r + (int64_t)rank * n] = v[r];
    }
    __syncwarp();
  }
}

// The refinement kernel of a mixed solve: the FP32-correction form for the pass's complex64 output,
// the all-FP64 form otherwise.
static void refine_launch(epb_ctx* ctx, const Eigh16Args& a) {
  const int64_t blocks = std::min<int64_t>(cdiv(a.batch, 4), (int64_t)ctx->sm_count * 8);
  if (a.U32 && !a.U64 && !a.mass && !a.flag_list && a.refine == 1)
    eigh16_refine_c64_kernel<<<(unsigned)blocks, 128, 0, ctx->stream>>>(a);
  else
    eigh16_refine2_kernel<<<(unsigned)blocks, 128, 0, ctx->stream>>>(a);
}

int eigh16_launch(epb_ctx* ctx, Eigh16Args& a, bool mixed) {
  if (a.batch == 0) return EPB_OK;
  const int threads = 128;  // 8 matrices per block
  const int64_t blocks_needed = cdiv(a.batch, threads / 16);
  auto grid_cap = [&](int per_sm) {
    int64_t cap = (int64_t)ctx->sm_count * per_sm;
    return (unsigned)(blocks_needed < cap ? blocks_needed : cap);
  };
  if (!mixed) {
    prof_begin(ctx, EPB_PROF_EIGH);
    eigh16_jacobi_kernel<<<grid_cap(8), threads, 0, ctx->stream>>>(a);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
    return EPB_OK;
  }
  EPB_CHECK_ARG(a.V32 != nullptr, "eigh16: mixed mode needs a V32 workspace");
  const size_t smem = 2 * 8 * E16 * E16 * sizeof(double2);
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(eigh16_refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  prof_begin(ctx, EPB_PROF_EIGH);
  eigh16_jacobi2c_kernel<<<(unsigned)std::min<int64_t>(cdiv(a.batch, 16), (int64_t)ctx->sm_count * 16), 128, 0,
                           ctx->stream>>>(a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  prof_begin(ctx, EPB_PROF_REFINE);
  refine_launch(ctx, a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// The two halves of the pass's mixed eigensolve of packed FP32 H(k+q) (n = 16), launched separately so that
// the pass can run the refinement of one batch beside the Jacobi of the next: FP32 Jacobi into V32 (unsorted
// FP32 vectors), then the refinement of V32 against H into U (sorted, complex64; FP64 residual, FP32
// correction). Stream-ordered on
// ctx->stream; the sweep-limit counter accumulates in the context status words.
// The pass's FP32 sweeps stop after a sweep whose rotations all stayed below 1e-2 rad: quadratic convergence
// leaves eigenvector mixing of O(1e-4), well inside the refinement's first-order range (|S'_kl| < 0.1 |gap|
// means mixing < 0.1), whose update then leaves O(1e-8), under the complex64 output's rounding. An FP32
// emulation of the sweeps gives 5.07 instead of 5.99 sweeps per warp of four matrices.
constexpr float PASS_ANGLE_STOP = 1e-2f;

static Eigh16Args pass_args(epb_ctx* ctx, const float* Hp, int64_t batch, float2* V32, float2* U) {
  Eigh16Args b{};
  b.Hp = Hp;
  b.U32 = U;
  b.n = E16;
  b.batch = batch;
  b.max_sweeps = 20;
  b.nonconv = ctx->dstat + 0;
  b.refine = 1;
  b.V32 = V32;
  b.angle_stop = PASS_ANGLE_STOP;
  return b;
}

int eigh16_mixed_jacobi(epb_ctx* ctx, const float* Hp, int64_t batch, float2* V32) {
  if (batch == 0) return EPB_OK;
  Eigh16Args b = pass_args(ctx, Hp, batch, V32, nullptr);
  const int64_t blocks = std::min<int64_t>(cdiv(batch, 16), (int64_t)ctx->sm_count * 16);
  prof_begin(ctx, EPB_PROF_EIGH);
  eigh16_jacobi2c_kernel<<<(unsigned)blocks, 128, 0, ctx->stream>>>(b);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int eigh16_mixed_refine(epb_ctx* ctx, const float* Hp, int64_t batch, float2* V32, float2* U, int64_t* gap_list,
                        int* gap_count, int gap_cap, float gap_rel) {
  if (batch == 0) return EPB_OK;
  Eigh16Args b = pass_args(ctx, Hp, batch, V32, U);
  b.gap_list = gap_list;
  b.gap_count = gap_count;
  b.gap_cap = gap_cap;
  b.gap_rel = gap_rel;
  prof_begin(ctx, EPB_PROF_REFINE);
  refine_launch(ctx, b);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// FP64 H(x) of the listed near-degenerate matrices (see eigh16_fixup_launch): a 1024-thread block per
// matrix; thread (e, s) adds entry (e % 16, e / 16) over the R vectors r = s mod 4, eight independent
// partial sums each (the loop is bound by the latency of one pass over the 3 MB of H(R)); the four
// quarters are added in a fixed order into hbuf[t] (256 complex per listed matrix).
constexpr int FIX_RB = 1024, FIX_HT = 1024, FIX_T = 256;
__global__ void __launch_bounds__(FIX_HT) eigh16_fixup_h_kernel(const int64_t* __restrict__ list,
                                                                const int* __restrict__ count, int cap,
                                                                const double2* __restrict__ ham,
                                                                const int4* __restrict__ rv, int64_t nr,
                                                                const double* __restrict__ xk,
                                                                const double* __restrict__ xq, int64_t nq,
                                                                double2* __restrict__ hbuf) {
  __shared__ double2 ph[FIX_RB];
  __shared__ double2 Hq[4][E16 * E16];
  const int nfix = min(*count, cap);
  const int e = threadIdx.x & 255, sq = threadIdx.x >> 8;
  for (int t = blockIdx.x; t < nfix; t += gridDim.x) {
    const int64_t b = list[t];
    const int64_t kb = b / nq, q = b - kb * nq;
    const double x0 = xk[3 * kb] + xq[3 * q], x1 = xk[3 * kb + 1] + xq[3 * q + 1], x2 = xk[3 * kb + 2] + xq[3 * q + 2];
    double2 acc[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc[u] = make_double2(0.0, 0.0);
    for (int64_t r0 = 0; r0 < nr; r0 += FIX_RB) {
      const int64_t r1 = nr - r0 < FIX_RB ? nr : r0 + FIX_RB;
      __syncthreads();
      for (int64_t r = r0 + threadIdx.x; r < r1; r += FIX_HT) {
        const int4 R = rv[r];
        ph[r - r0] = cis2pi(rdotx(R.x, R.y, R.z, x0, x1, x2));
      }
      __syncthreads();
      int64_t r = r0 + sq;
      for (; r + 28 < r1; r += 32) {
#pragma unroll
        for (int u = 0; u < 8; ++u) cfma(acc[u], ham[e + (r + 4 * u) * (E16 * E16)], ph[r + 4 * u - r0]);
      }
      for (; r < r1; r += 4) cfma(acc[0], ham[e + r * (E16 * E16)], ph[r - r0]);
    }
    double2 h = acc[0];
#pragma unroll
    for (int u = 1; u < 8; ++u) h = make_double2(h.x + acc[u].x, h.y + acc[u].y);
    Hq[sq][e] = h;
    __syncthreads();
    if (sq == 0)
      hbuf[(int64_t)t * (E16 * E16) + e] =
          make_double2((Hq[0][e].x + Hq[1][e].x) + (Hq[2][e].x + Hq[3][e].x),
                       (Hq[0][e].y + Hq[1][e].y) + (Hq[2][e].y + Hq[3][e].y));
    __syncthreads();  // ph and Hq are rewritten for the next matrix
  }
}

// FP64 re-solve of the listed matrices from their FP64 H(x) in hbuf, a 256-thread block per matrix, thread e
// owning entry (e % 16, e / 16):
//  * the refinement's complex64 eigenvectors V as the start: Lowdin orthonormalisation in FP64,
//    V' = V (I - F / 2), F = V^H V - I (leaves O(F^2) = 1e-14), then W = (H + sigma I) V';
//  * warp 0 runs the FP64 one-sided Jacobi on the columns of W, which are orthogonal except within the
//    near-degenerate pairs, so two or three sweeps finish it; the normalised columns are the eigenvectors
//    (both half-warps on the same matrix, the first writes them sorted).
__global__ void __launch_bounds__(FIX_T) eigh16_fixup_kernel(const int64_t* __restrict__ list, const int* __restrict__ count,
                                                             int cap, const double2* __restrict__ hbuf,
                                                             float2* __restrict__ U32) {
  __shared__ double2 Hs[E16 * E16];  // H[i][j] at i + 16 j
  __shared__ double2 Vs[E16 * E16];  // V[i][l] at i + 16 l
  __shared__ double2 Fs[E16 * E16];  // F[k][l] at k + 16 l, then W
  __shared__ double red[FIX_T / 32];
  const int nfix = min(*count, cap);
  const int e = threadIdx.x, lane = threadIdx.x & 31, ei = e & 15, el = e >> 4;
  for (int t = blockIdx.x; t < nfix; t += gridDim.x) {
    const int64_t b = list[t];
    const float2 v32 = U32[b * (E16 * E16) + e];
    Vs[e] = make_double2(v32.x, v32.y);
    const double2 h = hbuf[(int64_t)t * (E16 * E16) + e];
    Hs[e] = h;
    // sigma = 1.1 ||H||_F
    double f2 = h.x * h.x + h.y * h.y;
    for (int o = 16; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    if (lane == 0) red[e >> 5] = f2;
    __syncthreads();
    double hf = 0.0;
#pragma unroll
    for (int w = 0; w < FIX_T / 32; ++w) hf += red[w];
    const double sigma = hf > 0.0 ? 1.1 * sqrt(hf) : 1.0;
    // F = V^H V - I
    {
      double2 g = make_double2(ei == el ? -1.0 : 0.0, 0.0);
#pragma unroll
      for (int i = 0; i < E16; ++i) cfma_conj(g, Vs[i + E16 * ei], Vs[i + E16 * el]);
      Fs[e] = g;
    }
    __syncthreads();
    // V' = V - V F / 2
    double2 vp = Vs[e];
    {
      double2 c = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < E16; ++k) cfma(c, Vs[ei + E16 * k], Fs[k + E16 * el]);
      vp = make_double2(vp.x - 0.5 * c.x, vp.y - 0.5 * c.y);
    }
    __syncthreads();
    Vs[e] = vp;
    __syncthreads();
    // W = (H + sigma I) V'
    {
      double2 w = make_double2(sigma * vp.x, sigma * vp.y);
#pragma unroll
      for (int j = 0; j < E16; ++j) cfma(w, Hs[ei + E16 * j], Vs[j + E16 * el]);
      Fs[e] = w;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int l = lane & 15;
      double2 col[E16];
#pragma unroll
      for (int i = 0; i < E16; ++i) col[i] = Fs[i + E16 * l];
      onesided_sweeps<double>(col, 1e-15, 30);
      double nr2 = 0.0;
#pragma unroll
      for (int i = 0; i < E16; ++i) nr2 += col[i].x * col[i].x + col[i].y * col[i].y;
      const double inv = 1.0 / sqrt(nr2);
      double2 v[E16];
#pragma unroll
      for (int i = 0; i < E16; ++i) v[i] = make_double2(col[i].x * inv, col[i].y * inv);
      Eigh16Args a{};
      a.U32 = U32;
      a.n = E16;
      write_sorted(a, b, lane < 16, lane, l, E16, sqrt(nr2) - sigma, v);
    }
    __syncthreads();  // the shared matrices are rewritten for the next matrix
  }
}

int eigh16_fixup_launch(epb_ctx* ctx, const int64_t* list, const int* count, int cap, const double2* ham,
                        const int4* rv, int64_t nr, const double* xk, const double* xq, int64_t nq, float2* U32,
                        double2* hbuf) {
  if (cap <= 0) return EPB_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(cap, (int64_t)ctx->sm_count);
  prof_begin(ctx, EPB_PROF_REFINE);
  eigh16_fixup_h_kernel<<<grid, FIX_HT, 0, ctx->stream>>>(list, count, cap, ham, rv, nr, xk, xq, nq, hbuf);
  ++ctx->launches;
  eigh16_fixup_kernel<<<grid, FIX_T, 0, ctx->stream>>>(list, count, cap, hbuf, U32);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

}  // namespace epb
