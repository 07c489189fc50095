// Rotation + |g|^2 fold + in-place reduction of the mixed pass on the warp-level tensor cores
// (mma.sync m16n8k16, f16 operands, f32 accumulate), nw = 16 electrons, nm = 12 modes:
//
//   T[m, c]    = sum_iw conj(ukq[iw, m]) g[iw, c]       c = (n, jm), 16 x 192 per (k, q) block
//   ep[m, n, nu] = sum_jm T[m, (n, jm)] uph[jm, nu]      16 x 12 per n
//   g2 = |ep|^2 / (2 omega[nu, q]), summed into g2sum[nu, k]; full blocks of the sampled q written out
//
// (src/wannier_to_bloch_batched.jl:442-455, ext/ElectronPhononCUDAExt.jl:146-201). The per-(k, q) matrices
// are far below the smallest tcgen05 tile (M >= 64 with one operand shared by the whole tile), while a
// 16 x 16 x 16 warp MMA matches the 16-band rotation exactly, so one warp owns one (k, q) block:
//
//  * stage 1 as a real GEMM with M = 32 rows (Re T, Im T), K = 32 (Re g, Im g), N = 192 combos:
//      [Re T; Im T] = [[Re u^T, Im u^T]; [-Im u^T, Re u^T]] [Re g; Im g],
//    24 n8 tiles; the A fragments (from u) are loaded once per block, the B fragments (g) straight from
//    global memory with two 16-byte loads per lane per tile (fully coalesced: a tile is 1 KB);
//  * stage 2 per n with M = 16 (m), K = 32 (Re T jm 0..11 | pad | Im T jm 0..11 | pad), N = 24 columns
//    (Re ep, Im ep interleaved per mode, so one lane holds both parts of its modes). Stage 1's f32
//    accumulator fragment of an n8 tile is exactly one half of stage 2's A fragment, so T never leaves
//    registers. To avoid wasting a third of stage 1 on jm padding, the tiles of a pair of bands (n0, n1)
//    are (n0, jm 0..7), (n1, jm 0..7) and (n0, jm 8..11 | n1, jm 8..11): the shared tile feeds both
//    bands' stage 2, whose uph operand has zero rows where the other band's values sit.
//
// Precision (the |g|^2 <= 1e-5 per-block bar of the pass): every operand is split into two f16 planes,
// v = hi + lo (22 bits), the products hi*hi go to one f32 accumulator and hi*lo + lo*hi to another (so the
// small corrections are not truncated against the large sum), added in FP32 with round-to-nearest. The
// f16 range is respected by exact power-of-two scales: g by a bound on max|g| derived from the kR->kq
// operand (|g| <= 2 nr_ep max(|Re G|, |Im G|)) so that |g| <= 2^12 and |T| <= 2^14, u_ph by the bound on
// its largest element; the unitary ukq needs none. |ep|^2 is unscaled in FP32 before the fold.
#include <cuda_fp16.h>

#include <algorithm>

#include "epb_common.cuh"

namespace epb {

namespace {

__device__ __forceinline__ uint32_t h2bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// Split (x0, x1) into f16x2 planes hi + lo (x0 in the low half).
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(x0, x1);
  const float2 f = __half22float2(h);
  hi = h2bits(h);
  lo = h2bits(__floats2half2_rn(x0 - f.x, x1 - f.y));
}

__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// A fragment of a 16 x 16 f16 operand, hi and lo planes.
struct AFrag {
  uint32_t h[4], l[4];
};
// B fragment of a 16 x 8 operand.
struct BFrag {
  uint32_t h[2], l[2];
};

// acc_lead += A.h B.h;  acc_corr += A.h B.l + A.l B.h
__device__ __forceinline__ void mma3(float (&lead)[4], float (&corr)[4], const AFrag& a, const BFrag& b) {
  mma16816(lead, a.h[0], a.h[1], a.h[2], a.h[3], b.h[0], b.h[1]);
  mma16816(corr, a.h[0], a.h[1], a.h[2], a.h[3], b.l[0], b.l[1]);
  mma16816(corr, a.l[0], a.l[1], a.l[2], a.l[3], b.h[0], b.h[1]);
}

__device__ __forceinline__ void zero4(float (&v)[4]) { v[0] = v[1] = v[2] = v[3] = 0.f; }

// The lane's g values of one stage-1 tile column: combo c (complex column of 16 iw), rows iw = 2t, 2t+1
// (first float4: re, im, re, im) and 2t+8, 2t+9 (second).
struct GCol {
  float4 a, b;
};

__device__ __forceinline__ GCol load_gcol(const float* __restrict__ gb, int combo, int t) {
  const float4* p = reinterpret_cast<const float4*>(gb + 32 * combo + 4 * t);
  GCol c;
  c.a = __ldcs(p);      // read once: do not keep in L2
  c.b = __ldcs(p + 4);
  return c;
}

// B fragments (Re g for K step 0, Im g for K step 1) of a tile column, scaled by s.
__device__ __forceinline__ void gfrags(const GCol& c, float s, BFrag& re, BFrag& im) {
  split2(c.a.x * s, c.a.z * s, re.h[0], re.l[0]);
  split2(c.b.x * s, c.b.z * s, re.h[1], re.l[1]);
  split2(c.a.y * s, c.a.w * s, im.h[0], im.l[0]);
  split2(c.b.y * s, c.b.w * s, im.h[1], im.l[1]);
}

// Stage-1 tile: Re T (lead, corr) and Im T (lead, corr) for the tile's 8 combos.
struct S1Acc {
  float rl[4], rc[4], il[4], ic[4];
};

__device__ __forceinline__ void stage1_tile(S1Acc& acc, const AFrag& X, const AFrag& Y, const AFrag& Yn,
                                            const BFrag& gre, const BFrag& gim) {
  zero4(acc.rl);
  zero4(acc.rc);
  zero4(acc.il);
  zero4(acc.ic);
  mma3(acc.rl, acc.rc, X, gre);   // Re T  = Re u^T Re g + Im u^T Im g
  mma3(acc.rl, acc.rc, Y, gim);
  mma3(acc.il, acc.ic, Yn, gre);  // Im T = -Im u^T Re g + Re u^T Im g
  mma3(acc.il, acc.ic, X, gim);
}

// Stage-2 A fragment halves from a stage-1 tile: T = lead + corr (FP32, round-to-nearest), split in f16.
// lo16 holds rows g (c0, c1), hi16 rows g + 8 (c2, c3): a0a1 / a2a3 (or a4a5 / a6a7) of the next MMA.
struct THalf {
  uint32_t rh[2], rl[2], ih[2], il[2];
};

__device__ __forceinline__ THalf thalf(const S1Acc& a) {
  THalf t;
  split2(a.rl[0] + a.rc[0], a.rl[1] + a.rc[1], t.rh[0], t.rl[0]);
  split2(a.rl[2] + a.rc[2], a.rl[3] + a.rc[3], t.rh[1], t.rl[1]);
  split2(a.il[0] + a.ic[0], a.il[1] + a.ic[1], t.ih[0], t.il[0]);
  split2(a.il[2] + a.ic[2], a.il[3] + a.ic[3], t.ih[1], t.il[1]);
  return t;
}

// Stage-2 B fragments of u_ph for one n8 tile of the 24 output columns: K step 0 (Re T rows) and K step 1
// (Im T rows); b01 rows kk = 2t, 2t+1 (jm 0..7), b23 rows kk = 2t+8, 2t+9 in two variants: for the first
// band of a pair jm = kk (zero for kk >= 12, i.e. lanes t >= 2), for the second zero for kk < 12 (lanes
// t < 2) and jm = kk - 4. Each lane keeps only its nonzero variant, v.
struct PhFrag {
  uint32_t b01h[2], b01l[2];   // [ks]
  uint32_t vh[2], vl[2];       // [ks]
};

struct RotArgs {
  const float* g;        // (k, q) blocks of 2 nw^2 nm floats (complex64 g[iw, n, jm]), block stride g_stride
  int64_t g_stride;
  const float2* ukq;     // (nw, nw) complex64 per block
  const float2* uph;     // (nm, nm) complex64 per q
  const float* inv2w;    // (nm, nq) 1 / (2 omega)
  const unsigned* gmax;  // max |Re G|, |Im G| of the kR->kq operand (float bits, as written, pre-scale gscale)
  const unsigned* phmax; // max |Re uph|, |Im uph| (float bits)
  float gscale_inv;      // the kR->kq operand's power-of-two pre-scale undone (g = GEMM(G) with G scaled back)
  int nr_ep;
  int64_t nkb, nq;
  double* partial;       // (nm, warps, nkb): each warp's sum over its blocks of k, in a fixed slot
  double* sample;        // (nw, nw, nm, nsamp, nkb) or null
  int64_t stride, nsamp;
};

// exact power of two p with max_abs * p <= 2^target (1 when max_abs is 0 or not finite)
__device__ __forceinline__ float pow2_scale(float max_abs, int target) {
  if (!(max_abs > 0.f) || !isfinite(max_abs)) return 1.f;
  int e;
  frexpf(max_abs, &e);  // max_abs < 2^e
  return ldexpf(1.f, target - e);
}

}  // namespace

constexpr int ROT_MMA_WARPS = 12;

__global__ void __launch_bounds__(32 * ROT_MMA_WARPS, 1) eph_rot_mma_kernel(RotArgs a) {
  constexpr int NW = 16, NM = 12, ND = NW * NW * NM;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, t = lane & 3;  // mma group (row / column) and thread in group
  // scales (uniform): |g| <= 2 nr_ep max|G| -> <= 2^12; |uph| -> <= 1
  const float gmaxv = __uint_as_float(*a.gmax) * a.gscale_inv * 2.f * (float)a.nr_ep;
  const float sg = pow2_scale(gmaxv, 12);
  const float sph = pow2_scale(__uint_as_float(*a.phmax), 0);
  const float unscale = 1.f / (sg * sph);
  const float unscale2 = unscale * unscale;

  const int64_t nblk = a.nkb * a.nq;
  const int64_t nwarps = (int64_t)gridDim.x * ROT_MMA_WARPS;
  const int64_t gw = (int64_t)blockIdx.x * ROT_MMA_WARPS + warp;
  int64_t kcur = -1;
  double part[3] = {0.0, 0.0, 0.0};  // modes t, t + 4, t + 8 of block rows g, g + 8 over this warp's blocks of k
  // A warp meets each k in one run of consecutive blocks (k = blk / nq grows with blk), so its sum for k
  // goes to the slot (k, gw) with a plain store; rot_reduce_kernel adds the slots in a fixed order.
  auto flush = [&](int64_t k) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double v = part[j];
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 16);
      if (gq == 0) a.partial[(t + 4 * j) + NM * (gw + nwarps * k)] = v;
      part[j] = 0.0;
    }
  };

  for (int64_t blk = gw; blk < nblk; blk += nwarps) {
    const int64_t kl = blk / a.nq, q = blk - kl * a.nq;
    if (kl != kcur) {
      if (kcur >= 0) flush(kcur);
      kcur = kl;
    }
    const float* gb = a.g + blk * a.g_stride;
    // ---- stage-1 A fragments from u (rows m = gq, gq + 8; K = iw 2t, 2t+1, 2t+8, 2t+9) ----
    AFrag X, Y, Yn;  // Re u^T, Im u^T, -Im u^T
    {
      const float4* ub = reinterpret_cast<const float4*>(a.ukq + blk * NW * NW);
      // u[iw, m] at float2 index iw + 16 m: float4 index (iw + 16 m) / 2
      const float4 u00 = ub[(2 * t + 16 * gq) >> 1], u01 = ub[(2 * t + 8 + 16 * gq) >> 1];
      const float4 u10 = ub[(2 * t + 16 * (gq + 8)) >> 1], u11 = ub[(2 * t + 8 + 16 * (gq + 8)) >> 1];
      split2(u00.x, u00.z, X.h[0], X.l[0]);
      split2(u10.x, u10.z, X.h[1], X.l[1]);
      split2(u01.x, u01.z, X.h[2], X.l[2]);
      split2(u11.x, u11.z, X.h[3], X.l[3]);
      split2(u00.y, u00.w, Y.h[0], Y.l[0]);
      split2(u10.y, u10.w, Y.h[1], Y.l[1]);
      split2(u01.y, u01.w, Y.h[2], Y.l[2]);
      split2(u11.y, u11.w, Y.h[3], Y.l[3]);
      split2(-u00.y, -u00.w, Yn.h[0], Yn.l[0]);
      split2(-u10.y, -u10.w, Yn.h[1], Yn.l[1]);
      split2(-u01.y, -u01.w, Yn.h[2], Yn.l[2]);
      split2(-u11.y, -u11.w, Yn.h[3], Yn.l[3]);
    }
    // ---- stage-2 B fragments from u_ph (columns 2 nu + reim, nu = 4 nt + gq / 2) ----
    PhFrag P[3];
    {
      const float2* pb = a.uph + q * NM * NM;
      const int reim = gq & 1;
#pragma unroll
      for (int nt = 0; nt < 3; ++nt) {
        const int nu = 4 * nt + (gq >> 1);
        const float2* pc = pb + NM * nu;  // uph[jm, nu] = pc[jm]
        auto val = [&](int jm, int ks) -> float {  // B[kk = jm (+16 ks), col]
          if (jm < 0 || jm >= NM) return 0.f;
          const float2 v = pc[jm];
          const float x = ks == 0 ? (reim ? v.y : v.x) : (reim ? v.x : -v.y);
          return x * sph;
        };
        // rows kk = 2t+8, 2t+9: jm = kk for t < 2 (first band), jm = kk - 4 for t >= 2 (second band)
        const int jv = t < 2 ? 2 * t + 8 : 2 * t + 4;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          split2(val(2 * t, ks), val(2 * t + 1, ks), P[nt].b01h[ks], P[nt].b01l[ks]);
          split2(val(jv, ks), val(jv + 1, ks), P[nt].vh[ks], P[nt].vl[ks]);
        }
      }
    }
    const float* w2 = a.inv2w + q * NM;
    float wq[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) wq[j] = w2[t + 4 * j] * unscale2;
    const bool samp = a.sample && (q % a.stride == 0);
    double* sq = samp ? a.sample + (kl * a.nsamp + q / a.stride) * (int64_t)ND : nullptr;
    float bsum[3] = {0.f, 0.f, 0.f};

    // combos of the lane's column in the three tiles of pair p: stored combo index n + 16 jm
    auto combo = [&](int p, int tile) -> int {
      const int n0 = 2 * p;
      if (tile == 0) return n0 + 16 * gq;
      if (tile == 1) return n0 + 1 + 16 * gq;
      return gq < 4 ? n0 + 16 * (8 + gq) : n0 + 1 + 16 * (8 + gq - 4);
    };
    GCol gc[3];
#pragma unroll
    for (int tl = 0; tl < 3; ++tl) gc[tl] = load_gcol(gb, combo(0, tl), t);
#pragma unroll 1
    for (int p = 0; p < NW / 2; ++p) {
      // ---- stage 1 for the pair's three tiles, one at a time (each tile's g column is replaced by the next
      // pair's request as soon as it is split) ----
      THalf th[3];
#pragma unroll
      for (int tl = 0; tl < 3; ++tl) {
        BFrag gre, gim;
        gfrags(gc[tl], sg, gre, gim);
        if (p + 1 < NW / 2) gc[tl] = load_gcol(gb, combo(p + 1, tl), t);
        S1Acc s1;
        stage1_tile(s1, X, Y, Yn, gre, gim);
        th[tl] = thalf(s1);
      }
      const THalf &tA = th[0], &tB = th[1], &tC = th[2];
      // ---- stage 2 for n0 = 2p (tiles A, C; variant 0) and n1 = 2p + 1 (tiles B, C; variant 1) ----
#pragma unroll
      for (int nb = 0; nb < 2; ++nb) {
        const THalf& tf = nb == 0 ? tA : tB;
        // A fragments: K step 0 = Re T (a0a1 a2a3 from tile A/B, a4a5 a6a7 from tile C), step 1 = Im T
        AFrag ar, ai;
        ar.h[0] = tf.rh[0]; ar.h[1] = tf.rh[1]; ar.h[2] = tC.rh[0]; ar.h[3] = tC.rh[1];
        ar.l[0] = tf.rl[0]; ar.l[1] = tf.rl[1]; ar.l[2] = tC.rl[0]; ar.l[3] = tC.rl[1];
        ai.h[0] = tf.ih[0]; ai.h[1] = tf.ih[1]; ai.h[2] = tC.ih[0]; ai.h[3] = tC.ih[1];
        ai.l[0] = tf.il[0]; ai.l[1] = tf.il[1]; ai.l[2] = tC.il[0]; ai.l[3] = tC.il[1];
        const int n = 2 * p + nb;
#pragma unroll
        for (int nt = 0; nt < 3; ++nt) {
          BFrag br, bi;
          br.h[0] = P[nt].b01h[0]; br.l[0] = P[nt].b01l[0];
          bi.h[0] = P[nt].b01h[1]; bi.l[0] = P[nt].b01l[1];
          const bool mine = (nb == 0) == (t < 2);  // this lane's rows kk 2t+8, 2t+9 belong to band nb
          br.h[1] = mine ? P[nt].vh[0] : 0u;
          br.l[1] = mine ? P[nt].vl[0] : 0u;
          bi.h[1] = mine ? P[nt].vh[1] : 0u;
          bi.l[1] = mine ? P[nt].vl[1] : 0u;
          float lead[4], corr[4];
          zero4(lead);
          zero4(corr);
          mma3(lead, corr, ar, br);
          mma3(lead, corr, ai, bi);
          // columns 2t (Re ep), 2t + 1 (Im ep) of mode nu = 4 nt + t; rows m = gq (c0, c1), gq + 8 (c2, c3)
          const float e0r = lead[0] + corr[0], e0i = lead[1] + corr[1];
          const float e1r = lead[2] + corr[2], e1i = lead[3] + corr[3];
          const float v0 = (e0r * e0r + e0i * e0i) * wq[nt];
          const float v1 = (e1r * e1r + e1i * e1i) * wq[nt];
          bsum[nt] += v0 + v1;
          if (samp) {
            const int nu = 4 * nt + t;
            sq[gq + NW * n + NW * NW * nu] = (double)v0;
            sq[gq + 8 + NW * n + NW * NW * nu] = (double)v1;
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) part[j] += (double)bsum[j];
  }
  if (kcur >= 0) flush(kcur);
}

// g2sum[nu, k] += sum over the warps' slots in a fixed order: one 64-thread block per (mode, k), so that the
// blocks fit beside the pipeline's other kernels; each thread adds every 64th slot, then a fixed tree.
constexpr int ROT_RED_THREADS = 64;
__global__ void __launch_bounds__(ROT_RED_THREADS) rot_reduce_kernel(const double* __restrict__ partial,
                                                                     int64_t nwarps, double* __restrict__ g2sum) {
  constexpr int NM = 12;
  __shared__ double red[ROT_RED_THREADS / 32];
  const int nu = blockIdx.x % NM;
  const int64_t k = blockIdx.x / NM;
  double s = 0.0;
  for (int64_t w = threadIdx.x; w < nwarps; w += ROT_RED_THREADS) s += partial[nu + NM * (w + nwarps * k)];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int p = 0; p < ROT_RED_THREADS / 32; ++p) t += red[p];
    g2sum[nu + NM * k] += t;
  }
}

int64_t rot_mma_partial_doubles(epb_ctx* ctx, int64_t nkb) { return nkb * (int64_t)ctx->sm_count * ROT_MMA_WARPS * 12; }

int rot_mma_launch(epb_ctx* ctx, const float* g, int64_t g_stride, const float2* ukq, const float2* uph,
                   const float* inv2w, const unsigned* gmax, const unsigned* phmax, float gscale_inv, int nr_ep,
                   int64_t nkb, int64_t nq, double* g2sum, double* partial, double* sample, int64_t stride,
                   int64_t nsamp) {
  RotArgs a;
  a.g = g;
  a.g_stride = g_stride;
  a.ukq = ukq;
  a.uph = uph;
  a.inv2w = inv2w;
  a.gmax = gmax;
  a.phmax = phmax;
  a.gscale_inv = gscale_inv;
  a.nr_ep = nr_ep;
  a.nkb = nkb;
  a.nq = nq;
  a.partial = partial;
  a.sample = sample;
  a.stride = stride < 1 ? 1 : stride;
  a.nsamp = nsamp;
  const int64_t nblk = nkb * nq;
  if (nblk == 0) return EPB_OK;
  const int64_t want = cdiv(nblk, ROT_MMA_WARPS);
  const unsigned grid = (unsigned)std::min<int64_t>(want, (int64_t)ctx->sm_count);
  const int64_t nwarps = (int64_t)grid * ROT_MMA_WARPS;
  EPB_CUDA(cudaMemsetAsync(partial, 0, sizeof(double) * 12 * nwarps * nkb, ctx->stream));
  eph_rot_mma_kernel<<<grid, 32 * ROT_MMA_WARPS, 0, ctx->stream>>>(a);
  EPB_LAUNCH_CHECK();
  rot_reduce_kernel<<<(unsigned)(12 * nkb), ROT_RED_THREADS, 0, ctx->stream>>>(partial, nwarps, g2sum);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

}  // namespace epb
