// Split-precision complex Fourier contractions on the 5th-generation tensor cores (tcgen05).
//
// A complex GEMM C = A B (A: M x K op_r block, B: K x N phase) is run as a real GEMM with
// re/im-interleaved rows,
//     A2[2i, :]   = [ Re A_i | -Im A_i ],    A2[2i+1, :] = [ Im A_i | Re A_i ],
//     B2[:, j]    = [ Re B_j ;  Im B_j ],
// so that C2 = A2 B2 holds (Re C_ij, Im C_ij) as consecutive rows, i.e. column j of C2 is the
// complex64 column j of C. Every real operand value v is split into bf16 planes
// v = v_h + v_m + v_l (each the bf16 rounding of the remainder), and the product is accumulated
// in FP32 TMEM from the six terms h*h + h*m + m*h + m*m + h*l + l*h (split BF16x3): the dropped
// terms are O(2^-24) relative, the FP32 level.
//
// Operands live in global memory already in the shared-memory image the MMA reads: 128-row x
// 64-column K-major tiles with the SWIZZLE_128B pattern, 16 KB each, planes stored one after the
// other. A stage is therefore a handful of plain 1-D bulk copies (cp.async.bulk) completing on an
// mbarrier; no tensor map and no multicast is involved.
//
// Kernel: persistent, one CTA per SM, 6 warps:
//   warp 0      bulk-copy producer (one thread), STAGES-deep ring of operand stages
//   warp 1      MMA issuer (one thread): 4 K-substeps x 6 products per stage into a TMEM
//               accumulator of 128 lanes x NT columns, restarted for every 64-wide K chunk; two
//               accumulators alternate by chunk so the epilogue of one chunk overlaps the next chunk's MMAs
//   warps 2-5   epilogue: tcgen05.ld of each chunk's accumulators, added into FP32 registers with
//               round-to-nearest (the tensor core's own accumulation truncates), FP32 stores to C
// Every wait is bounded (clock64 budget); on timeout the kernel raises an error flag, drains its
// own copies and MMAs, frees TMEM and returns (EPB_ERR_TIMEOUT on the host).
#include <algorithm>
#include <cstring>

#include "epb_common.cuh"

#include "epb_umma.cuh"

namespace epb {

using namespace umma;

constexpr int TILE_BYTES = 16384;  // 128 rows x 64 bf16

// ---------------------------------------------------------------------------------------------
// Split of a real value into NPL bf16 (or f16) planes.
template <bool BF16>
__device__ __forceinline__ uint16_t to_half_bits(double v) {
  if (BF16) {
    __nv_bfloat16 h = __double2bfloat16(v);
    return *reinterpret_cast<uint16_t*>(&h);
  } else {
    __half h = __double2half(v);
    return *reinterpret_cast<uint16_t*>(&h);
  }
}
template <bool BF16>
__device__ __forceinline__ double from_half_bits(uint16_t b) {
  if (BF16) {
    __nv_bfloat16 h = *reinterpret_cast<__nv_bfloat16*>(&b);
    return (double)__bfloat162float(h);
  } else {
    __half h = *reinterpret_cast<__half*>(&b);
    return (double)__half2float(h);
  }
}

// Store v split into NPL planes at byte offset `off` of plane 0 (planes `plane_bytes` apart).
template <bool BF16, int NPL>
__device__ __forceinline__ void store_split(uint8_t* base, int64_t plane_bytes, int64_t off, double v) {
  double r = v;
#pragma unroll
  for (int p = 0; p < NPL; ++p) {
    uint16_t b = to_half_bits<BF16>(r);
    *reinterpret_cast<uint16_t*>(base + p * plane_bytes + off) = b;
    r -= from_half_bits<BF16>(b);
  }
}

// Global byte offset of element (row, k) in a pre-tiled plane with KC 64-wide K chunks.
__device__ __forceinline__ int64_t tiled_offset(int64_t row, int64_t k, int64_t KC) {
  int64_t rt = row >> 7, kc = k >> 6;
  return (rt * KC + kc) * TILE_BYTES + sw128_offset((uint32_t)(row & 127), (uint32_t)(k & 63));
}

// ---------------------------------------------------------------------------------------------
// Packers. Each thread produces 8 consecutive K' values of one row, i.e. one 16-byte chunk of the
// swizzled tile per plane. The K' axis holds the cos coefficients at [0, K) and the sin
// coefficients at [koff, koff + K) with koff = round_up(K, 8); everything else is zero.

template <bool BF16, int NPL>
__device__ __forceinline__ void store_split8(uint8_t* base, int64_t plane_bytes, int64_t off, const double* v) {
  double r[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) r[e] = v[e];
#pragma unroll
  for (int p = 0; p < NPL; ++p) {
    uint16_t b[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      b[e] = to_half_bits<BF16>(r[e]);
      r[e] -= from_half_bits<BF16>(b[e]);
    }
    uint4 w;
    w.x = (uint32_t)b[0] | ((uint32_t)b[1] << 16);
    w.y = (uint32_t)b[2] | ((uint32_t)b[3] << 16);
    w.z = (uint32_t)b[4] | ((uint32_t)b[5] << 16);
    w.w = (uint32_t)b[6] | ((uint32_t)b[7] << 16);
    *reinterpret_cast<uint4*>(base + p * plane_bytes + off) = w;
  }
}

// The same split of FP32 values, in FP32 arithmetic: each remainder is exact in FP32, so the planes sum
// to the FP32 value exactly (while the remainders stay normal, |v| >= 2^-100) and its rounding (2^-24
// relative) is the only difference from the FP64 split.
template <bool BF16>
__device__ __forceinline__ uint16_t f32_to_half_bits(float v) {
  if (BF16) {
    __nv_bfloat16 h = __float2bfloat16_rn(v);
    return *reinterpret_cast<uint16_t*>(&h);
  } else {
    __half h = __float2half_rn(v);
    return *reinterpret_cast<uint16_t*>(&h);
  }
}
template <bool BF16>
__device__ __forceinline__ float half_bits_to_f32(uint16_t b) {
  if (BF16) return __bfloat162float(*reinterpret_cast<__nv_bfloat16*>(&b));
  return __half2float(*reinterpret_cast<__half*>(&b));
}
template <bool BF16, int NPL>
__device__ __forceinline__ void store_split8_f32(uint8_t* base, int64_t plane_bytes, int64_t off, const float* v) {
  float r[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) r[e] = v[e];
#pragma unroll
  for (int p = 0; p < NPL; ++p) {
    uint16_t b[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      b[e] = f32_to_half_bits<BF16>(r[e]);
      r[e] -= half_bits_to_f32<BF16>(b[e]);
    }
    uint4 w;
    w.x = (uint32_t)b[0] | ((uint32_t)b[1] << 16);
    w.y = (uint32_t)b[2] | ((uint32_t)b[3] << 16);
    w.z = (uint32_t)b[4] | ((uint32_t)b[5] << 16);
    w.w = (uint32_t)b[6] | ((uint32_t)b[7] << 16);
    *reinterpret_cast<uint4*>(base + p * plane_bytes + off) = w;
  }
}

__host__ __device__ __forceinline__ int64_t sin_offset(int64_t K) { return (K + 7) / 8 * 8; }
__host__ __device__ __forceinline__ int64_t kchunks(int64_t K) { return (sin_offset(K) + K + 63) / 64; }

// Generic complex operand A (M x K complex, column-major, leading dim ld) -> A2 rows 2i / 2i+1.
template <bool BF16, int NPL>
__global__ void pack_a_complex_kernel(const double2* __restrict__ a, int64_t ld, int64_t M, int64_t K,
                                      int64_t rows_pad, int64_t KC, uint8_t* __restrict__ planes,
                                      int64_t plane_bytes) {
  const int64_t nch = KC * 8, koff = sin_offset(K);
  const int64_t total = rows_pad * nch;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t ch = idx % nch, row = idx / nch;
    int64_t i = row >> 1;
    int part = (int)(row & 1);
    double v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      int64_t k = ch * 8 + e;
      double x = 0.0;
      if (i < M) {
        if (k < K) {
          double2 z = a[i + k * ld];
          x = part == 0 ? z.x : z.y;
        } else if (k >= koff && k < koff + K) {
          double2 z = a[i + (k - koff) * ld];
          x = part == 0 ? -z.y : z.x;
        }
      }
      v[e] = x;
    }
    store_split8<BF16, NPL>(planes, plane_bytes, tiled_offset(row, ch * 8, KC), v);
  }
}

// Hermitian operand (nw x nw per R, column-major op_r (nw^2 x K)) -> packed real rows:
// rows [0, nw(nw+1)/2): Re H_ij (i <= j, column by column), then Im H_ij (i < j).
__device__ __forceinline__ void herm_row_to_ij(int row, int nw, int& i, int& j, int& part) {
  const int nre = nw * (nw + 1) / 2;
  int r = row;
  part = 0;
  if (r >= nre) {
    part = 1;
    r -= nre;
    int jj = 1;
    while (r >= jj) {
      r -= jj;
      ++jj;
    }
    i = r;
    j = jj;
    return;
  }
  int jj = 0;
  while (r >= jj + 1) {
    r -= jj + 1;
    ++jj;
  }
  i = r;
  j = jj;
}

template <bool BF16, int NPL>
__global__ void pack_a_herm_kernel(const double2* __restrict__ op, int nw, int64_t K, int64_t rows_pad,
                                   int64_t KC, uint8_t* __restrict__ planes, int64_t plane_bytes) {
  const int64_t nch = KC * 8, koff = sin_offset(K);
  const int64_t total = rows_pad * nch;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t ch = idx % nch, row = idx / nch;
    double v[8];
    int i = 0, j = 0, part = 0;
    const bool live = row < (int64_t)nw * nw;
    if (live) herm_row_to_ij((int)row, nw, i, j, part);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      int64_t k = ch * 8 + e;
      double x = 0.0;
      if (live) {
        if (k < K) {
          double2 z = op[(i + (int64_t)j * nw) + k * (int64_t)nw * nw];
          x = part == 0 ? z.x : z.y;        // cos coefficient: Re h (real row) / Im h (imag row)
        } else if (k >= koff && k < koff + K) {
          double2 z = op[(i + (int64_t)j * nw) + (k - koff) * (int64_t)nw * nw];
          x = part == 0 ? -z.y : z.x;       // sin coefficient: -Im h (real row) / Re h (imag row)
        }
      }
      v[e] = x;
    }
    store_split8<BF16, NPL>(planes, plane_bytes, tiled_offset(row, ch * 8, KC), v);
  }
}

// The Hermitian-packed rows of H(R) modulated by the phases of a batch of k points, for
//   H(k + q) = sum_R [H_R exp(2 pi i R.k)] exp(2 pi i R.q):
// batch b holds rows b * rows_pad .. b * rows_pad + nw^2 - 1 of A, and the B operand is the phase planes
// of the q list, shared by every k of the pass. Same row and K' layout as pack_a_herm_kernel.
template <bool BF16, int NPL>
__global__ void pack_a_herm_mod_kernel(const double2* __restrict__ op, const int4* __restrict__ rv, int nw,
                                       int64_t K, const double* __restrict__ xk, int64_t nk, int64_t rows_pad,
                                       int64_t KC, uint8_t* __restrict__ planes, int64_t plane_bytes) {
  const int64_t nch = KC * 8, koff = sin_offset(K);
  const int64_t total = nk * rows_pad * nch;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t rowg = idx / nch, ch = idx - rowg * nch;
    const int64_t b = rowg / rows_pad, row = rowg - b * rows_pad;
    double v[8];
    int i = 0, j = 0, part = 0;
    const bool live = row < (int64_t)nw * nw;
    if (live) herm_row_to_ij((int)row, nw, i, j, part);
    const double x0 = xk[3 * b], x1 = xk[3 * b + 1], x2 = xk[3 * b + 2];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int64_t kk = ch * 8 + e;
      double x = 0.0;
      if (live) {
        const bool cosc = kk < K, sinc = kk >= koff && kk < koff + K;
        if (cosc || sinc) {
          const int64_t p = cosc ? kk : kk - koff;
          const int4 r = rv[p];
          const double2 h = cmul(op[(i + (int64_t)j * nw) + p * (int64_t)nw * nw], cis2pi(rdotx(r.x, r.y, r.z, x0, x1, x2)));
          // cos coefficient: Re h (real row) / Im h (imag row); sin coefficient: -Im h / Re h
          x = cosc ? (part == 0 ? h.x : h.y) : (part == 0 ? -h.y : h.x);
        }
      }
      v[e] = x;
    }
    store_split8<BF16, NPL>(planes, plane_bytes, tiled_offset(rowg, ch * 8, KC), v);
  }
}

// Phase operand: row j of B2 = [cos 2 pi R.x_j | sin 2 pi R.x_j] (K-major), x_j = xa[:, p / nb] +
// xb[:, p % nb] with p = pidx[j] (pidx != null) or pair0 + j when xb != null (x_{k+q} for pairs of
// a k list and a q list), else x_j = xa[:, j].
// A thread writes 8 consecutive R of one point. The first is evaluated directly; an R that follows its
// predecessor by (1, 0, 0) (R lists are sorted by reverse(R), so R1 varies fastest) takes the previous
// value times exp(2 pi i x_1) (at most 7 products: a few 1e-16), any other R is evaluated directly. The values are rounded to FP32
// and split in FP32 (exact: the planes hold the FP32 value), so the kernel stays on the HBM write bound.
template <bool BF16, int NPL>
__global__ void pack_b_phase_kernel(const int4* __restrict__ rv, int64_t K, const double* __restrict__ xa,
                                    const double* __restrict__ xb, int64_t nb, const int64_t* __restrict__ pidx,
                                    int64_t pair0, int64_t N, int64_t rows_pad, int64_t KC,
                                    uint8_t* __restrict__ planes, int64_t plane_bytes) {
  const int koff = (int)sin_offset(K);
  const int ncos = koff / 8;  // chunks covering [0, koff)
  const int nch = (int)KC * 8;
  const int64_t total = rows_pad * ncos;  // one thread per (point, 8 R vectors): cos and sin chunks
  const bool idx32 = total <= 0x7fffffff;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t j;
    int ch;
    if (idx32) {
      const uint32_t i = (uint32_t)idx, jj = i / (uint32_t)ncos;
      j = jj;
      ch = (int)(i - jj * (uint32_t)ncos);
    } else {
      j = idx / ncos;
      ch = (int)(idx - j * ncos);
    }
    float c[8], sn[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) c[e] = sn[e] = 0.f;
    if (j < N) {
      double x0, x1, x2;
      if (xb) {
        const int64_t pj = pidx ? pidx[j] : pair0 + j;
        const int64_t ja = pj / nb, jb = pj - ja * nb;
        x0 = xa[3 * ja] + xb[3 * jb];
        x1 = xa[3 * ja + 1] + xb[3 * jb + 1];
        x2 = xa[3 * ja + 2] + xb[3 * jb + 2];
      } else {
        x0 = xa[3 * j];
        x1 = xa[3 * j + 1];
        x2 = xa[3 * j + 2];
      }
      const double2 step = cis2pi(x0);
      double2 z = make_double2(1.0, 0.0);
      int4 rp = make_int4(0, 0, 0, 0);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int q = ch * 8 + e;
        if (q < K) {
          const int4 r = rv[q];
          if (e > 0 && r.x == rp.x + 1 && r.y == rp.y && r.z == rp.z)
            z = cmul(z, step);
          else
            z = cis2pi(rdotx(r.x, r.y, r.z, x0, x1, x2));
          rp = r;
          c[e] = (float)z.x;
          sn[e] = (float)z.y;
        }
      }
    }
    store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(j, ch * 8, KC), c);
    store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(j, koff + ch * 8, KC), sn);
    // trailing zero chunks beyond koff + koff (when KC*64 > 2*koff)
    for (int z = 2 * ncos + ch; z < nch; z += ncos) {
      const float zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(j, (int64_t)z * 8, KC), zero);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// The GEMM kernel.
struct SplitGemmArgs {
  const uint8_t* A;
  const uint8_t* B;
  int64_t a_plane_bytes, b_plane_bytes;
  int KC;                     // 64-wide K chunks
  int64_t m_tiles, n_tiles;   // 128-row A tiles; NT-wide B column tiles
  int m_fastest;              // tile order: m fastest (B reuse) or n fastest (A reuse)
  int64_t m_tiles_per_batch;  // rows of a batch = m_tiles_per_batch * 128 (padded)
  int64_t m_valid;            // valid rows per batch
  int64_t n_valid;            // valid columns
  float* C;
  int64_t c_batch_stride, ldc_n;
  int* err;
  long long timeout;
  // grouped mode (grp != nullptr): group g owns the B column tiles [grp[g], grp[g + 1]) and multiplies the
  // A block grp_a[g] (m_tiles_per_batch tiles); m_tiles = m_tiles_per_batch, n_tiles = grp[ngrp]
  const int64_t* grp;
  const int64_t* grp_a;
  int64_t ngrp;
  // power-of-two scale applied to C in the epilogue (undoing an operand's pre-scale); 0 = none
  float cscale;
  // A-resident kernel: column tiles per work unit (a unit = one A tile and a run of column tiles)
  int64_t n_per_unit;
};

template <bool BF16, int NPL>
struct Products;
// Product lists (plane of A, plane of B), smallest terms first.
template <>
struct Products<true, 3> {  // split BF16x3: terms down to O(2^-16) relative kept
  static constexpr int N = 6;
  static __device__ __forceinline__ constexpr int a(int i) {
    return i == 0 ? 2 : i == 1 ? 0 : i == 2 ? 1 : i == 3 ? 1 : 0;
  }
  static __device__ __forceinline__ constexpr int b(int i) {
    return i == 0 ? 0 : i == 1 ? 2 : i == 2 ? 1 : i == 3 ? 0 : i == 4 ? 1 : 0;
  }
};
template <bool BF16>
struct Products<BF16, 2> {  // two-plane splits (BF16x2 or FP16x2): h*l + l*h + h*h
  static constexpr int N = 3;
  static __device__ __forceinline__ constexpr int a(int i) { return i == 0 ? 1 : 0; }
  static __device__ __forceinline__ constexpr int b(int i) { return i == 1 ? 1 : 0; }
};

template <bool BF16, int NPL, int NT>
struct GemmCfg {
  static constexpr int B_SUB = NT / 128 > 0 ? NT / 128 : 1;    // 128-row B sub-tiles per stage
  static constexpr int B_TILE = NT >= 128 ? TILE_BYTES : TILE_BYTES * NT / 128;
  static constexpr int STAGE = NPL * TILE_BYTES + NPL * B_SUB * B_TILE;
  static constexpr int STAGES = (200 * 1024) / STAGE > 4 ? 4 : (200 * 1024) / STAGE;
  static constexpr int SMEM = STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  // two accumulators (leading h*h term, correction terms) x two alternating buffers
  static constexpr int TMEM_COLS = 4 * NT < 32 ? 32 : 4 * NT;
};

// Accumulator promotion. The tensor core adds each K-step's products into its FP32 accumulator with
// truncation (round toward zero), so a long K loop loses about half an ulp of the running sum per step
// and every |C| comes out biased low: with the 92 K-steps of the 729-vector Re sum this measured a
// -3.4e-6 relative bias of |g|^2 in the full pass. The kernels therefore restart the accumulator after
// every 64-wide K chunk (four K-steps; the A-resident kernel after every two) and the epilogue adds each
// chunk's lead + correction accumulators into FP32 registers with round-to-nearest, which leaves ~2e-7
// (numpy emulation of the truncating accumulator; the pass's measured |g|^2 error barely moves at two
// chunks and grows by a third at four). `run` holds the tile row's NT running sums; the two TMEM buffers alternate by
// chunk, so the MMAs of the next chunk overlap the epilogue of this one.
// NT running sums of one tile row: columns [0, NT) of the lead accumulator at tacc and of the correction
// accumulator ACC_STRIDE columns further.
template <int NT, int CB = 16, int ACC_STRIDE = NT>
__device__ __forceinline__ void promote_chunk(uint32_t tacc, float (&run)[NT], bool first) {
#pragma unroll
  for (int c0 = 0; c0 < NT; c0 += CB) {
    uint32_t r[2 * CB];
    if (CB == 16) {
      tmem_ld16_nowait(tacc + c0, r);
      tmem_ld16_nowait(tacc + ACC_STRIDE + c0, r + 16);
    } else {
      tmem_ld8_nowait(tacc + c0, r);
      tmem_ld8_nowait(tacc + ACC_STRIDE + c0, r + 8);
    }
    tmem_wait_ld(r);
#pragma unroll
    for (int j = 0; j < CB; ++j) {
      const float v = __uint_as_float(r[j]) + __uint_as_float(r[CB + j]);
      run[c0 + j] = first ? v : run[c0 + j] + v;
    }
  }
}

// C[row, col0 + j] = run[j] (times cscale when set) for the valid columns of one tile row.
template <int NT>
__device__ __forceinline__ void store_row(const SplitGemmArgs& a, const float (&run)[NT], float* cb, bool row_ok,
                                          int64_t col0) {
  if (!row_ok) return;
  float* p = cb + col0 * a.ldc_n;
#pragma unroll
  for (int j = 0; j < NT; ++j, p += a.ldc_n)
    if (col0 + j < a.n_valid) *p = a.cscale != 0.f ? run[j] * a.cscale : run[j];
}

template <bool BF16, int NPL, int NT>
__global__ void __launch_bounds__(192, 1) split_gemm_kernel(SplitGemmArgs a) {
  using Cfg = GemmCfg<BF16, NPL, NT>;
  using Pr = Products<BF16, NPL>;
  constexpr int STAGES = Cfg::STAGES;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * Cfg::STAGE);
  uint64_t* full = bars;                 // [STAGES]
  uint64_t* empty = bars + STAGES;       // [STAGES]
  uint64_t* tfull = bars + 2 * STAGES;   // [2]
  uint64_t* tempty = tfull + 2;          // [2]
  uint64_t* done = tempty + 2;           // [1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* err = a.err;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 128);
    }
    mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int64_t total = a.m_tiles * a.n_tiles;
  constexpr uint32_t IDESC = idesc_f16(128, NT, BF16);

  if (warp == 0 && lane == 0) {
    // ---------------- producer ----------------
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    uint32_t inflight = 0;      // bit s: stage s has copies that nobody has waited for yet
    uint32_t inflight_ph = 0;   // parity of that stage's in-flight phase
    for (int64_t t = blockIdx.x; t < total && ok; t += gridDim.x) {
      int64_t mt = a.m_fastest ? t % a.m_tiles : t / a.n_tiles;
      int64_t nt = a.m_fastest ? t / a.m_tiles : t % a.n_tiles;
      if (a.grp) {  // the group of column tile nt (binary search), then its A block
        int64_t lo = 0, hi = a.ngrp;
        while (hi - lo > 1) {
          const int64_t mid = (lo + hi) >> 1;
          if (a.grp[mid] <= nt) lo = mid; else hi = mid;
        }
        mt += a.grp_a[lo] * a.m_tiles_per_batch;
      }
      for (int kc = 0; kc < a.KC; ++kc) {
        if (!mbar_wait(&empty[s], ph ^ 1u, err, a.timeout)) {
          ok = false;
          break;
        }
        inflight &= ~(1u << s);
        uint8_t* st = smem + s * Cfg::STAGE;
        mbar_arrive_expect_tx(&full[s], Cfg::STAGE);
        for (int p = 0; p < NPL; ++p)
          bulk_g2s(st + p * TILE_BYTES, a.A + p * a.a_plane_bytes + (mt * a.KC + kc) * (int64_t)TILE_BYTES,
                   TILE_BYTES, &full[s]);
        for (int p = 0; p < NPL; ++p)
          for (int sb = 0; sb < Cfg::B_SUB; ++sb) {
            int64_t bt = nt * Cfg::B_SUB + sb;  // 128-row sub-tile (or partial tile when NT < 128)
            const uint8_t* src = a.B + p * a.b_plane_bytes + (bt * a.KC + kc) * (int64_t)Cfg::B_TILE;
            bulk_g2s(st + NPL * TILE_BYTES + (p * Cfg::B_SUB + sb) * Cfg::B_TILE, src, Cfg::B_TILE, &full[s]);
          }
        inflight |= 1u << s;
        inflight_ph = (inflight_ph & ~(1u << s)) | (ph << s);
        if (++s == STAGES) {
          s = 0;
          ph ^= 1u;
        }
      }
    }
    // drain: wait (bounded) for every stage whose copies may still be landing
    for (int q = 0; q < STAGES; ++q)
      if (inflight & (1u << q)) {
        long long t0 = clock64();
        while (!mbar_try_wait(&full[q], (inflight_ph >> q) & 1u) && clock64() - t0 < a.timeout) {
        }
      }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    int64_t sg = 0;  // K chunks issued so far: chunk sg goes to TMEM buffer sg & 1
    for (int64_t t = blockIdx.x; t < total && ok; t += gridDim.x) {
      for (int kc = 0; kc < a.KC; ++kc, ++sg) {
        const int b = (int)(sg & 1);
        const uint32_t use = (uint32_t)(sg >> 1) & 1u;
        if (!mbar_wait(&tempty[b], use ^ 1u, err, a.timeout)) {
          ok = false;
          break;
        }
        tc_fence_after();
        // accumulator 0 (columns [0, NT)) takes the leading h*h product, accumulator 1 (columns
        // [NT, 2NT)) all correction products: the tensor core aligns addends to the accumulator, so
        // O(2^-16) corrections added onto the O(1) sum would lose their low bits.
        const uint32_t dcol = tmem + b * 2 * NT;
        if (!mbar_wait(&full[s], ph, err, a.timeout)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t st = smem_u32(smem + s * Cfg::STAGE);
#pragma unroll
        for (int sub = 0; sub < 4; ++sub) {
#pragma unroll
          for (int pr = 0; pr < Pr::N; ++pr) {
            const bool lead = Pr::a(pr) == 0 && Pr::b(pr) == 0;
            uint64_t ad = smem_desc_sw128(st + Pr::a(pr) * TILE_BYTES + sub * 32);
            uint64_t bd = smem_desc_sw128(st + NPL * TILE_BYTES + Pr::b(pr) * Cfg::B_SUB * Cfg::B_TILE + sub * 32);
            // the first MMA into each accumulator of the chunk overwrites it
            const bool first = sub == 0 && (lead || pr == 0);
            mma_f16(dcol + (lead ? 0u : (uint32_t)NT), ad, bd, IDESC, first ? 0u : 1u);
          }
        }
        mma_commit(&empty[s]);
        mma_commit(&tfull[b]);  // the chunk's accumulators are ready for promotion
        if (++s == STAGES) {
          s = 0;
          ph ^= 1u;
        }
      }
    }
    // all issued MMAs must retire before TMEM is released
    mma_commit(done);
    long long t0 = clock64();
    while (!mbar_try_wait(done, 0) && clock64() - t0 < a.timeout) {
    }
  } else if (warp >= 2) {
    // ---------------- epilogue ----------------
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
    const int row_in_tile = quarter * 32 + lane;
    int64_t sg = 0;
    bool go = true;
    for (int64_t t = blockIdx.x; t < total && go; t += gridDim.x) {
      float run[NT];
      for (int kc = 0; kc < a.KC; ++kc, ++sg) {
        const int b = (int)(sg & 1);
        const uint32_t use = (uint32_t)(sg >> 1) & 1u;
        bool okw = mbar_wait(&tfull[b], use, err, a.timeout);
        if (!__all_sync(0xffffffffu, okw)) {  // warp-uniform: the TMEM loads below are .sync.aligned
          go = false;
          break;
        }
        tc_fence_after();
        promote_chunk<NT>(tmem + ((uint32_t)(quarter * 32) << 16) + b * 2 * NT, run, kc == 0);
        tc_fence_before();
        mbar_arrive(&tempty[b]);
      }
      if (!go) break;
      int64_t mt = a.m_fastest ? t % a.m_tiles : t / a.n_tiles;
      int64_t nt = a.m_fastest ? t / a.m_tiles : t % a.n_tiles;
      const int64_t batch = mt / a.m_tiles_per_batch;
      const int64_t row = (mt % a.m_tiles_per_batch) * 128 + row_in_tile;
      store_row<NT>(a, run, a.C + batch * a.c_batch_stride + row, row < a.m_valid, nt * NT);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, Cfg::TMEM_COLS);
}

// A-resident form of the same GEMM for short K (KC <= ARES_KC, i.e. K' <= 256): a work unit is one
// 128-row A tile and a run of n_per_unit column tiles. The whole A tile (all K chunks, all planes) is
// copied into shared memory once per unit and every column tile of the run streams only its B chunks,
// so each 128 x 128 output tile costs one B tile of L2 traffic instead of an A and a B tile (the
// kR->kq GEMM of the pass, K' = 256, is bound by that feed). A has its own full / empty barrier pair:
// the MMA thread commits `a_empty` after the unit's last MMA, the producer waits on it before it
// overwrites A. Same products and accumulators as split_gemm_kernel, the promotion after every second K
// chunk (ARES_PROMO), eight epilogue warps (two per TMEM lane quarter, each holding half of a row's running
// sums); no grouped mode.
constexpr int ARES_KC = 4, ARES_STAGES = 2;
// K chunks per accumulator promotion in the A-resident kernel: the accumulators restart every
// 64 * ARES_PROMO K values (the truncation bias grows with that length: about 3e-7 of |g|^2 at 128)
constexpr int ARES_PROMO = 2;
constexpr int ARES_EPI = 2;  // epilogue warps per TMEM lane quarter (each promotes NT / ARES_EPI columns of a row)
constexpr int ARES_THREADS = 64 + 32 * 4 * ARES_EPI;  // producer, MMA issuer, epilogue warps
template <bool BF16, int NPL, int NT>
struct AresCfg {
  using G = GemmCfg<BF16, NPL, NT>;
  static constexpr int A_BYTES = ARES_KC * NPL * TILE_BYTES;
  static constexpr int STAGE = NPL * G::B_SUB * G::B_TILE;  // B chunks of one K step
  static constexpr int SMEM = A_BYTES + ARES_STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int TMEM_COLS = G::TMEM_COLS;
};

template <bool BF16, int NPL, int NT>
// (8 epilogue warps, each promoting half of a tile row's columns: 128 registers; one CTA of this kernel
// leaves room on its SM for one CTA of the FP32 Jacobi, which the pass runs beside it on another stream.
// Sixteen epilogue warps, tried, left no room for it and made the pass slower)
__global__ void __launch_bounds__(ARES_THREADS, 1) split_gemm_ares_kernel(SplitGemmArgs a) {
  using Cfg = AresCfg<BF16, NPL, NT>;
  using G = GemmCfg<BF16, NPL, NT>;
  using Pr = Products<BF16, NPL>;
  constexpr int STAGES = ARES_STAGES;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* bst = smem + Cfg::A_BYTES;  // B stages
  uint64_t* bars = reinterpret_cast<uint64_t*>(bst + STAGES * Cfg::STAGE);
  uint64_t* full = bars;                 // [STAGES]
  uint64_t* empty = bars + STAGES;       // [STAGES]
  uint64_t* tfull = bars + 2 * STAGES;   // [2]
  uint64_t* tempty = tfull + 2;          // [2]
  uint64_t* afull = tempty + 2;          // [1]
  uint64_t* aempty = afull + 1;          // [1]
  uint64_t* done = aempty + 1;           // [1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* err = a.err;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], ARES_THREADS - 64);
    }
    mbar_init(afull, 1);
    mbar_init(aempty, 1);
    mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int64_t npu = a.n_per_unit;
  const int64_t nsplit = (a.n_tiles + npu - 1) / npu;
  const int64_t nunits = a.m_tiles * nsplit;
  constexpr uint32_t IDESC = idesc_f16(128, NT, BF16);

  if (warp == 0 && lane == 0) {
    // ---------------- producer ----------------
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    uint32_t inflight = 0, inflight_ph = 0;  // B stages whose copies nobody has waited for yet
    bool a_inflight = false;
    uint32_t a_ph = 0;
    int64_t uu = 0;
    for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++uu) {
      const int64_t mt = u / nsplit, n0 = (u % nsplit) * npu;
      const int64_t n1 = n0 + npu < a.n_tiles ? n0 + npu : a.n_tiles;
      if (!mbar_wait(aempty, (uint32_t)(uu & 1) ^ 1u, err, a.timeout)) break;
      mbar_arrive_expect_tx(afull, (uint32_t)(a.KC * NPL * TILE_BYTES));
      for (int kc = 0; kc < a.KC; ++kc)
        for (int p = 0; p < NPL; ++p)
          bulk_g2s(smem + (kc * NPL + p) * TILE_BYTES,
                   a.A + p * a.a_plane_bytes + (mt * a.KC + kc) * (int64_t)TILE_BYTES, TILE_BYTES, afull);
      a_inflight = true;
      a_ph = (uint32_t)(uu & 1);
      for (int64_t nt = n0; nt < n1 && ok; ++nt) {
        for (int kc = 0; kc < a.KC; ++kc) {
          if (!mbar_wait(&empty[s], ph ^ 1u, err, a.timeout)) {
            ok = false;
            break;
          }
          inflight &= ~(1u << s);
          uint8_t* st = bst + s * Cfg::STAGE;
          mbar_arrive_expect_tx(&full[s], Cfg::STAGE);
          for (int p = 0; p < NPL; ++p)
            for (int sb = 0; sb < G::B_SUB; ++sb) {
              const int64_t bt = nt * G::B_SUB + sb;
              const uint8_t* src = a.B + p * a.b_plane_bytes + (bt * a.KC + kc) * (int64_t)G::B_TILE;
              bulk_g2s(st + (p * G::B_SUB + sb) * G::B_TILE, src, G::B_TILE, &full[s]);
            }
          inflight |= 1u << s;
          inflight_ph = (inflight_ph & ~(1u << s)) | (ph << s);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
    }
    // drain: wait (bounded) for every copy that may still be landing
    for (int q = 0; q < STAGES; ++q)
      if (inflight & (1u << q)) {
        long long t0 = clock64();
        while (!mbar_try_wait(&full[q], (inflight_ph >> q) & 1u) && clock64() - t0 < a.timeout) {
        }
      }
    if (a_inflight) {
      long long t0 = clock64();
      while (!mbar_try_wait(afull, a_ph) && clock64() - t0 < a.timeout) {
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    int64_t tc = 0, uu = 0;  // output tiles and units of this CTA so far
    const uint32_t abase = smem_u32(smem);
    for (int64_t u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++uu) {
      const int64_t n0 = (u % nsplit) * npu;
      const int64_t n1 = n0 + npu < a.n_tiles ? n0 + npu : a.n_tiles;
      if (!mbar_wait(afull, (uint32_t)(uu & 1), err, a.timeout)) break;
      tc_fence_after();
      for (int64_t nt = n0; nt < n1 && ok; ++nt) {
        for (int kc = 0; kc < a.KC; ++kc) {  // promotion period tc (ARES_PROMO chunks) -> TMEM buffer tc & 1
          const int b = (int)(tc & 1);
          const uint32_t use = (uint32_t)(tc >> 1) & 1u;
          const bool pstart = kc % ARES_PROMO == 0, pend = kc % ARES_PROMO == ARES_PROMO - 1 || kc == a.KC - 1;
          if (pstart && !mbar_wait(&tempty[b], use ^ 1u, err, a.timeout)) {
            ok = false;
            break;
          }
          tc_fence_after();
          // accumulator 0 takes the leading h*h product, accumulator 1 the correction products
          const uint32_t dcol = tmem + b * 2 * NT;
          if (!mbar_wait(&full[s], ph, err, a.timeout)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = smem_u32(bst + s * Cfg::STAGE);
#pragma unroll
          for (int sub = 0; sub < 4; ++sub) {
#pragma unroll
            for (int pr = 0; pr < Pr::N; ++pr) {
              const bool lead = Pr::a(pr) == 0 && Pr::b(pr) == 0;
              uint64_t ad = smem_desc_sw128(abase + (kc * NPL + Pr::a(pr)) * TILE_BYTES + sub * 32);
              uint64_t bd = smem_desc_sw128(st + Pr::b(pr) * G::B_SUB * G::B_TILE + sub * 32);
              const bool first = pstart && sub == 0 && (lead || pr == 0);
              mma_f16(dcol + (lead ? 0u : (uint32_t)NT), ad, bd, IDESC, first ? 0u : 1u);
            }
          }
          mma_commit(&empty[s]);
          if (pend) {
            mma_commit(&tfull[b]);
            ++tc;
          }
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
      mma_commit(aempty);  // the A tile may be overwritten once this unit's MMAs have completed
    }
    // all issued MMAs must retire before TMEM is released
    mma_commit(done);
    long long t0 = clock64();
    while (!mbar_try_wait(done, 0) && clock64() - t0 < a.timeout) {
    }
  } else if (warp >= 2) {
    // ---------------- epilogue ----------------
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
    const int row_in_tile = quarter * 32 + lane;
    const int half = (warp - 2) >> 2;  // ARES_EPI warps per lane quarter: columns [half NH, half NH + NH)
    constexpr int NH = NT / ARES_EPI;
    int64_t tc = 0;
    bool go = true;
    for (int64_t u = blockIdx.x; u < nunits && go; u += gridDim.x) {
      const int64_t mt = u / nsplit, n0 = (u % nsplit) * npu;
      const int64_t n1 = n0 + npu < a.n_tiles ? n0 + npu : a.n_tiles;
      const int64_t batch = mt / a.m_tiles_per_batch;
      const int64_t row = (mt % a.m_tiles_per_batch) * 128 + row_in_tile;
      float* cb = a.C + batch * a.c_batch_stride + row;
      const bool row_ok = row < a.m_valid;
      for (int64_t nt = n0; nt < n1 && go; ++nt) {
        float run[NH];
        for (int kc = 0; kc < a.KC; kc += ARES_PROMO, ++tc) {
          const int b = (int)(tc & 1);
          const uint32_t use = (uint32_t)(tc >> 1) & 1u;
          bool okw = mbar_wait(&tfull[b], use, err, a.timeout);
          if (!__all_sync(0xffffffffu, okw)) {  // warp-uniform: the TMEM loads below are .sync.aligned
            go = false;
            break;
          }
          tc_fence_after();
          promote_chunk<NH, 16, NT>(tmem + ((uint32_t)(quarter * 32) << 16) + b * 2 * NT + half * NH, run, kc == 0);
          tc_fence_before();
          mbar_arrive(&tempty[b]);
        }
        if (go) store_row<NH>(a, run, cb, row_ok, nt * NT + half * NH);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, Cfg::TMEM_COLS);
}

// w = 1 / (2 omega) in FP32 (the |g|^2 weight of the rotation kernel), per q and mode, once per pass.
__global__ void inv2w_kernel(const double* __restrict__ omega, float* __restrict__ w, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    w[i] = (float)(0.5 / omega[i]);
}

// ---------------------------------------------------------------------------------------------
// Host-side helpers.
struct Planes {
  uint8_t* p = nullptr;
  int64_t rows_pad = 0, KC = 0, plane_bytes = 0;
  int npl = 0;
};

static int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

static int64_t plane_bytes_for(int64_t rows_pad, int64_t KC) { return rows_pad / 128 * KC * TILE_BYTES; }

static unsigned grid_for(epb_ctx* ctx, int64_t total) {
  int64_t g = cdiv(total, 256);
  int64_t cap = (int64_t)ctx->sm_count * 16;
  return (unsigned)(g < cap ? (g < 1 ? 1 : g) : cap);
}

template <bool BF16, int NPL, int NT>
static int launch_split_gemm(epb_ctx* ctx, SplitGemmArgs& a) {
  using Cfg = GemmCfg<BF16, NPL, NT>;
  static_assert(Cfg::STAGES >= 2, "split GEMM needs at least two stages");
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(split_gemm_kernel<BF16, NPL, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  Cfg::SMEM));
    attr = true;
  }
  int64_t total = a.m_tiles * a.n_tiles;
  if (total == 0) return EPB_OK;
  unsigned grid = (unsigned)(total < ctx->sm_count ? total : ctx->sm_count);
  split_gemm_kernel<BF16, NPL, NT><<<grid, 192, Cfg::SMEM, ctx->stream>>>(a);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

template <bool BF16, int NPL, int NT>
static int launch_split_gemm_ares(epb_ctx* ctx, SplitGemmArgs& a) {
  using Cfg = AresCfg<BF16, NPL, NT>;
  static_assert(Cfg::SMEM <= 227 * 1024, "A-resident GEMM: shared memory over the per-CTA limit");
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(split_gemm_ares_kernel<BF16, NPL, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  Cfg::SMEM));
    attr = true;
  }
  EPB_CHECK_ARG(a.KC <= ARES_KC && !a.grp && a.n_per_unit >= 1, "A-resident GEMM: K' over %d or grouped",
                64 * ARES_KC);
  const int64_t units = a.m_tiles * cdiv(a.n_tiles, a.n_per_unit);
  if (units == 0) return EPB_OK;
  const unsigned grid = (unsigned)(units < ctx->sm_count ? units : ctx->sm_count);
  split_gemm_ares_kernel<BF16, NPL, NT><<<grid, ARES_THREADS, Cfg::SMEM, ctx->stream>>>(a);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Precision configuration of the mixed path (split BF16x3, six products).
constexpr bool MX_BF16 = true;
constexpr int MX_NPL = 3;
constexpr int MX_NT = 128;

int split_gemm(epb_ctx* ctx, int prof_id, const Planes& A, const Planes& B, int64_t m_tiles_per_batch,
               int64_t batches, int64_t m_valid, int64_t n_valid, bool m_fastest, float* C,
               int64_t c_batch_stride, int64_t ldc_n) {
  int* err = ctx->dstat + 2;
  SplitGemmArgs a{};
  a.A = A.p;
  a.B = B.p;
  a.a_plane_bytes = A.plane_bytes;
  a.b_plane_bytes = B.plane_bytes;
  a.KC = (int)A.KC;
  a.m_tiles = m_tiles_per_batch * batches;
  a.n_tiles = cdiv(n_valid, MX_NT);
  a.m_fastest = m_fastest ? 1 : 0;
  a.m_tiles_per_batch = m_tiles_per_batch;
  a.m_valid = m_valid;
  a.n_valid = n_valid;
  a.C = C;
  a.c_batch_stride = c_batch_stride;
  a.ldc_n = ldc_n;
  a.err = err;
  a.timeout = 4000000000LL;  // ~2 s at 2 GHz
  EPB_CHECK_ARG(A.KC == B.KC, "split GEMM: K chunk mismatch");
  EPB_CHECK_ARG(B.rows_pad >= a.n_tiles * MX_NT, "split GEMM: B planes too small");
  prof_begin(ctx, prof_id);
  int st = launch_split_gemm<MX_BF16, MX_NPL, MX_NT>(ctx, a);
  prof_end(ctx);
  return st;
}

// The FP16x2 configuration (two FP16 planes per operand, three products: h*h, h*l, l*h, about 22 bits),
// for operands pre-scaled by a power of two into FP16's range; cscale undoes the scale on C.
int split_gemm_h(epb_ctx* ctx, int prof_id, const Planes& A, const Planes& B, int64_t m_tiles_per_batch,
                 int64_t batches, int64_t m_valid, int64_t n_valid, bool m_fastest, float* C, int64_t c_batch_stride,
                 int64_t ldc_n, float cscale, int form /* 1 A-resident when K' <= 256, 0 streamed operands */) {
  SplitGemmArgs a{};
  a.A = A.p;
  a.B = B.p;
  a.a_plane_bytes = A.plane_bytes;
  a.b_plane_bytes = B.plane_bytes;
  a.KC = (int)A.KC;
  a.m_tiles = m_tiles_per_batch * batches;
  a.n_tiles = cdiv(n_valid, MX_NT);
  a.m_fastest = m_fastest ? 1 : 0;
  a.m_tiles_per_batch = m_tiles_per_batch;
  a.m_valid = m_valid;
  a.n_valid = n_valid;
  a.C = C;
  a.c_batch_stride = c_batch_stride;
  a.ldc_n = ldc_n;
  a.err = ctx->dstat + 2;
  a.timeout = 4000000000LL;
  a.cscale = cscale;
  EPB_CHECK_ARG(A.KC == B.KC && A.npl == 2 && B.npl == 2, "FP16x2 GEMM: operand planes mismatch");
  EPB_CHECK_ARG(B.rows_pad >= a.n_tiles * MX_NT, "FP16x2 GEMM: B planes too small");
  prof_begin(ctx, prof_id);
  int st;
  if (a.KC <= ARES_KC && form == 1) {
    // A-resident: a unit is one A tile and n_per_unit column tiles; enough units for ~16 per CTA, at
    // least 8 column tiles per unit (the A copy is then under 1/8 of the unit's traffic)
    const int64_t want = cdiv(16 * (int64_t)ctx->sm_count, std::max<int64_t>(a.m_tiles, 1));
    const int64_t nsplit = std::max<int64_t>(1, std::min<int64_t>(want, a.n_tiles / 8));
    a.n_per_unit = cdiv(a.n_tiles, nsplit);
    st = launch_split_gemm_ares<false, 2, MX_NT>(ctx, a);
  } else {
    st = launch_split_gemm<false, 2, MX_NT>(ctx, a);
  }
  prof_end(ctx);
  return st;
}

// Check the device error flag raised by bounded waits (one sync).
int split_gemm_check(epb_ctx* ctx) {
  int* h = (int*)ctx->pinned;
  EPB_CUDA(cudaMemcpyAsync(h, ctx->dstat + 2, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(ctx->dstat + 2, 0, sizeof(int), ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*h) {
    set_error("tensor-core GEMM: a bounded wait timed out (kernel wound down)");
    return EPB_ERR_TIMEOUT;
  }
  return EPB_OK;
}

int pack_a_complex(epb_ctx* ctx, const double2* a, int64_t ld, int64_t M, int64_t K, Planes& out, uint8_t* mem) {
  out.rows_pad = round_up(2 * M, 128);
  out.KC = kchunks(K);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  int64_t total = out.rows_pad * out.KC * 8;
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_a_complex_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
      a, ld, M, K, out.rows_pad, out.KC, out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int pack_a_herm(epb_ctx* ctx, const double2* op, int nw, int64_t K, Planes& out, uint8_t* mem) {
  out.rows_pad = round_up((int64_t)nw * nw, 128);
  out.KC = kchunks(K);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  int64_t total = out.rows_pad * out.KC * 8;
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_a_herm_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(op, nw, K, out.rows_pad, out.KC,
                                                                                    out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// A operand of H(k + q) for nk k points (batches of rows_pad_k rows each).
int pack_a_herm_mod(epb_ctx* ctx, const double2* op, const epb_rset* rs, int nw, const double* xk, int64_t nk,
                    int64_t rows_pad_k, Planes& out, uint8_t* mem) {
  out.rows_pad = nk * rows_pad_k;
  out.KC = kchunks(rs->nr);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  const int64_t total = out.rows_pad * out.KC * 8;
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_a_herm_mod_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
      op, rs->dev, nw, rs->nr, xk, nk, rows_pad_k, out.KC, out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int pack_b_phase(epb_ctx* ctx, const epb_rset* rs, const double* xa, const double* xb, int64_t nb, int64_t N,
                 Planes& out, uint8_t* mem, const int64_t* pidx = nullptr, int64_t pair0 = 0) {
  out.rows_pad = round_up(N, MX_NT);
  out.KC = kchunks(rs->nr);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  int64_t total = out.rows_pad * (sin_offset(rs->nr) / 8);
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_b_phase_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
      rs->dev, rs->nr, xa, xb, nb, pidx, pair0, N, out.rows_pad, out.KC, out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Phase planes in the FP16x2 configuration (|phase| <= 1: no scaling needed).
int pack_b_phase_h(epb_ctx* ctx, const epb_rset* rs, const double* xa, const double* xb, int64_t nb, int64_t N,
                   Planes& out, uint8_t* mem) {
  out.rows_pad = round_up(N, MX_NT);
  out.KC = kchunks(rs->nr);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = 2;
  out.p = mem;
  int64_t total = out.rows_pad * (sin_offset(rs->nr) / 8);
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_b_phase_kernel<false, 2><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
      rs->dev, rs->nr, xa, xb, nb, nullptr, 0, N, out.rows_pad, out.KC, out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int64_t planes_bytes(int64_t rows, int64_t K) {
  return MX_NPL * plane_bytes_for(round_up(rows, 128), kchunks(K));
}

__global__ void c64_to_c128_kernel(const float2* __restrict__ in, double2* __restrict__ out, int64_t M,
                                   int64_t N, int64_t ldin, int64_t ldout) {
  int64_t total = M * N;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = idx % M, j = idx / M;
    float2 v = in[i + j * ldin];
    out[i + j * ldout] = make_double2(v.x, v.y);
  }
}

// ---- packed operands that live across calls (outer-q loop) ----------------------------------
int64_t oq_a_bytes(int64_t M, int64_t K) { return planes_bytes(2 * M, K); }
int64_t oq_b_bytes(int64_t N, int64_t K) { return MX_NPL * plane_bytes_for(round_up(N, MX_NT), kchunks(K)); }
int oq_pack_a(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, int64_t K, uint8_t* mem) {
  Planes A;
  return pack_a_complex(ctx, op, ld, M, K, A, mem);
}
int oq_pack_b(epb_ctx* ctx, const epb_rset* rs, const double* x, int64_t N, uint8_t* mem) {
  Planes B;
  return pack_b_phase(ctx, rs, x, nullptr, 1, N, B, mem);
}
// C (complex64 columns of M, column stride ldc complex) = A (op packed by oq_pack_a, M x K) times the phase
// columns [n0, n0 + nn) of the N points packed by oq_pack_b; n0 a multiple of 128. No host sync: a bounded
// wait that timed out is reported by the next split_gemm_check.
int oq_gemm(epb_ctx* ctx, int prof_id, const uint8_t* a_mem, int64_t M, int64_t K, const uint8_t* b_mem, int64_t N,
            int64_t n0, int64_t nn, float2* C, int64_t ldc) {
  EPB_CHECK_ARG(n0 % MX_NT == 0 && n0 + nn <= N, "oq_gemm: bad column range");
  Planes A, B;
  A.rows_pad = round_up(2 * M, 128);
  A.KC = kchunks(K);
  A.plane_bytes = plane_bytes_for(A.rows_pad, A.KC);
  A.npl = MX_NPL;
  A.p = const_cast<uint8_t*>(a_mem);
  B.rows_pad = round_up(N, MX_NT);
  B.KC = A.KC;
  B.plane_bytes = plane_bytes_for(B.rows_pad, B.KC);
  B.npl = MX_NPL;
  B.p = const_cast<uint8_t*>(b_mem) + (n0 / 128) * B.KC * (int64_t)TILE_BYTES;
  B.rows_pad -= n0;
  return split_gemm(ctx, prof_id, A, B, A.rows_pad / 128, 1, 2 * M, nn, true, (float*)C, 0, 2 * ldc);
}

// epb_fourier(..., EPB_PREC_MIXED): pack op_r and the phases, split GEMM, widen to c128.
int fourier_mixed(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                  const double* xk, int64_t N, double2* out, int64_t ldo) {
  if (M == 0 || N == 0) return EPB_OK;
  const int64_t K = rs->nr;
  const int64_t a_bytes = planes_bytes(2 * M, K);
  const int64_t b_bytes = MX_NPL * plane_bytes_for(round_up(N, MX_NT), kchunks(K));
  const int64_t c_bytes = 8 * M * N;
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_SPLIT_A, a_bytes + b_bytes + c_bytes + 1024, &ws));
  uint8_t* base = (uint8_t*)(((uintptr_t)ws + 1023) & ~uintptr_t(1023));
  Planes A, B;
  EPB_TRY(pack_a_complex(ctx, op, ld, M, K, A, base));
  EPB_TRY(pack_b_phase(ctx, rs, xk, nullptr, 1, N, B, base + a_bytes));
  float* C = (float*)(base + a_bytes + b_bytes);
  // C column j = complex64 column of length M (2M floats)
  EPB_TRY(split_gemm(ctx, EPB_PROF_UMMA_H, A, B, A.rows_pad / 128, 1, 2 * M, N, true, C, 0, 2 * M));
  c64_to_c128_kernel<<<grid_for(ctx, M * N), 256, 0, ctx->stream>>>((const float2*)C, out, M, N, M, ldo);
  EPB_LAUNCH_CHECK();
  return split_gemm_check(ctx);
}

// =============================================================================================
// Band energies on the tensor cores: the Hermitian-packed H(R) planes of a model, and H(x) for a
// list of points as packed FP32 matrices (n^2 floats per point: Re of i <= j, then Im of i < j).

struct BandPlanes {
  uint8_t* mem = nullptr;
  Planes H;
};

int band_planes_prepare(epb_ctx* ctx, const double2* ham, int nw, const epb_rset* rs, void** out) {
  const int64_t hb = MX_NPL * plane_bytes_for(round_up((int64_t)nw * nw, 128), kchunks(rs->nr));
  BandPlanes* bp = new BandPlanes();
  if (cudaMalloc(&bp->mem, hb + 1024) != cudaSuccess) {
    cudaGetLastError();
    delete bp;
    set_error("band planes: allocation of %lld bytes failed", (long long)hb);
    return EPB_ERR_OOM;
  }
  uint8_t* base = (uint8_t*)(((uintptr_t)bp->mem + 1023) & ~uintptr_t(1023));
  int st = pack_a_herm(ctx, ham, nw, rs->nr, bp->H, base);
  if (st != EPB_OK) {
    cudaFree(bp->mem);
    delete bp;
    return st;
  }
  *out = bp;
  return EPB_OK;
}

void band_planes_free(void* p) {
  BandPlanes* bp = (BandPlanes*)p;
  if (!bp) return;
  cudaFree(bp->mem);
  delete bp;
}

// Largest point count per call of band_hk_packed (bounds its phase-plane workspace).
int64_t band_hk_chunk(const epb_rset* rs) {
  const int64_t per = MX_NPL * kchunks(rs->nr) * TILE_BYTES / 128;  // plane bytes per point
  int64_t c = ((int64_t)768 << 20) / per;
  c = c / MX_NT * MX_NT;
  return c < MX_NT ? MX_NT : c;
}

// Hp[:, j] = packed H(x_j), points as in pack_b_phase_kernel; N <= band_hk_chunk(rs).
int band_hk_packed(epb_ctx* ctx, const void* planes, const epb_rset* rs, int nw, const double* xa, const double* xb,
                   int64_t nb, const int64_t* pidx, int64_t pair0, int64_t N, float* Hp) {
  if (N == 0) return EPB_OK;
  const BandPlanes* bp = (const BandPlanes*)planes;
  const int64_t bbytes = MX_NPL * plane_bytes_for(round_up(N, MX_NT), kchunks(rs->nr));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PAIR3, bbytes + 1024, &ws));
  uint8_t* base = (uint8_t*)(((uintptr_t)ws + 1023) & ~uintptr_t(1023));
  Planes B;
  EPB_TRY(pack_b_phase(ctx, rs, xa, xb, nb, N, B, base, pidx, pair0));
  const int64_t n2 = (int64_t)nw * nw;
  return split_gemm(ctx, EPB_PROF_UMMA_H, bp->H, B, bp->H.rows_pad / 128, 1, n2, N, true, Hp, 0, n2);
}

// =============================================================================================
// Mixed-precision e-ph pass.

struct MixedModel {
  uint8_t* mem = nullptr;
  Planes H;   // H(R), Hermitian-packed rows (nw^2), K = nr_el
  Planes EP;  // g(Re, Rp), complex rows (2 * nw^2 nm nr_ep), K = nr_el
  double ep_absmax = 0.0;  // max |Re|, |Im| of g(Re, Rp): scales the FP16x2 kR->kq operand
};

// max(|Re|, |Im|) over n complex values into *out (non-negative doubles order like their bit patterns).
__global__ void absmax_c128_kernel(const double2* __restrict__ v, int64_t n, unsigned long long* __restrict__ out) {
  double mx = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    mx = fmax(mx, fmax(fabs(v[i].x), fabs(v[i].y)));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

int mixed_model_prepare(epb_ctx* ctx, epb_model* m) {
  const int64_t nw = m->nw, nd_ep = m->nw * m->nw * m->nm * m->nr_ep;
  const int64_t hb = MX_NPL * plane_bytes_for(round_up(nw * nw, 128), kchunks(m->nr_el));
  const int64_t eb = MX_NPL * plane_bytes_for(round_up(2 * nd_ep, 128), kchunks(m->nr_el));
  MixedModel* mm = new MixedModel();
  cudaError_t e = cudaMalloc(&mm->mem, hb + eb + 1024);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete mm;
    set_error("mixed model planes: allocation of %lld bytes failed", (long long)(hb + eb));
    return EPB_ERR_OOM;
  }
  uint8_t* base = (uint8_t*)(((uintptr_t)mm->mem + 1023) & ~uintptr_t(1023));
  int st = pack_a_herm(ctx, m->ham, (int)nw, m->nr_el, mm->H, base);
  if (st == EPB_OK) st = pack_a_complex(ctx, m->epmat, nd_ep, nd_ep, m->nr_el, mm->EP, base + hb);
  if (st != EPB_OK) {
    cudaFree(mm->mem);
    delete mm;
    return st;
  }
  m->mixed = mm;  // owned by the model from here on (freed with it on any later failure)
  // max |g(Re, Rp)| (one sync at model creation)
  unsigned long long* d = reinterpret_cast<unsigned long long*>(ctx->dstat + 16);  // status words 16-17
  EPB_CUDA(cudaMemsetAsync(d, 0, 8, ctx->stream));
  absmax_c128_kernel<<<grid_for(ctx, nd_ep * m->nr_el), 256, 0, ctx->stream>>>(m->epmat, nd_ep * m->nr_el, d);
  EPB_LAUNCH_CHECK();
  unsigned long long h = 0;
  EPB_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(&mm->ep_absmax, &h, 8);
  return EPB_OK;
}

void mixed_model_free(epb_model* m) {
  if (!m || !m->mixed) return;
  MixedModel* mm = (MixedModel*)m->mixed;
  if (mm->mem) cudaFree(mm->mem);
  delete mm;
  m->mixed = nullptr;
}

// g(k, Rp) rotated on the k leg from the tensor-core Fourier output (complex64, "el" row order, one
// column of nd = nw^2 nm nr_ep per k): out[iw, n, mp, k] = sum_jw g[iw, jw, mp, k] uk[jw, n, k], FP64.
__global__ void rr_rotate_c64_kernel(const float2* __restrict__ g, const double2* __restrict__ uk,
                                     double2* __restrict__ out, int nw, int nband, int nm, int nr_ep, int64_t kc) {
  const int64_t M = (int64_t)nm * nr_ep;
  const int64_t total = (int64_t)nw * nband * M * kc;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int iw = (int)(idx % nw);
    int64_t r = idx / nw;
    const int n = (int)(r % nband);
    r /= nband;
    const int64_t mp = r % M, k = r / M;
    const float2* gb = g + ((k * M + mp) * nw) * nw;
    const double2* ub = uk + (k * nband + n) * nw;
    double2 acc = make_double2(0.0, 0.0);
    for (int jw = 0; jw < nw; ++jw) {
      const float2 v = gb[iw + jw * nw];
      cfma(acc, make_double2(v.x, v.y), ub[jw]);
    }
    out[idx] = acc;
  }
}

// get_eph_RR_to_kR on the tensor cores: g(k, Rp) = sum_Re e^{2 pi i k.Re} g(Re, Rp) as a split-BF16x3 GEMM
// against the model's operand planes (epb_model_create with the mixed flag), then the k-leg rotation
// by uk (nw x nband x nk, FP64) into out (nw nband nm nr_ep x nk, c128). Stream-ordered; the GEMM's
// timeout flag is left for the caller's split_gemm_check.
int mixed_rr_to_kR(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double2* uk, int nband,
                   double2* out) {
  MixedModel* mm = (MixedModel*)m->mixed;
  EPB_CHECK_ARG(mm, "mixed RR->kR: the model was created without the mixed operand planes");
  if (nk == 0) return EPB_OK;
  const int64_t nw = m->nw, nm = m->nm, nd_ep = nw * nw * nm * m->nr_ep;
  const int64_t KC_el = kchunks(m->nr_el);
  int64_t kc = ((int64_t)768 << 20) / (8 * nd_ep);
  kc = std::max<int64_t>(1, std::min<int64_t>(kc, 256));
  kc = std::min(kc, nk);
  const int64_t bbytes = MX_NPL * plane_bytes_for(round_up(kc, MX_NT), KC_el);
  const int64_t cbytes = 8 * nd_ep * kc;
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS4, bbytes + cbytes + 2048, &ws));
  uint8_t* base = (uint8_t*)(((uintptr_t)ws + 1023) & ~uintptr_t(1023));
  float* C0 = (float*)(base + ((bbytes + 1023) & ~int64_t(1023)));
  const int64_t outk = nw * nband * nm * m->nr_ep;
  for (int64_t k0 = 0; k0 < nk; k0 += kc) {
    const int64_t kn = std::min(kc, nk - k0);
    Planes Bk;
    EPB_TRY(pack_b_phase(ctx, m->rs_el, xk + 3 * k0, nullptr, 1, kn, Bk, base));
    EPB_TRY(split_gemm(ctx, EPB_PROF_UMMA_RR, mm->EP, Bk, mm->EP.rows_pad / 128, 1, 2 * nd_ep, kn, false, C0, 0,
                       2 * nd_ep));
    const int64_t total = nw * nband * nm * m->nr_ep * kn;
    prof_begin(ctx, EPB_PROF_RR_ROT);
    rr_rotate_c64_kernel<<<grid_for(ctx, total), 256, 0, ctx->stream>>>((const float2*)C0, uk + k0 * nw * nband,
                                                                        out + k0 * outk, (int)nw, nband, (int)nm,
                                                                        (int)m->nr_ep, kn);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

// RR->kR rotation on the k leg fused with the packing of the kR->kq operand:
//   G_k[iw, n, nu, p] = sum_jw g_k[iw, jw, nu, p] uk[jw, n]      (src/wannier_to_bloch_batched.jl:190-203)
// written straight into the split planes of A2 for the batched kR->kq GEMM: batch k, rows
// 2r / 2r+1 (r = iw + nw (n + nw nu)), K' = [cos p | sin p] with koff = round_up(nr_ep, 8).
template <bool BF16, int NPL>
__global__ void rr_rotate_pack_kernel(const float2* __restrict__ gk, const double2* __restrict__ uk, int nw,
                                      int nband, int nm, int nr_ep, int64_t nk, int64_t rows_pad_k, int64_t KC,
                                      uint8_t* __restrict__ planes, int64_t plane_bytes, double scale = 1.0,
                                      unsigned* __restrict__ absmax = nullptr) {
  // FP32 products and sums (g is FP32; the planes hold at most 24 bits), u rounded to FP32 once per row
  const int nd = nw * nband * nm;  // complex rows r per k
  const int koff = (int)sin_offset(nr_ep);
  const int npc = koff / 8;        // 8-wide p chunks
  const int64_t total = nk * nd * npc;
  const int64_t ndata = (int64_t)nw * nw * nm * nr_ep;  // complex length of g_k
  const float sc = (float)scale;
  const bool idx32 = total <= 0x7fffffff;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int r, pc;
    int64_t k;
    if (idx32) {
      const uint32_t i = (uint32_t)idx, rest = i / (uint32_t)nd;
      r = (int)(i - rest * (uint32_t)nd);
      k = rest / (uint32_t)npc;
      pc = (int)(rest - (uint32_t)k * (uint32_t)npc);
    } else {
      const int64_t rest = idx / nd;
      r = (int)(idx - rest * nd);
      k = rest / npc;
      pc = (int)(rest - k * npc);
    }
    const int iw = r % nw, n = (r / nw) % nband, nu = r / (nw * nband);
    const float2* g = gk + k * ndata + iw + (int64_t)nw * nw * nu;
    const double2* u = uk + (k * nband + n) * nw;
    float2 acc[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] = make_float2(0.f, 0.f);
    for (int jw = 0; jw < nw; ++jw) {
      const double2 ud = u[jw];
      const float2 uf = make_float2((float)ud.x, (float)ud.y);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int p = pc * 8 + e;
        if (p < nr_ep) cfma(acc[e], g[(int64_t)nw * jw + (int64_t)nw * nw * nm * p], uf);
      }
    }
    float re[8], im[8], t[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      re[e] = acc[e].x * sc;
      im[e] = acc[e].y * sc;
      t[e] = -im[e];
    }
    if (absmax) {  // max |Re G|, |Im G| of the written (scaled) values: bounds the kR->kq output
      float mx = 0.f;
#pragma unroll
      for (int e = 0; e < 8; ++e) mx = fmaxf(mx, fmaxf(fabsf(re[e]), fabsf(im[e])));
      if (__activemask() == 0xffffffffu) {  // whole warp: one atomic; a partial last warp: one per thread
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) atomicMax(absmax, __float_as_uint(mx));
      } else {
        atomicMax(absmax, __float_as_uint(mx));
      }
    }
    const int64_t row0 = k * rows_pad_k + 2 * r;
    // real row: [Re G | -Im G];  imaginary row: [Im G | Re G]
    store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(row0, pc * 8, KC), re);
    store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(row0, koff + pc * 8, KC), t);
    store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(row0 + 1, pc * 8, KC), im);
    store_split8_f32<BF16, NPL>(planes, plane_bytes, tiled_offset(row0 + 1, koff + pc * 8, KC), re);
  }
}

__global__ void c128_to_c64_kernel(const double2* __restrict__ in, float2* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

// The same conversion, also raising *absmax (float bits) to the largest |Re|, |Im| converted.
__global__ void c128_to_c64_absmax_kernel(const double2* __restrict__ in, float2* __restrict__ out, int64_t n,
                                          unsigned* __restrict__ absmax) {
  float mx = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 v = make_float2((float)in[i].x, (float)in[i].y);
    out[i] = v;
    mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(absmax, __float_as_uint(mx));
}

int rot_mma_launch(epb_ctx* ctx, const float* g, int64_t g_stride, const float2* ukq, const float2* uph,
                   const float* inv2w, const unsigned* gmax, const unsigned* phmax, float gscale_inv, int nr_ep,
                   int64_t nkb, int64_t nq, double* g2sum, double* partial, double* sample, int64_t stride,
                   int64_t nsamp);
int64_t rot_mma_partial_doubles(epb_ctx* ctx, int64_t nkb);

// ---- windowed kR->kq of the Boltzmann consumer on the tensor cores --------------------------------
// A2 planes of G_k = g(k, Rp) u_k (nband columns of u_k) for nk points, one block of bte_rows_pad(nw, nband,
// nm) rows per k, through the model's g(Re, Rp) planes (mixed flag of epb_model_create).
int64_t bte_rows_pad(int64_t nw, int64_t nband, int64_t nm) { return round_up(2 * nw * nband * nm, 128); }
int64_t bte_a2_bytes(epb_model* m, int64_t nk, int64_t nband) {
  return MX_NPL * plane_bytes_for(bte_rows_pad(m->nw, nband, m->nm) * nk, kchunks(m->nr_ep));
}
int64_t bte_b_bytes(epb_model* m, int64_t ncols) { return MX_NPL * plane_bytes_for(round_up(ncols, MX_NT), kchunks(m->nr_ep)); }

int bte_pack_kR(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double2* uk, int nband, uint8_t* a2) {
  MixedModel* mm = (MixedModel*)m->mixed;
  EPB_CHECK_ARG(mm, "windowed kR->kq: the model was created without the mixed operand planes");
  if (nk == 0) return EPB_OK;
  const int64_t nw = m->nw, nm = m->nm, nd_ep = nw * nw * nm * m->nr_ep;
  const int64_t KC_el = kchunks(m->nr_el), KC_ep = kchunks(m->nr_ep);
  const int64_t rpk = bte_rows_pad(nw, nband, nm);
  const int64_t a2_plane = plane_bytes_for(rpk * nk, KC_ep);
  if (rpk != 2 * nw * nband * nm) EPB_CUDA(cudaMemsetAsync(a2, 0, MX_NPL * a2_plane, ctx->stream));
  int64_t kc = ((int64_t)768 << 20) / (8 * nd_ep);
  kc = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(kc, 256), nk));
  const int64_t bbytes = MX_NPL * plane_bytes_for(round_up(kc, MX_NT), KC_el);
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS4, bbytes + 8 * nd_ep * kc + 2048, &ws));
  uint8_t* base = (uint8_t*)(((uintptr_t)ws + 1023) & ~uintptr_t(1023));
  float* C0 = (float*)(base + ((bbytes + 1023) & ~int64_t(1023)));
  for (int64_t k0 = 0; k0 < nk; k0 += kc) {
    const int64_t kn = std::min(kc, nk - k0);
    Planes Bk;
    EPB_TRY(pack_b_phase(ctx, m->rs_el, xk + 3 * k0, nullptr, 1, kn, Bk, base));
    EPB_TRY(split_gemm(ctx, EPB_PROF_UMMA_RR, mm->EP, Bk, mm->EP.rows_pad / 128, 1, 2 * nd_ep, kn, false, C0, 0,
                       2 * nd_ep));
    const int64_t total = kn * nw * nband * nm * (sin_offset(m->nr_ep) / 8);
    prof_begin(ctx, EPB_PROF_RR_ROT);
    rr_rotate_pack_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
        (const float2*)C0, uk + k0 * nw * nband, (int)nw, nband, (int)nm, (int)m->nr_ep, kn, rpk, KC_ep,
        a2 + k0 * rpk / 128 * KC_ep * TILE_BYTES, a2_plane);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

// C (complex64 columns of nw nband nm rows, column stride ldc complex) for ncols phase columns x (3 x ncols;
// ncols a multiple of 128): column tile t of group g multiplies the A2 block grp_a[g] (see bte_pack_kR),
// tiles [grp[g], grp[g + 1]). Stream-ordered; the timeout flag is left for split_gemm_check.
int bte_kq_grouped(epb_ctx* ctx, epb_model* m, const uint8_t* a2, int64_t nk_a2, int nband, const double* x,
                   int64_t ncols, const int64_t* grp, const int64_t* grp_a, int64_t ngrp, uint8_t* bmem, float2* C,
                   int64_t ldc) {
  EPB_CHECK_ARG(ncols % MX_NT == 0, "windowed kR->kq: column count must be a multiple of 128");
  if (ncols == 0 || ngrp == 0) return EPB_OK;
  const int64_t KC_ep = kchunks(m->nr_ep), rpk = bte_rows_pad(m->nw, nband, m->nm);
  Planes A, B;
  A.rows_pad = rpk * nk_a2;
  A.KC = KC_ep;
  A.plane_bytes = plane_bytes_for(A.rows_pad, KC_ep);
  A.npl = MX_NPL;
  A.p = const_cast<uint8_t*>(a2);
  EPB_TRY(pack_b_phase(ctx, m->rs_ep, x, nullptr, 1, ncols, B, bmem));
  int* err = ctx->dstat + 2;
  SplitGemmArgs a{};
  a.A = A.p;
  a.B = B.p;
  a.a_plane_bytes = A.plane_bytes;
  a.b_plane_bytes = B.plane_bytes;
  a.KC = (int)KC_ep;
  a.m_tiles = rpk / 128;
  a.n_tiles = ncols / MX_NT;
  a.m_fastest = 1;
  a.m_tiles_per_batch = rpk / 128;
  a.m_valid = 2 * m->nw * nband * m->nm;
  a.n_valid = ncols;
  a.C = (float*)C;
  a.c_batch_stride = 0;
  a.ldc_n = 2 * ldc;
  a.err = err;
  a.timeout = 4000000000LL;
  a.grp = grp;
  a.grp_a = grp_a;
  a.ngrp = ngrp;
  prof_begin(ctx, EPB_PROF_UMMA_KQ);
  int st = launch_split_gemm<MX_BF16, MX_NPL, MX_NT>(ctx, a);
  prof_end(ctx);
  return st;
}

// Rotation + |g|^2 fold + in-place reduction, FP32, one (k, q) block at a time per CTA:
//   T[m, n, jm] = sum_iw conj(ukq[iw, m]) g[iw, n, jm]  (thread per column (n, jm), g column in registers)
//   ep[m, n, nu] = sum_jm T[m, n, jm] uph[jm, nu]        (thread per (m, n), all nu in registers)
// g2 = |ep|^2 / (2 omega) accumulated in FP64 per thread, reduced per CTA into g2sum[nu, k].
// The next block's operands (g 24 KB, ukq 2 KB, uph 1.1 KB) are fetched with cp.async into the
// other half of a double buffer while the current block computes; two CTAs fit on an SM.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <int NW, int NM>
struct RotSmem {
  static constexpr int NB = NW, NT = NW * NW * NM, NC = NB * NM;  // NC columns (n, jm) of g
  static constexpr int GLD = NW + 2;                // padded column stride (complex): conflict-free float4 reads
  static constexpr int G = NC * GLD * 8, U = NW * NB * 8, PH = NM * NM * 8;
  static constexpr int BUF = G + U + PH;            // bytes of one operand buffer
  static constexpr int TLD = NB + 1;                // padded stride of T: conflict-free stores
  static constexpr int TOTAL = 2 * BUF + TLD * NC * 8;  // two buffers + T
};

// Thread tiles (256 threads, nw = 16, nm = 12):
//   stage 1: thread (mg, cg): m = 4 mg .. 4 mg + 3 (mg uniform per warp pair, so u reads broadcast),
//            c = cg + 64 j, j = 0..2; two iw per 16-byte load.
//   stage 2: thread (mng, ng): mn = mng + 64 i, i = 0..3, nu = 3 ng .. 3 ng + 2 (ng uniform per warp).
template <int NW, int NM>
__global__ void __launch_bounds__(256, 2) eph_rot_reduce_f32_kernel(
    const float* __restrict__ g, int64_t g_stride, const float2* __restrict__ ukq, const float2* __restrict__ uph,
    const float* __restrict__ inv2w, int64_t nkb, int64_t nq, double* __restrict__ g2sum,
    double* __restrict__ sample, int64_t stride, int64_t nsamp) {
  static_assert(NW == 16 && NM == 12, "thread tiling written for nw = 16, nm = 12");
  using L = RotSmem<NW, NM>;
  constexpr int NB = NW, NT = L::NT, NC = L::NC, GLD = L::GLD, TLD = L::TLD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* ts = reinterpret_cast<float2*>(smem_raw + 2 * L::BUF);
  __shared__ double red[NM];
  for (int e = threadIdx.x; e < NM; e += blockDim.x) red[e] = 0.0;
  double part[3] = {0.0, 0.0, 0.0};
  const int tid = threadIdx.x;
  const int mg = tid >> 6, cg = tid & 63;          // stage 1
  const int mng = tid & 63, ng = tid >> 6;         // stage 2
  const int64_t nblk = nkb * nq;
  auto prefetch = [&](int64_t blk, int64_t q, int buf) {
    if (blk < nblk) {
      unsigned char* dst = smem_raw + buf * L::BUF;
      const char* gs = reinterpret_cast<const char*>(g + blk * g_stride);
      const char* us = reinterpret_cast<const char*>(ukq + blk * NW * NB);
      const char* ps = reinterpret_cast<const char*>(uph + q * NM * NM);
      // g: column c (NW complex = 128 B = 8 chunks) goes to the padded slot c * GLD
      for (int ch = tid; ch < NC * 8; ch += blockDim.x) {
        const int c = ch >> 3, w = ch & 7;
        cp_async16(dst + (c * GLD) * 8 + 16 * w, gs + 128 * c + 16 * w);
      }
      for (int ch = tid; ch < L::U / 16; ch += blockDim.x) cp_async16(dst + L::G + 16 * ch, us + 16 * ch);
      for (int ch = tid; ch < L::PH / 16; ch += blockDim.x) cp_async16(dst + L::G + L::U + 16 * ch, ps + 16 * ch);
    }
    cp_async_commit();
  };
  auto flush = [&](int64_t k) {
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      atomicAdd(&red[3 * ng + j], part[j]);
      part[j] = 0.0;
    }
    __syncthreads();
    if (tid < NM) {
      atomicAdd(&g2sum[tid + NM * k], red[tid]);
      red[tid] = 0.0;
    }
  };
  int64_t kcur = -1;
  int buf = 0;
  // (k, q) of the block, advanced by the grid stride without 64-bit divisions in the loop
  const int64_t dk = gridDim.x / nq, dq = gridDim.x % nq;
  int64_t kl = blockIdx.x / nq, q = blockIdx.x % nq;
  prefetch(blockIdx.x, q, 0);
  for (int64_t blk = blockIdx.x; blk < nblk; blk += gridDim.x, buf ^= 1) {
    int64_t kn = kl + dk, qn = q + dq;
    if (qn >= nq) {
      qn -= nq;
      ++kn;
    }
    prefetch(blk + gridDim.x, qn, buf ^ 1);
    if (kl != kcur) {  // uniform across the CTA
      if (kcur >= 0) flush(kcur);
      kcur = kl;
    }
    cp_async_wait1();
    __syncthreads();
    const unsigned char* cb = smem_raw + buf * L::BUF;
    const float4* g4 = reinterpret_cast<const float4*>(cb);              // (iw, iw+1) pairs, column stride GLD/2
    const float4* u4 = reinterpret_cast<const float4*>(cb + L::G);       // column m: 8 float4
    const float2* ps = reinterpret_cast<const float2*>(cb + L::G + L::U);
    // ---- stage 1: T[m, c] = sum_iw conj(u[iw, m]) g[iw, c] ----
    {
      float2 acc[4][3];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[i][j] = make_float2(0.f, 0.f);
#pragma unroll
      for (int ip = 0; ip < NW / 2; ++ip) {
        float4 uu[4], gg[3];
#pragma unroll
        for (int i = 0; i < 4; ++i) uu[i] = u4[(4 * mg + i) * (NW / 2) + ip];
#pragma unroll
        for (int j = 0; j < 3; ++j) gg[j] = g4[(cg + 64 * j) * (GLD / 2) + ip];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            cfma_conj(acc[i][j], make_float2(uu[i].x, uu[i].y), make_float2(gg[j].x, gg[j].y));
            cfma_conj(acc[i][j], make_float2(uu[i].z, uu[i].w), make_float2(gg[j].z, gg[j].w));
          }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) ts[(4 * mg + i) + TLD * (cg + 64 * j)] = acc[i][j];
    }
    __syncthreads();
    // ---- stage 2: ep[mn, nu] = sum_jm T[mn, jm] uph[jm, nu], g2, partial sums ----
    {
      float2 acc[4][3];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[i][j] = make_float2(0.f, 0.f);
#pragma unroll
      for (int jm = 0; jm < NM; ++jm) {
        float2 tt[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int mn = mng + 64 * i, m = mn & (NB - 1), n = mn / NB;
          tt[i] = ts[m + TLD * (n + NB * jm)];
        }
        float2 pp[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) pp[j] = ps[jm + NM * (3 * ng + j)];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) cfma(acc[i][j], tt[i], pp[j]);
      }
      const bool samp = sample && ((uint32_t)q % (uint32_t)stride == 0);
      double* sq = samp ? sample + ((kl * nsamp) + (uint32_t)q / (uint32_t)stride) * (int64_t)NT : nullptr;
      const float* w2 = inv2w + q * NM;  // 1 / (2 omega) of this q, FP32
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int nu = 3 * ng + j;
        const float inv2w_nu = w2[nu];
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float v = (acc[i][j].x * acc[i][j].x + acc[i][j].y * acc[i][j].y) * inv2w_nu;
          s += v;
          if (samp) sq[mng + 64 * i + NB * NB * nu] = (double)v;
        }
        part[j] += (double)s;
      }
    }
    __syncthreads();  // the next iteration's prefetch overwrites this buffer
    kl = kn;
    q = qn;
  }
  if (kcur >= 0) flush(kcur);
}

// The same rotation + |g|^2 fold + reduction for any (nw, nm) the tiled kernel above does not cover: one
// CTA per (k, q) block, operands and T in shared memory, FP32 arithmetic, the per-mode sums of a block
// added in shared memory (FP64) and then once into g2sum. Same inputs and outputs as the tiled kernel.
__global__ void __launch_bounds__(256) eph_rot_reduce_gen_kernel(
    const float2* __restrict__ g, int64_t g_stride, const float2* __restrict__ ukq, const float2* __restrict__ uph,
    const double* __restrict__ omega, int nw, int nm, int64_t nkb, int64_t nq, double* __restrict__ g2sum,
    double* __restrict__ sample, int64_t stride, int64_t nsamp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nw2 = nw * nw, nd = nw2 * nm;
  float2* gs = reinterpret_cast<float2*>(smem_raw);  // g[iw, n, jm]
  float2* ts = gs + nd;                                // T[m, n, jm]
  float2* us = ts + nd;                                // u_kq[iw, m]
  float2* ps = us + nw2;                               // u_ph[jm, nu]
  double* red = reinterpret_cast<double*>(ps + nm * nm);
  const int64_t nblk = nkb * nq;
  for (int64_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const int64_t kl = blk / nq, q = blk % nq;
    for (int e = threadIdx.x; e < nd; e += blockDim.x) gs[e] = g[blk * g_stride + e];
    for (int e = threadIdx.x; e < nw2; e += blockDim.x) us[e] = ukq[blk * nw2 + e];
    for (int e = threadIdx.x; e < nm * nm; e += blockDim.x) ps[e] = uph[q * nm * nm + e];
    for (int e = threadIdx.x; e < nm; e += blockDim.x) red[e] = 0.0;
    __syncthreads();
    for (int e = threadIdx.x; e < nd; e += blockDim.x) {
      const int m = e % nw, r = e / nw;  // r = n + nw jm
      float2 acc = make_float2(0.f, 0.f);
      for (int iw = 0; iw < nw; ++iw) cfma_conj(acc, us[iw + nw * m], gs[iw + nw * r]);
      ts[e] = acc;
    }
    __syncthreads();
    const bool samp = sample && (q % stride == 0);
    double* sq = samp ? sample + ((kl * nsamp) + q / stride) * (int64_t)nd : nullptr;
    for (int e = threadIdx.x; e < nd; e += blockDim.x) {
      const int mn = e % nw2, nu = e / nw2;
      float2 acc = make_float2(0.f, 0.f);
      for (int jm = 0; jm < nm; ++jm) cfma(acc, ts[mn + nw2 * jm], ps[jm + nm * nu]);
      const float v = (acc.x * acc.x + acc.y * acc.y) * (float)(0.5 / omega[q * nm + nu]);
      if (samp) sq[e] = (double)v;
      atomicAdd(&red[nu], (double)v);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nm; e += blockDim.x) atomicAdd(&g2sum[e + nm * kl], red[e]);
    __syncthreads();  // red and the operand buffers are rewritten by the next block
  }
}

int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* xk,
                int64_t N, double2* out, int64_t ldo);
int eigh_async(epb_ctx* ctx, double2* A, int64_t n, int64_t batch, double* E, bool want_v, const double* mass,
               int prec);
int eigh_mixed_packed(epb_ctx* ctx, const float* Hp, int64_t n, int64_t batch, float2* U, double* E);
int eigh16_mixed_jacobi(epb_ctx* ctx, const float* Hp, int64_t batch, float2* V32);
int eigh16_mixed_refine(epb_ctx* ctx, const float* Hp, int64_t batch, float2* V32, float2* U, int64_t* gap_list,
                        int* gap_count, int gap_cap, float gap_rel);
int eigh16_fixup_launch(epb_ctx* ctx, const int64_t* list, const int* count, int cap, const double2* ham,
                        const int4* rv, int64_t nr, const double* xk, const double* xq, int64_t nq, float2* U32,
                        double2* hbuf);
// Near-degenerate k+q matrices: H(k+q) is formed at the FP32 level (error ~1e-7 of max |lambda|), which turns
// the eigenvectors of a pair with gap g by about that error over g and so reaches |g|^2 (a pair with a
// relative gap of 6.5e-4 measured 1.0e-5 per-block |g|^2 error). Matrices whose smallest gap is below
// PASS_GAP_REL * max |lambda| are listed by the refinement and re-solved from an FP64 H(k+q); the rest then
// stay under about 3e-6. About 1e-4 of random k+q points fall below the threshold.
constexpr float PASS_GAP_REL = 2e-3f;

// The whole mixed pass after the q side (omega, u_ph in FP64) has been computed.
int mixed_pass(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double* xq, int64_t nq,
               const double2* uph, const double* omega, double* ek_out, double* g2sum, double* g2_sample,
               int64_t sample_stride, int64_t kbi_max, bool defer_checks) {
  MixedModel* mm = (MixedModel*)m->mixed;
  const int64_t nw = m->nw, nm = m->nm, nw2 = nw * nw;
  const int64_t nd = nw2 * nm, nd_ep = nd * m->nr_ep;
  const bool tiled = nw == 16 && nm == 12;  // the register-tiled rotation; other shapes take the generic kernel
  const size_t gen_smem = 8 * (size_t)(2 * nw2 * nm + nw2 + nm * nm) + 8 * (size_t)nm;
  EPB_CHECK_ARG(nq < (int64_t(1) << 31) && (!g2_sample || (sample_stride >= 1 && sample_stride < (int64_t(1) << 31))),
                "mixed pass: nq = %lld and the sample stride %lld must lie in 1 .. 2^31 - 1", (long long)nq,
                (long long)sample_stride);
  EPB_CHECK_ARG(tiled || gen_smem <= 200 * 1024,
                "mixed pass: a (k, q) block of nw=%lld, nm=%lld needs %zu bytes of shared memory (over 200 KB); use "
                "the FP64 pass", (long long)nw, (long long)nm, gen_smem);
  const int64_t KO = 256;                               // RR->kR batch (one read of the g(Re,Rp) planes)
  const int64_t kbi = kbi_max < KO ? kbi_max : KO;      // H(k+q) / kR->kq batch
  const int64_t KC_ep = kchunks(m->nr_ep), KC_el = kchunks(m->nr_el);
  const int64_t rows_pad_k = round_up(2 * nd, 128);
  // ---- workspace ----
  size_t off = 0;
  auto carve = [&](int64_t bytes) {
    size_t o = off;
    off += ((size_t)bytes + 1023) & ~size_t(1023);
    return o;
  };
  const size_t o_bp = carve(MX_NPL * plane_bytes_for(round_up(nq, MX_NT), KC_ep));
  const size_t o_uph = carve(8 * nm * nm * nq);
  const size_t o_hk = carve(16 * nw2 * KO);
  const size_t o_bk = carve(MX_NPL * plane_bytes_for(round_up(KO, MX_NT), KC_el));
  const size_t o_c0 = carve(4 * 2 * nd_ep * KO);
  const size_t o_a2 = carve(MX_NPL * plane_bytes_for(rows_pad_k * KO, KC_ep));
  const size_t o_bqel = carve(MX_NPL * plane_bytes_for(round_up(nq, MX_NT), KC_el));  // q phases over Re
  const size_t o_ah = carve(MX_NPL * plane_bytes_for(kbi * mm->H.rows_pad, KC_el));     // modulated H(R) rows
  const size_t o_c1 = carve(4 * nw2 * kbi * nq);
  const size_t o_u32 = carve(8 * nw2 * kbi * nq);
  const size_t o_c2 = carve(4 * 2 * nd * kbi * nq);
  const size_t o_w2 = carve(4 * nm * nq);  // 1 / (2 omega), FP32
  const size_t o_mx = carve(16);           // float bits: max |G| of the outer batch, max |u_ph|
  const size_t o_rp = carve(8 * rot_mma_partial_doubles(ctx, kbi));  // per-warp mode sums of the rotation
  // the inner-batch pipeline (register-tiled shape, streams allowed): second buffers of packed H(k+q) and
  // g(k, q), and the FP32 Jacobi vectors of both parities
  const bool pipe = tiled && !ctx->prof_on;
  const size_t o_c1b = carve(pipe ? 4 * nw2 * kbi * nq : 0);
  const size_t o_c2b = carve(pipe ? 4 * 2 * nd * kbi * nq : 0);
  const size_t o_v32 = carve(tiled ? (pipe ? 2 : 1) * 8 * nw2 * kbi * nq : 0);
  // list of the near-degenerate matrices of an inner batch (refinement -> FP64 re-solve) and its count
  const int gap_cap = (int)std::min<int64_t>(kbi * nq, std::max<int64_t>(4096, kbi * nq / 64));
  const size_t o_gap = carve(tiled ? 8 * (int64_t)gap_cap + 256 : 0);
  const size_t o_gaph = carve(tiled ? 16 * 256 * (int64_t)gap_cap : 0);  // their FP64 H(k+q), nw = 16
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS1, off + 1024, &ws));
  uint8_t* base = (uint8_t*)(((uintptr_t)ws + 1023) & ~uintptr_t(1023));
  float2* uph32 = (float2*)(base + o_uph);
  double2* Hk = (double2*)(base + o_hk);
  float* C0 = (float*)(base + o_c0);
  float* C1 = (float*)(base + o_c1);
  float2* U32 = (float2*)(base + o_u32);
  float* C2 = (float*)(base + o_c2);
  const int64_t nsamp = g2_sample ? (nq + sample_stride - 1) / sample_stride : 0;

  // ---- q side: phase planes of the q list, u_ph in complex64 ----
  // kR->kq in the FP16x2 configuration (three products): G_k is pre-scaled by a power of two that keeps
  // |G| <= sqrt(nw) nr_el max|g(Re,Rp)| below 2^14 (FP16 range), the epilogue multiplies it back out
  Planes Bp;
  EPB_TRY(pack_b_phase_h(ctx, m->rs_ep, xq, nullptr, 1, nq, Bp, base + o_bp));
  // H(k+q) is (H(R) modulated by k) x (q phases over Re): the q side is packed once for the pass
  Planes Bq_el;
  EPB_TRY(pack_b_phase(ctx, m->rs_el, xq, nullptr, 1, nq, Bq_el, base + o_bqel));
  double gbound = std::sqrt((double)nw) * (double)m->nr_el * (mm->ep_absmax > 0.0 ? mm->ep_absmax : 1.0);
  const int e2 = std::max(-120, std::min(120, 14 - (int)std::ceil(std::log2(gbound))));
  const double a2_scale = std::ldexp(1.0, e2);
  const float a2_unscale = (float)std::ldexp(1.0, -e2);
  unsigned* gmax = (unsigned*)(base + o_mx);
  unsigned* phmax = gmax + 1;
  EPB_CUDA(cudaMemsetAsync(gmax, 0, 2 * sizeof(unsigned), ctx->stream));
  c128_to_c64_absmax_kernel<<<grid_for(ctx, nm * nm * nq), 256, 0, ctx->stream>>>(uph, uph32, nm * nm * nq, phmax);
  EPB_LAUNCH_CHECK();
  float* inv2w = (float*)(base + o_w2);
  inv2w_kernel<<<grid_for(ctx, nm * nq), 256, 0, ctx->stream>>>(omega, inv2w, nm * nq);
  EPB_LAUNCH_CHECK();
  Planes A2;
  A2.rows_pad = rows_pad_k * KO;
  A2.KC = KC_ep;
  A2.plane_bytes = plane_bytes_for(A2.rows_pad, KC_ep);
  A2.npl = 2;
  A2.p = base + o_a2;
  if (rows_pad_k != 2 * nd) EPB_CUDA(cudaMemsetAsync(A2.p, 0, 2 * A2.plane_bytes, ctx->stream));

  // side stream for the kR->kq GEMM (not while the per-family profile is recorded: it times each family
  // on the main stream)
  bool side = false;
  if (!ctx->prof_on) {
    EPB_TRY(side_stream(ctx));
    side = true;
  }
  if (pipe) EPB_TRY(pipe_streams(ctx));
  // Inner-batch pipeline: batch i (buffer parity p = i & 1) runs the H(k+q) GEMM and the FP32 Jacobi on the
  // caller's stream, the kR->kq GEMM on the side stream, and the FP64 refinement + rotation on the tail
  // stream, so the tail work of batch i overlaps the H GEMM and Jacobi of batch i + 1 (different pipes:
  // FP64 and warp tensor cores beside FP32 and tcgen05). Events per parity: H GEMM, Jacobi, kR->kq,
  // refinement, rotation done. A buffer of parity p is rewritten only after its last reader (of batch
  // i - 2) has finished: the caller's stream waits for refinement[p] before the H GEMM (packed H and the
  // Jacobi vectors), the side stream waits for rotation[p] before kR->kq (g). The refined vectors and the
  // rotation's partial sums stay single: their writer and reader are both on the tail stream.
  cudaEvent_t* evH = ctx->pipe_ev + 0;
  cudaEvent_t* evJ = ctx->pipe_ev + 2;
  cudaEvent_t* evK = ctx->pipe_ev + 4;
  cudaEvent_t* evR = ctx->pipe_ev + 6;
  cudaEvent_t* evT = ctx->pipe_ev + 8;
  bool recK[2] = {false, false}, recR[2] = {false, false}, recT[2] = {false, false};
  int64_t bi = 0;  // inner batches so far (buffer parity across outer batches)
  const cudaStream_t main_stream = ctx->stream;
  for (int64_t ko = 0; ko < nk; ko += KO) {
    if (pipe) {
      // the previous outer batch's kR->kq GEMMs read A2 and its rotations read gmax: both are rewritten below
      for (int p = 0; p < 2; ++p) {
        if (recK[p]) EPB_CUDA(cudaStreamWaitEvent(main_stream, evK[p], 0));
        if (recT[p]) EPB_CUDA(cudaStreamWaitEvent(main_stream, evT[p], 0));
      }
    }
    const int64_t nko = nk - ko < KO ? nk - ko : KO;
    const double* xko = xk + 3 * ko;
    // electrons at k (FP64: the k side is 0.01% of the pass and fixes the k-leg gauge)
    EPB_TRY(fourier_f64(ctx, m->ham, nw2, nw2, m->rs_el, xko, nko, Hk, nw2));
    EPB_TRY(eigh_async(ctx, Hk, nw, nko, ek_out + nw * ko, true, nullptr, EPB_PREC_FP64));
    // RR->kR on the tensor cores: C0[:, k] = g(k) (complex64, "el" row order)
    Planes Bk;
    EPB_TRY(pack_b_phase(ctx, m->rs_el, xko, nullptr, 1, nko, Bk, base + o_bk));
    EPB_TRY(split_gemm(ctx, EPB_PROF_UMMA_RR, mm->EP, Bk, mm->EP.rows_pad / 128, 1, 2 * nd_ep, nko, false, C0, 0,
                       2 * nd_ep));
    // k-leg rotation by u_k fused into the A2 packing of the kR->kq GEMM
    {
      const int64_t total = nko * nd * (sin_offset(m->nr_ep) / 8);
      // the previous outer batch's rotations (readers of gmax) precede this on the stream
      EPB_CUDA(cudaMemsetAsync(gmax, 0, sizeof(unsigned), ctx->stream));
      prof_begin(ctx, EPB_PROF_RR_ROT);
      rr_rotate_pack_kernel<false, 2><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
          (const float2*)C0, Hk, (int)nw, (int)nw, (int)nm, (int)m->nr_ep, nko, rows_pad_k, KC_ep, A2.p, A2.plane_bytes,
          a2_scale, gmax);
      prof_end(ctx);
      EPB_LAUNCH_CHECK();
    }
    for (int64_t ki = 0; ki < nko; ki += kbi) {
      const int64_t nki = nko - ki < kbi ? nko - ki : kbi;
      const int64_t np = nki * nq;
      if (pipe) {
        const int p = (int)(bi++ & 1);
        float* C1p = p ? (float*)(base + o_c1b) : C1;
        float* C2p = p ? (float*)(base + o_c2b) : C2;
        float2* V32p = (float2*)(base + o_v32) + (size_t)p * nw2 * kbi * nq;
        if (recR[p]) EPB_CUDA(cudaStreamWaitEvent(main_stream, evR[p], 0));  // C1p, V32p free again
        Planes Ah;
        EPB_TRY(pack_a_herm_mod(ctx, m->ham, m->rs_el, (int)nw, xko + 3 * ki, nki, mm->H.rows_pad, Ah, base + o_ah));
        EPB_TRY(split_gemm(ctx, EPB_PROF_UMMA_H, Ah, Bq_el, mm->H.rows_pad / 128, nki, nw2, nq, true, C1p, nw2 * nq,
                           nw2));
        EPB_CUDA(cudaEventRecord(evH[p], main_stream));
        // side: kR->kq into C2p once the rotation of batch i - 2 has read it
        Planes A2i = A2;
        A2i.p = A2.p + ki * rows_pad_k / 128 * KC_ep * TILE_BYTES;
        EPB_CUDA(cudaStreamWaitEvent(ctx->side, evH[p], 0));
        if (recT[p]) EPB_CUDA(cudaStreamWaitEvent(ctx->side, evT[p], 0));
        ctx->stream = ctx->side;
        int st = split_gemm_h(ctx, EPB_PROF_UMMA_KQ, A2i, Bp, rows_pad_k / 128, nki, 2 * nd, nq, false, C2p,
                              2 * nd * nq, 2 * nd, a2_unscale, ctx->cur_kq_ares);
        if (st == EPB_OK) st = cudaEventRecord(evK[p], ctx->side) == cudaSuccess ? EPB_OK : EPB_ERR_CUDA;
        ctx->stream = main_stream;
        EPB_TRY(st);
        recK[p] = true;
        // caller's stream: FP32 Jacobi of the packed H(k+q)
        EPB_TRY(eigh16_mixed_jacobi(ctx, C1p, np, V32p));
        EPB_CUDA(cudaEventRecord(evJ[p], main_stream));
        // tail: FP64 refinement, then the rotation + |g|^2 fold + reduction
        EPB_CUDA(cudaStreamWaitEvent(ctx->tail, evJ[p], 0));
        EPB_CUDA(cudaStreamWaitEvent(ctx->tail, evK[p], 0));
        ctx->stream = ctx->tail;
        {
          int64_t* gl = (int64_t*)(base + o_gap);
          int* gc = (int*)(base + o_gap + 8 * (size_t)gap_cap);
          if (cudaMemsetAsync(gc, 0, sizeof(int), ctx->stream) != cudaSuccess) st = EPB_ERR_CUDA;
          if (st == EPB_OK) st = eigh16_mixed_refine(ctx, C1p, np, V32p, U32, gl, gc, gap_cap, PASS_GAP_REL);
          if (st == EPB_OK)
            st = eigh16_fixup_launch(ctx, gl, gc, gap_cap, m->ham, m->rs_el->dev, m->nr_el, xko + 3 * ki, xq, nq, U32,
                                     (double2*)(base + o_gaph));
        }
        if (st == EPB_OK) st = cudaEventRecord(evR[p], ctx->tail) == cudaSuccess ? EPB_OK : EPB_ERR_CUDA;
        if (st == EPB_OK) {
          if (ctx->cur_rot == 0) {
            st = rot_mma_launch(ctx, C2p, 2 * nd, U32, uph32, inv2w, gmax, phmax, a2_unscale, (int)m->nr_ep, nki, nq,
                                g2sum + nm * (ko + ki), (double*)(base + o_rp),
                                g2_sample ? g2_sample + (ko + ki) * nsamp * nd : nullptr, sample_stride, nsamp);
          } else {
            constexpr int RS = RotSmem<16, 12>::TOTAL;
            static bool pattr = false;
            if (!pattr && cudaFuncSetAttribute(eph_rot_reduce_f32_kernel<16, 12>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, RS) == cudaSuccess)
              pattr = true;
            const unsigned grid = (unsigned)std::min<int64_t>(np, (int64_t)ctx->sm_count * 2);
            eph_rot_reduce_f32_kernel<16, 12><<<grid, 256, RS, ctx->stream>>>(
                C2p, 2 * nd, U32, uph32, inv2w, nki, nq, g2sum + nm * (ko + ki),
                g2_sample ? g2_sample + (ko + ki) * nsamp * nd : nullptr, sample_stride, nsamp);
            ++ctx->launches;
            if (cudaGetLastError() != cudaSuccess) st = EPB_ERR_CUDA;
          }
        }
        if (st == EPB_OK) st = cudaEventRecord(evT[p], ctx->tail) == cudaSuccess ? EPB_OK : EPB_ERR_CUDA;
        ctx->stream = main_stream;
        if (st == EPB_ERR_CUDA) set_error("mixed pass pipeline: a launch or event on the tail stream failed");
        EPB_TRY(st);
        recR[p] = recT[p] = true;
        continue;
      }
      // H(k+q) on the tensor cores: Hermitian-packed rows of H(R) exp(2 pi i R.k) per k times the q phases,
      // then FP32 solve + FP64 refinement
      Planes Ah;
      EPB_TRY(pack_a_herm_mod(ctx, m->ham, m->rs_el, (int)nw, xko + 3 * ki, nki, mm->H.rows_pad, Ah, base + o_ah));
      EPB_TRY(split_gemm(ctx, EPB_PROF_UMMA_H, Ah, Bq_el, mm->H.rows_pad / 128, nki, nw2, nq, true, C1, nw2 * nq,
                         nw2));
      // kR->kq on the tensor cores, batched over the k of this inner batch. It needs neither the
      // eigensolvers' results nor their resources (the FP32 Jacobi holds no shared memory), so outside the
      // per-family profile it runs on the side stream beside them: it starts once the H(k+q) GEMM has
      // finished (by then the previous batch's rotation, the last reader of C2, is done as well) and the
      // rotation below waits for it.
      Planes A2i = A2;
      A2i.p = A2.p + ki * rows_pad_k / 128 * KC_ep * TILE_BYTES;
      if (side) {
        EPB_CUDA(cudaEventRecord(ctx->side_ev[0], ctx->stream));
        EPB_CUDA(cudaStreamWaitEvent(ctx->side, ctx->side_ev[0], 0));
        cudaStream_t main_stream = ctx->stream;
        ctx->stream = ctx->side;
        const int st = split_gemm_h(ctx, EPB_PROF_UMMA_KQ, A2i, Bp, rows_pad_k / 128, nki, 2 * nd, nq, false, C2,
                                    2 * nd * nq, 2 * nd, a2_unscale, ctx->cur_kq_ares);
        ctx->stream = main_stream;
        EPB_TRY(st);
        EPB_CUDA(cudaEventRecord(ctx->side_ev[1], ctx->side));
      }
      if (tiled) {  // the same solve as the pipeline's: FP32 Jacobi, refinement, FP64 re-solve of near-degenerate
        float2* V32 = (float2*)(base + o_v32);
        int64_t* gl = (int64_t*)(base + o_gap);
        int* gc = (int*)(base + o_gap + 8 * (size_t)gap_cap);
        EPB_TRY(eigh16_mixed_jacobi(ctx, C1, np, V32));
        EPB_CUDA(cudaMemsetAsync(gc, 0, sizeof(int), ctx->stream));
        EPB_TRY(eigh16_mixed_refine(ctx, C1, np, V32, U32, gl, gc, gap_cap, PASS_GAP_REL));
        EPB_TRY(eigh16_fixup_launch(ctx, gl, gc, gap_cap, m->ham, m->rs_el->dev, m->nr_el, xko + 3 * ki, xq, nq, U32,
                                    (double2*)(base + o_gaph)));
      } else {
        EPB_TRY(eigh_mixed_packed(ctx, C1, nw, np, U32, nullptr));
      }
      if (side) {
        EPB_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1], 0));
      } else {
        EPB_TRY(split_gemm_h(ctx, EPB_PROF_UMMA_KQ, A2i, Bp, rows_pad_k / 128, nki, 2 * nd, nq, false, C2,
                             2 * nd * nq, 2 * nd, a2_unscale, ctx->cur_kq_ares));
      }
      // rotations, g2, in-place reduction
      if (!tiled) {
        static bool gattr = false;
        if (!gattr) {
          EPB_CUDA(cudaFuncSetAttribute(eph_rot_reduce_gen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
          gattr = true;
        }
        const unsigned grid = (unsigned)std::min<int64_t>(np, (int64_t)ctx->sm_count * 4);
        prof_begin(ctx, EPB_PROF_ROT);
        eph_rot_reduce_gen_kernel<<<grid, 256, gen_smem, ctx->stream>>>(
            (const float2*)C2, nd, U32, uph32, omega, (int)nw, (int)nm, nki, nq, g2sum + nm * (ko + ki),
            g2_sample ? g2_sample + (ko + ki) * nsamp * nd : nullptr, sample_stride, nsamp);
        prof_end(ctx);
        EPB_LAUNCH_CHECK();
      } else if (ctx->cur_rot == 0) {
        prof_begin(ctx, EPB_PROF_ROT);
        const int st = rot_mma_launch(ctx, C2, 2 * nd, U32, uph32, inv2w, gmax, phmax, a2_unscale, (int)m->nr_ep, nki,
                                      nq, g2sum + nm * (ko + ki), (double*)(base + o_rp),
                                      g2_sample ? g2_sample + (ko + ki) * nsamp * nd : nullptr, sample_stride, nsamp);
        prof_end(ctx);
        EPB_TRY(st);
      } else {
        int64_t nblk = np;
        constexpr int RS = RotSmem<16, 12>::TOTAL;
        static bool rattr = false;
        if (!rattr) {
          EPB_CUDA(cudaFuncSetAttribute(eph_rot_reduce_f32_kernel<16, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, RS));
          rattr = true;
        }
        unsigned grid = (unsigned)(nblk < (int64_t)ctx->sm_count * 2 ? nblk : (int64_t)ctx->sm_count * 2);
        prof_begin(ctx, EPB_PROF_ROT);
        eph_rot_reduce_f32_kernel<16, 12><<<grid, 256, RS, ctx->stream>>>(
            C2, 2 * nd, U32, uph32, inv2w, nki, nq, g2sum + nm * (ko + ki),
            g2_sample ? g2_sample + (ko + ki) * nsamp * nd : nullptr, sample_stride, nsamp);
        prof_end(ctx);
        EPB_LAUNCH_CHECK();
      }
    }
  }
  if (pipe) {  // join the side and tail streams back into the caller's stream
    for (int p = 0; p < 2; ++p) {
      if (recK[p]) EPB_CUDA(cudaStreamWaitEvent(main_stream, evK[p], 0));
      if (recT[p]) EPB_CUDA(cudaStreamWaitEvent(main_stream, evT[p], 0));
    }
  }
  return defer_checks ? EPB_OK : split_gemm_check(ctx);
}

}  // namespace epb
