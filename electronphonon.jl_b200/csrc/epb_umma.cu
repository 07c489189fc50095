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
//               accumulator of 128 lanes x NT columns; two accumulators alternate so the epilogue
//               of one tile overlaps the MMAs of the next
//   warps 2-5   epilogue: tcgen05.ld of the accumulator, FP32 stores to C
// Every wait is bounded (clock64 budget); on timeout the kernel raises an error flag, drains its
// own copies and MMAs, frees TMEM and returns (EPB_ERR_TIMEOUT on the host).
#include "epb_common.cuh"
#include "epb_umma.cuh"

struct epb_model;

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
// Packers. All write every element of the padded planes (zeros in the padding).

// Generic complex operand A (M x K complex, column-major, leading dim ld) -> A2 (2M_pad x K2_pad).
template <bool BF16, int NPL>
__global__ void pack_a_complex_kernel(const double2* __restrict__ a, int64_t ld, int64_t M, int64_t K,
                                      int64_t rows_pad, int64_t KC, uint8_t* __restrict__ planes,
                                      int64_t plane_bytes) {
  const int64_t Kp = KC * 64;
  const int64_t total = rows_pad * Kp;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t k = idx % Kp, row = idx / Kp;
    double v = 0.0;
    int64_t i = row >> 1;
    int part = (int)(row & 1);
    if (i < M) {
      if (k < K) {
        double2 x = a[i + k * ld];
        v = part == 0 ? x.x : x.y;
      } else if (k < 2 * K) {
        double2 x = a[i + (k - K) * ld];
        v = part == 0 ? -x.y : x.x;
      }
    }
    store_split<BF16, NPL>(planes, plane_bytes, tiled_offset(row, k, KC), v);
  }
}

// Hermitian operand (nw x nw per R, column-major op_r (nw^2 x K)) -> packed real rows:
// rows [0, nw(nw+1)/2): Re H_ij (i <= j, ordered j-major), rows after: Im H_ij (i < j).
__device__ __forceinline__ void herm_row_to_ij(int row, int nw, int& i, int& j, int& part) {
  const int nre = nw * (nw + 1) / 2;
  int r = row;
  part = 0;
  if (r >= nre) {
    part = 1;
    r -= nre;
    // strictly upper: column j has j entries (i < j)
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
  const int64_t Kp = KC * 64;
  const int64_t total = rows_pad * Kp;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t k = idx % Kp, row = idx / Kp;
    double v = 0.0;
    if (row < (int64_t)nw * nw && k < 2 * K) {
      int i, j, part;
      herm_row_to_ij((int)row, nw, i, j, part);
      int64_t kk = k < K ? k : k - K;
      double2 x = op[(i + (int64_t)j * nw) + kk * (int64_t)nw * nw];
      if (part == 0)
        v = k < K ? x.x : -x.y;   // Re H = Re h cos - Im h sin
      else
        v = k < K ? x.y : x.x;    // Im H = Im h cos + Re h sin
    }
    store_split<BF16, NPL>(planes, plane_bytes, tiled_offset(row, k, KC), v);
  }
}

// Phase operand: column j of B2 = [cos 2 pi R.x_j (K) ; sin 2 pi R.x_j (K) ; 0], stored as the
// K-major row j. x_j = xa[:, ja] + xb[:, jb] with (ja, jb) = (j / nb, j % nb) when xb != null
// (x_{k+q} for every pair of a k batch), else x_j = xa[:, j].
template <bool BF16, int NPL>
__global__ void pack_b_phase_kernel(const int4* __restrict__ rv, int64_t K, const double* __restrict__ xa,
                                    const double* __restrict__ xb, int64_t nb, int64_t N, int64_t rows_pad,
                                    int64_t KC, uint8_t* __restrict__ planes, int64_t plane_bytes) {
  const int64_t total = rows_pad * K;  // one thread per (point, R): writes both cos and sin
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t p = idx % K, j = idx / K;
    double c = 0.0, s = 0.0;
    if (j < N) {
      double x0, x1, x2;
      if (xb) {
        int64_t ja = j / nb, jb = j % nb;
        x0 = xa[3 * ja] + xb[3 * jb];
        x1 = xa[3 * ja + 1] + xb[3 * jb + 1];
        x2 = xa[3 * ja + 2] + xb[3 * jb + 2];
      } else {
        x0 = xa[3 * j];
        x1 = xa[3 * j + 1];
        x2 = xa[3 * j + 2];
      }
      int4 r = rv[p];
      double t = rdotx(r.x, r.y, r.z, x0, x1, x2);
      double2 e = cis2pi(t);
      c = e.x;
      s = e.y;
    }
    store_split<BF16, NPL>(planes, plane_bytes, tiled_offset(j, p, KC), c);
    store_split<BF16, NPL>(planes, plane_bytes, tiled_offset(j, K + p, KC), s);
  }
  // zero the K padding columns [2K, Kp)
  const int64_t Kp = KC * 64;
  const int64_t npad = Kp - 2 * K;
  if (npad > 0) {
    const int64_t tp = rows_pad * npad;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < tp;
         idx += (int64_t)gridDim.x * blockDim.x) {
      int64_t k = 2 * K + idx % npad, j = idx / npad;
      store_split<BF16, NPL>(planes, plane_bytes, tiled_offset(j, k, KC), 0.0);
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
    int64_t u = 0;
    for (int64_t t = blockIdx.x; t < total && ok; t += gridDim.x, ++u) {
      const int b = (int)(u & 1);
      const uint32_t use = (uint32_t)(u >> 1) & 1u;
      if (!mbar_wait(&tempty[b], use ^ 1u, err, a.timeout)) break;
      tc_fence_after();
      // accumulator 0 (columns [0, NT)) takes the leading h*h product, accumulator 1 (columns
      // [NT, 2NT)) all correction products: the tensor core aligns addends to the accumulator, so
      // O(2^-16) corrections added onto the O(1) sum would lose their low bits.
      const uint32_t dcol = tmem + b * 2 * NT;
      for (int kc = 0; kc < a.KC; ++kc) {
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
            // first MMA into each accumulator of the tile overwrites it
            const bool first = kc == 0 && sub == 0 && (lead || pr == 0);
            mma_f16(dcol + (lead ? 0u : (uint32_t)NT), ad, bd, IDESC, first ? 0u : 1u);
          }
        }
        mma_commit(&empty[s]);
        if (++s == STAGES) {
          s = 0;
          ph ^= 1u;
        }
      }
      if (ok) mma_commit(&tfull[b]);
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
    int64_t u = 0;
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x, ++u) {
      const int b = (int)(u & 1);
      const uint32_t use = (uint32_t)(u >> 1) & 1u;
      bool okw = mbar_wait(&tfull[b], use, err, a.timeout);
      if (!__all_sync(0xffffffffu, okw)) break;  // warp-uniform: the TMEM loads below are .sync.aligned
      tc_fence_after();
      int64_t mt = a.m_fastest ? t % a.m_tiles : t / a.n_tiles;
      int64_t nt = a.m_fastest ? t / a.m_tiles : t % a.n_tiles;
      const int64_t batch = mt / a.m_tiles_per_batch;
      const int64_t row = (mt % a.m_tiles_per_batch) * 128 + row_in_tile;
      float* cb = a.C + batch * a.c_batch_stride + row;
      const bool row_ok = row < a.m_valid;
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += 16) {
        float v[16], w[16];
        const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + b * 2 * NT + c0;
        tmem_ld16(ta, v);
        tmem_ld16(ta + NT, w);
        if (row_ok) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            int64_t col = nt * NT + c0 + j;
            if (col < a.n_valid) cb[col * a.ldc_n] = (float)((double)v[j] + (double)w[j]);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, Cfg::TMEM_COLS);
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
  out.KC = cdiv(2 * K, 64);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  int64_t total = out.rows_pad * out.KC * 64;
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_a_complex_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
      a, ld, M, K, out.rows_pad, out.KC, out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int pack_a_herm(epb_ctx* ctx, const double2* op, int nw, int64_t K, Planes& out, uint8_t* mem) {
  out.rows_pad = round_up((int64_t)nw * nw, 128);
  out.KC = cdiv(2 * K, 64);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  int64_t total = out.rows_pad * out.KC * 64;
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_a_herm_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(op, nw, K, out.rows_pad, out.KC,
                                                                                    out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int pack_b_phase(epb_ctx* ctx, const epb_rset* rs, const double* xa, const double* xb, int64_t nb, int64_t N,
                 Planes& out, uint8_t* mem) {
  out.rows_pad = round_up(N, MX_NT);
  out.KC = cdiv(2 * rs->nr, 64);
  out.plane_bytes = plane_bytes_for(out.rows_pad, out.KC);
  out.npl = MX_NPL;
  out.p = mem;
  int64_t total = out.rows_pad * rs->nr;
  prof_begin(ctx, EPB_PROF_SPLIT);
  pack_b_phase_kernel<MX_BF16, MX_NPL><<<grid_for(ctx, total), 256, 0, ctx->stream>>>(
      rs->dev, rs->nr, xa, xb, nb, N, out.rows_pad, out.KC, out.p, out.plane_bytes);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int64_t planes_bytes(int64_t rows, int64_t K) {
  return MX_NPL * plane_bytes_for(round_up(rows, 128), cdiv(2 * K, 64));
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

// epb_fourier(..., EPB_PREC_MIXED): pack op_r and the phases, split GEMM, widen to c128.
int fourier_mixed(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                  const double* xk, int64_t N, double2* out, int64_t ldo) {
  if (M == 0 || N == 0) return EPB_OK;
  const int64_t K = rs->nr;
  const int64_t a_bytes = planes_bytes(2 * M, K);
  const int64_t b_bytes = MX_NPL * plane_bytes_for(round_up(N, MX_NT), cdiv(2 * K, 64));
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

int mixed_model_prepare(epb_ctx* ctx, epb_model* m) {
  (void)ctx;
  (void)m;
  set_error("mixed-precision model planes are not available in this build");
  return EPB_ERR_UNSUPPORTED;
}

void mixed_model_free(epb_model* m) { (void)m; }

int mixed_pass_batch(epb_ctx* ctx, epb_model* m, const double* xk_b, int64_t nkb, const double* xq, int64_t nq,
                     const double2* uk_b, const double2* uph, const double* omega, const double2* phase,
                     double* g2sum_b, double* g2_sample_b, int64_t sample_stride, int64_t* stats) {
  (void)ctx; (void)m; (void)xk_b; (void)nkb; (void)xq; (void)nq; (void)uk_b; (void)uph; (void)omega;
  (void)phase; (void)g2sum_b; (void)g2_sample_b; (void)sample_stride; (void)stats;
  set_error("mixed-precision pass is not available in this build");
  return EPB_ERR_UNSUPPORTED;
}

}  // namespace epb
