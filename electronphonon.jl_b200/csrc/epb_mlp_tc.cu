// Surrogate inference on the tensor cores: the whole MLP of a 128-point tile in one CTA.
//
// Per tile (persistent CTAs, 128 threads = 4 warps, one row / TMEM lane per thread):
//  * Fourier features of the 128 points (FP64 argument reduction, FP32 sincospi) are written as BF16
//    straight into the A operand tile in shared memory (128 rows x nin, K-major, SWIZZLE_128B, 16 KB
//    per 64-column chunk);
//  * each layer is one batch of tcgen05.mma.kind::f16 (M = 128, N = fan_out <= 256, K = 16 per
//    instruction, BF16 x BF16 -> FP32 in TMEM) against the layer's weights, which a single
//    cp.async.bulk per 64-column chunk brings from a pre-built BF16 image (B operand rows = outputs,
//    K-major, same swizzle) into shared memory; the next layer's weights are fetched while the
//    epilogue of this one runs;
//  * the epilogue reads the accumulator (tcgen05.ld 32x32b), adds the FP32 bias, applies SiLU and
//    stores the BF16 activations back into the A tile (the next layer's operand); after the output
//    layer it writes the FP32 normalised predictions.
// The predictions differ from the FP32 kernels by BF16 rounding; the culling margins are calibrated
// with this same path. Every mbarrier wait is bounded: on timeout the CTA raises the context's error
// flag, waits (bounded) for its own copies and MMAs, frees TMEM and returns.
#include "epb_mlp.cuh"
#include "epb_umma.cuh"

namespace epb {

using namespace umma;

struct MlpTcArgs {
  const int4* fvec;
  int nf;
  const double* xa;
  const double* xb;
  int64_t nb;
  const int64_t* pidx;
  int64_t pair0;
  int64_t n;
  const uint8_t* wimg;       // weight image
  const float* params;       // biases
  int nlayer;                // hidden + output layers
  int fin[9], fout[9];
  int64_t woff[9];           // byte offset of each layer in the image
  int64_t boff[9];           // bias offsets in params
  float* out;                // n x nout
  int* err;
  long long timeout;
};

constexpr int TC_A_BYTES = 4 * 16384;          // 128 x 256 bf16
constexpr int TC_W_BYTES = 4 * 256 * 128;      // 256 x 256 bf16
constexpr int TC_SMEM = TC_A_BYTES + TC_W_BYTES + 1024 /*align*/ + 64 /*barriers*/;

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

__global__ void __launch_bounds__(128, 1) mlp_infer_tc_kernel(MlpTcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* As = smem;
  uint8_t* Ws = smem + TC_A_BYTES;
  uint64_t* wbar = reinterpret_cast<uint64_t*>(Ws + TC_W_BYTES);
  uint64_t* mbar = wbar + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  __shared__ int s_abort;
  volatile int* err = a.err;
  const int tid = threadIdx.x, warp = tid >> 5;

  if (tid == 0) {
    mbar_init(wbar, 1);
    mbar_init(mbar, 1);
    fence_barrier_init();
    s_abort = 0;
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int64_t ntiles = (a.n + 127) / 128;
  uint32_t wph = 0, mph = 0;       // barrier parities
  bool w_pending = false;          // a weight load was issued and not yet waited for
  bool m_pending = false;          // MMAs were issued and not yet waited for

  auto load_weights = [&](int l) {  // thread 0 only
    const int chunks = a.fin[l] / 64;
    const uint32_t cb = (uint32_t)a.fout[l] * 128u;
    mbar_arrive_expect_tx(wbar, cb * chunks);
    for (int c = 0; c < chunks; ++c) bulk_g2s(Ws + c * cb, a.wimg + a.woff[l] + (int64_t)c * cb, cb, wbar);
  };

  if (tid == 0 && (int64_t)blockIdx.x < ntiles) {
    load_weights(0);
    w_pending = true;
  }
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // ---- features -> A (row tid) ----
    {
      const int64_t j = tile * 128 + tid;
      double x0 = 0, x1 = 0, x2 = 0;
      const bool live = j < a.n;
      if (live) {
        if (a.xb) {
          const int64_t p = a.pidx ? a.pidx[j] : a.pair0 + j;
          const int64_t ja = p / a.nb, jb = p % a.nb;
          x0 = a.xa[3 * ja] + a.xb[3 * jb];
          x1 = a.xa[3 * ja + 1] + a.xb[3 * jb + 1];
          x2 = a.xa[3 * ja + 2] + a.xb[3 * jb + 2];
        } else {
          x0 = a.xa[3 * j];
          x1 = a.xa[3 * j + 1];
          x2 = a.xa[3 * j + 2];
        }
      }
      for (int f0 = 0; f0 < a.nf; f0 += 4) {  // 4 vectors = 8 values = one 16-byte unit
        uint32_t w4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float c = 0.f, s = 0.f;
          if (live) {
            const int4 v = a.fvec[f0 + q];
            const double t = rdotx(v.x, v.y, v.z, x0, x1, x2);
            sincospif(2.0f * (float)(t - rint(t)), &s, &c);
          }
          w4[q] = pack_bf16x2(c, s);
        }
        const int k = 2 * f0;  // first K column of the unit
        *reinterpret_cast<uint4*>(As + (k >> 6) * 16384 + sw128_offset(tid, k & 63)) =
            make_uint4(w4[0], w4[1], w4[2], w4[3]);
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    for (int l = 0; l < a.nlayer; ++l) {
      const int fin = a.fin[l], fout = a.fout[l];
      // ---- MMAs of layer l (one thread) ----
      if (tid == 0) {
        bool ok = mbar_wait(wbar, wph, err, a.timeout);
        if (ok) {
          w_pending = false;
          wph ^= 1u;
          tc_fence_after();
          const uint32_t idesc = idesc_f16(128, fout, true);
          const uint32_t cb = (uint32_t)fout * 128u;
          for (int c = 0; c < fin / 64; ++c)
#pragma unroll
            for (int sub = 0; sub < 4; ++sub) {
              const uint64_t ad = smem_desc_sw128(smem_u32(As + c * 16384 + sub * 32));
              const uint64_t bd = smem_desc_sw128(smem_u32(Ws + c * cb + sub * 32));
              mma_f16(tmem, ad, bd, idesc, (c | sub) ? 1u : 0u);
            }
          mma_commit(mbar);
          m_pending = true;
        } else {
          s_abort = 1;
        }
      }
      __syncthreads();
      if (s_abort) break;
      // ---- wait for the accumulator ----
      const bool okm = mbar_wait(mbar, mph, err, a.timeout);
      if (!okm) s_abort = 1;
      __syncthreads();
      if (s_abort) break;
      mph ^= 1u;
      if (tid == 0) {
        m_pending = false;
        // the weight buffer is free: fetch the next layer (or the first layer of the next tile)
        const int nl = l + 1 < a.nlayer ? l + 1 : 0;
        if (l + 1 < a.nlayer || tile + gridDim.x < ntiles) {
          load_weights(nl);
          w_pending = true;
        }
      }
      tc_fence_after();
      // ---- epilogue: row tid, TMEM lane tid ----
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
      const float* bias = a.params + a.boff[l];
      if (l + 1 < a.nlayer) {
        for (int c0 = 0; c0 < fout; c0 += 16) {
          float v[16];
          tmem_ld16(trow + c0, v);
          uint32_t h[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            float z0 = v[2 * q] + bias[c0 + 2 * q], z1 = v[2 * q + 1] + bias[c0 + 2 * q + 1];
            z0 = z0 / (1.0f + __expf(-z0));
            z1 = z1 / (1.0f + __expf(-z1));
            h[q] = pack_bf16x2(z0, z1);
          }
          uint8_t* base = As + (c0 >> 6) * 16384;
          *reinterpret_cast<uint4*>(base + sw128_offset(tid, c0 & 63)) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4*>(base + sw128_offset(tid, (c0 & 63) + 8)) = make_uint4(h[4], h[5], h[6], h[7]);
        }
        fence_async_smem();
      } else {
        const int64_t j = tile * 128 + tid;
        for (int c0 = 0; c0 < fout; c0 += 16) {
          float v[16];
          tmem_ld16(trow + c0, v);
          if (j < a.n) {
            float4* o = reinterpret_cast<float4*>(a.out + j * fout + c0);
#pragma unroll
            for (int q = 0; q < 4; ++q)
              o[q] = make_float4(v[4 * q] + bias[c0 + 4 * q], v[4 * q + 1] + bias[c0 + 4 * q + 1],
                                 v[4 * q + 2] + bias[c0 + 4 * q + 2], v[4 * q + 3] + bias[c0 + 4 * q + 3]);
          }
        }
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
    if (s_abort) break;
  }
  // wind down: no copy or MMA of this CTA may still be in flight when TMEM and shared memory go away
  if (tid == 0) {
    if (m_pending) {
      long long t0 = clock64();
      while (!mbar_try_wait(mbar, mph) && clock64() - t0 < a.timeout) {
      }
    }
    if (w_pending) {
      long long t0 = clock64();
      while (!mbar_try_wait(wbar, wph) && clock64() - t0 < a.timeout) {
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

// BF16 weight image: layer l, 64-column chunk c of its inputs: fout rows x 128 bytes, element (o, i)
// = W_l[i * fout + o] at sw128_offset(o, i % 64) of chunk i / 64.
__global__ void mlp_pack_tc_kernel(const float* __restrict__ params, int64_t woff_param, int fin, int fout,
                                   uint8_t* __restrict__ img) {
  const int64_t total = (int64_t)fin * fout;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / fout), o = (int)(e % fout);
    const __nv_bfloat16 v = __float2bfloat16_rn(params[woff_param + e]);
    *reinterpret_cast<__nv_bfloat16*>(img + (int64_t)(i >> 6) * fout * 128 + sw128_offset(o, i & 63)) = v;
  }
}

bool mlp_tc_eligible(const epb_mlp* m) {
  if (m->infer_mode != 1 || m->nhidden + 1 > 9) return false;
  for (int l = 0; l <= m->nhidden; ++l) {
    const int fi = m->fan_in[l], fo = m->fan_out[l];
    if (fi % 64 || fi > 256 || fo % 16 || fo > 256) return false;
  }
  return m->nf % 4 == 0;
}

static int mlp_tc_prepare(epb_ctx* ctx, epb_mlp* m) {
  if (!m->tc_dirty && m->tc_image) return EPB_OK;
  int64_t bytes = 0;
  for (int l = 0; l <= m->nhidden; ++l) bytes += (int64_t)m->fan_in[l] * m->fan_out[l] * 2;
  if (!m->tc_image) {
    if (cudaMalloc(&m->tc_image, bytes) != cudaSuccess) {
      cudaGetLastError();
      m->tc_image = nullptr;
      set_error("surrogate: weight image allocation failed");
      return EPB_ERR_OOM;
    }
  }
  int64_t off = 0;
  for (int l = 0; l <= m->nhidden; ++l) {
    const int64_t cnt = (int64_t)m->fan_in[l] * m->fan_out[l];
    mlp_pack_tc_kernel<<<(unsigned)std::min<int64_t>(cdiv(cnt, 256), (int64_t)ctx->sm_count * 8), 256, 0,
                         ctx->stream>>>(m->params, m->w_off[l], m->fan_in[l], m->fan_out[l], m->tc_image + off);
    EPB_LAUNCH_CHECK();
    off += cnt * 2;
  }
  m->tc_dirty = false;
  return EPB_OK;
}

// Normalised predictions (n x nout FP32) of the points (as in mlp_features_kernel) on the tensor cores.
int mlp_predict_tc(epb_ctx* ctx, const epb_mlp* mc, const double* xa, const double* xb, int64_t nb, const int64_t* pidx,
                   int64_t pair0, int64_t n, float* out) {
  if (n == 0) return EPB_OK;
  epb_mlp* m = const_cast<epb_mlp*>(mc);  // the weight image is a cache of the parameters
  EPB_TRY(mlp_tc_prepare(ctx, m));
  static bool attr = false;
  if (!attr) {
    EPB_CUDA(cudaFuncSetAttribute(mlp_infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    attr = true;
  }
  MlpTcArgs a{};
  a.fvec = m->fvec;
  a.nf = m->nf;
  a.xa = xa;
  a.xb = xb;
  a.nb = nb;
  a.pidx = pidx;
  a.pair0 = pair0;
  a.n = n;
  a.wimg = m->tc_image;
  a.params = m->params;
  a.nlayer = m->nhidden + 1;
  int64_t off = 0;
  for (int l = 0; l < a.nlayer; ++l) {
    a.fin[l] = m->fan_in[l];
    a.fout[l] = m->fan_out[l];
    a.woff[l] = off;
    a.boff[l] = m->b_off[l];
    off += (int64_t)m->fan_in[l] * m->fan_out[l] * 2;
  }
  a.out = out;
  a.err = ctx->dstat + 5;
  a.timeout = 4000000000LL;
  const int64_t tiles = cdiv(n, 128);
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)ctx->sm_count);
  mlp_infer_tc_kernel<<<grid, 128, TC_SMEM, ctx->stream>>>(a);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// Read back and clear the surrogate kernel's timeout flag (one sync).
int mlp_tc_check(epb_ctx* ctx) {
  int* h = (int*)ctx->pinned;
  EPB_CUDA(cudaMemcpyAsync(h, ctx->dstat + 5, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(ctx->dstat + 5, 0, sizeof(int), ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*h) {
    set_error("surrogate tensor-core kernel: a bounded wait timed out (kernel wound down)");
    return EPB_ERR_TIMEOUT;
  }
  return EPB_OK;
}

}  // namespace epb
