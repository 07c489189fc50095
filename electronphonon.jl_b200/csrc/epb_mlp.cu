// Learned energy surrogate: an MLP on Fourier features of k, trained and run by this library's own
// kernels, that predicts the band energies E_n(k) of a Wannier Hamiltonian so that k and k+q
// points whose every band lies outside the energy window (filter.jl:19,40-72) by more than the
// calibrated margin are culled before the full interpolation. There is no counterpart in the
// reference; its role is to shrink the set of points that the plain path (Fourier + eigenvalues)
// has to evaluate, without changing the kept set.
//
// Network: phi(k) = [cos 2 pi f.k, sin 2 pi f.k] for nf integer vectors f (nin = 2 nf inputs),
// nhidden hidden layers of width `hidden` with SiLU activation (z * sigmoid(z)), a linear output of
// nout values; the outputs are the normalised energies (E_n - mu_n) / s_n with per-band mean mu_n and
// standard deviation s_n of the training targets.
//
// Parameters (FP32, one flat array): for layer l = 0 .. nhidden, W_l (in_l x out_l, row-major,
// W[i * out + o]) followed by b_l (out_l).
//
// Training: mean-squared error over the batch and the outputs, L = sum (y_pred - y)^2 / (B nout),
// Adam (beta1 0.9, beta2 0.999, eps 1e-8) with a cosine learning-rate schedule from lr to lr_final.
// Each step: gather a batch through a per-epoch bijective shuffle, forward (register-tiled SGEMM with
// fused bias + SiLU epilogue that also stores the pre-activation), loss gradient, backward (weight
// gradients split over the batch into per-split partial sums so that the reduction order is fixed,
// data gradients with the fused SiLU' epilogue), Adam over all parameters. One epoch is captured as
// a CUDA graph and replayed; the step counter, schedule and shuffle keys live on the device.
#include <cmath>
#include <vector>

#include "epb_mlp.cuh"

namespace epb {

constexpr int MLP_SPLITS = 8;  // weight-gradient partial sums per step (over the batch)

// ---- features ----------------------------------------------------------------------------------
// Point j: x = xa[:, a_j] + xb[:, b_j] with (a_j, b_j) = (pair / nb, pair % nb), pair = pidx[j] or
// pair0 + j (xb == null: x = xa[:, j]). Row j of X: [cos 2 pi f.x, sin 2 pi f.x] per vector f, with
// the reduction f.x - rint(f.x) done in FP64.
__global__ void mlp_features_kernel(const int4* __restrict__ fvec, int nf, const double* __restrict__ xa,
                                    const double* __restrict__ xb, int64_t nb, const int64_t* __restrict__ pidx,
                                    int64_t pair0, int64_t n, float* __restrict__ X) {
  const int64_t total = n * nf;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = idx / nf;
    const int f = (int)(idx % nf);
    double x0, x1, x2;
    if (xb) {
      const int64_t p = pidx ? pidx[j] : pair0 + j;
      const int64_t ja = p / nb, jb = p % nb;
      x0 = xa[3 * ja] + xb[3 * jb];
      x1 = xa[3 * ja + 1] + xb[3 * jb + 1];
      x2 = xa[3 * ja + 2] + xb[3 * jb + 2];
    } else {
      x0 = xa[3 * j];
      x1 = xa[3 * j + 1];
      x2 = xa[3 * j + 2];
    }
    const int4 v = fvec[f];
    const double t = rdotx(v.x, v.y, v.z, x0, x1, x2);
    const float r = (float)(t - rint(t));
    float s, c;
    sincospif(2.0f * r, &s, &c);
    reinterpret_cast<float2*>(X)[j * nf + f] = make_float2(c, s);
  }
}

// ---- SGEMM with fused epilogues --------------------------------------------------------------------
// C (M x N, row-major, ldc) = op(A) (M x K) * op(B) (K x N), FP32, 64 x 64 x 16 tiles, 256 threads,
// 4 x 4 outputs per thread. A(m,k) = TA ? A[k lda + m] : A[m lda + k]; B(k,n) = TB ? B[n ldb + k] :
// B[k ldb + n]. M, N, K, lda, ldb, ldc multiples of 4 and 16-byte aligned bases (host-checked).
// blockIdx.z selects a split of K of length kps; EPI_STORE writes split s at C + s c_split.
enum { EPI_STORE = 0, EPI_HIDDEN = 1, EPI_HIDDEN_NOZ = 2, EPI_OUT = 3, EPI_DACT = 4 };

struct SgemmArgs {
  const float* A;
  const float* B;
  float* C;
  const float* bias;
  float* Z;           // EPI_HIDDEN: pre-activation out
  const float* Zp;    // EPI_DACT: pre-activation of the layer below
  int M, N, K, kps;
  int lda, ldb, ldc;
  int64_t c_split;    // EPI_STORE: element offset of split s's output (C + s c_split)
};

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) mlp_sgemm_kernel(SgemmArgs a) {
  __shared__ __align__(16) float As[2][16][68];
  __shared__ __align__(16) float Bs[2][16][68];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const int kb = blockIdx.z * a.kps;
  const int ke = min(a.K, kb + a.kps);
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;

  float4 ra, rb;
  auto load = [&](int k0) {
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!TA) {
      const int m = tid >> 2, kq = (tid & 3) * 4;
      ra = (m0 + m < a.M && k0 + kq < ke) ? *reinterpret_cast<const float4*>(a.A + (int64_t)(m0 + m) * a.lda + k0 + kq)
                                          : z4;
    } else {
      const int k = tid >> 4, mq = (tid & 15) * 4;
      ra = (k0 + k < ke && m0 + mq < a.M) ? *reinterpret_cast<const float4*>(a.A + (int64_t)(k0 + k) * a.lda + m0 + mq)
                                          : z4;
    }
    if (!TB) {
      const int k = tid >> 4, nq = (tid & 15) * 4;
      rb = (k0 + k < ke && n0 + nq < a.N) ? *reinterpret_cast<const float4*>(a.B + (int64_t)(k0 + k) * a.ldb + n0 + nq)
                                          : z4;
    } else {
      const int n = tid >> 2, kq = (tid & 3) * 4;
      rb = (n0 + n < a.N && k0 + kq < ke) ? *reinterpret_cast<const float4*>(a.B + (int64_t)(n0 + n) * a.ldb + k0 + kq)
                                          : z4;
    }
  };
  auto store = [&](int buf) {
    if (!TA) {
      const int m = tid >> 2, kq = (tid & 3) * 4;
      As[buf][kq + 0][m] = ra.x;
      As[buf][kq + 1][m] = ra.y;
      As[buf][kq + 2][m] = ra.z;
      As[buf][kq + 3][m] = ra.w;
    } else {
      const int k = tid >> 4, mq = (tid & 15) * 4;
      *reinterpret_cast<float4*>(&As[buf][k][mq]) = ra;
    }
    if (!TB) {
      const int k = tid >> 4, nq = (tid & 15) * 4;
      *reinterpret_cast<float4*>(&Bs[buf][k][nq]) = rb;
    } else {
      const int n = tid >> 2, kq = (tid & 3) * 4;
      Bs[buf][kq + 0][n] = rb.x;
      Bs[buf][kq + 1][n] = rb.y;
      Bs[buf][kq + 2][n] = rb.z;
      Bs[buf][kq + 3][n] = rb.w;
    }
  };

  int buf = 0;
  if (kb < ke) {
    load(kb);
    store(0);
  }
  __syncthreads();
  for (int k0 = kb; k0 < ke; k0 += 16) {
    const bool more = k0 + 16 < ke;
    if (more) load(k0 + 16);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float4 av = *reinterpret_cast<const float4*>(&As[buf][k][ty * 4]);
      const float4 bv = *reinterpret_cast<const float4*>(&Bs[buf][k][tx * 4]);
      const float ar[4] = {av.x, av.y, av.z, av.w};
      const float br[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(ar[i], br[j], acc[i][j]);
    }
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }

  const int n = n0 + tx * 4;
  if (n >= a.N) return;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= a.M) break;
    float v[4] = {acc[i][0], acc[i][1], acc[i][2], acc[i][3]};
    const int64_t o = (int64_t)m * a.ldc + n;
    if (EPI == EPI_STORE) {
      *reinterpret_cast<float4*>(a.C + (int64_t)blockIdx.z * a.c_split + o) = make_float4(v[0], v[1], v[2], v[3]);
    } else if (EPI == EPI_HIDDEN || EPI == EPI_HIDDEN_NOZ) {
      const float4 b4 = *reinterpret_cast<const float4*>(a.bias + n);
      const float z[4] = {v[0] + b4.x, v[1] + b4.y, v[2] + b4.z, v[3] + b4.w};
      if (EPI == EPI_HIDDEN) *reinterpret_cast<float4*>(a.Z + o) = make_float4(z[0], z[1], z[2], z[3]);
      float h[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) h[j] = z[j] * sigmoidf_(z[j]);
      *reinterpret_cast<float4*>(a.C + o) = make_float4(h[0], h[1], h[2], h[3]);
    } else if (EPI == EPI_OUT) {
      const float4 b4 = *reinterpret_cast<const float4*>(a.bias + n);
      *reinterpret_cast<float4*>(a.C + o) = make_float4(v[0] + b4.x, v[1] + b4.y, v[2] + b4.z, v[3] + b4.w);
    } else {  // EPI_DACT: dX * silu'(Zp)
      const float4 z4 = *reinterpret_cast<const float4*>(a.Zp + o);
      const float z[4] = {z4.x, z4.y, z4.z, z4.w};
      float h[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float s = sigmoidf_(z[j]);
        h[j] = v[j] * (s * (1.0f + z[j] * (1.0f - s)));
      }
      *reinterpret_cast<float4*>(a.C + o) = make_float4(h[0], h[1], h[2], h[3]);
    }
  }
}

// splits > 1 (EPI_STORE only): split s covers K rows [s kps, (s + 1) kps), kps = a.kps if set.
template <bool TA, bool TB, int EPI>
static int sgemm(epb_ctx* ctx, SgemmArgs a, int splits) {
  EPB_CHECK_ARG(a.M % 4 == 0 && a.N % 4 == 0 && a.K % 4 == 0 && a.lda % 4 == 0 && a.ldb % 4 == 0 &&
                    a.ldc % 4 == 0,
                "MLP GEMM: sizes must be multiples of 4 (M=%d N=%d K=%d)", a.M, a.N, a.K);
  if (splits < 1) splits = 1;
  if (a.kps <= 0) a.kps = (int)(cdiv(cdiv(a.K, splits), 16) * 16);
  dim3 grid((unsigned)cdiv(a.N, 64), (unsigned)cdiv(a.M, 64), (unsigned)splits);
  mlp_sgemm_kernel<TA, TB, EPI><<<grid, 256, 0, ctx->stream>>>(a);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

// ---- training kernels ----------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Bijection of [0, n) keyed by (seed, epoch): a keyed permutation of [0, 2^bits) (xor, odd
// multiply, xorshift, twice) with cycle walking back into [0, n).
__device__ __forceinline__ int64_t shuffle_index(int64_t i, int64_t n, int bits, uint64_t seed, int64_t epoch) {
  const uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  const uint64_t k0 = splitmix64(seed ^ (uint64_t)epoch * 0x632BE59BD9B4E019ull);
  const uint64_t k1 = splitmix64(k0), k2 = splitmix64(k1) | 1ull, k3 = splitmix64(k2) | 1ull;
  const int sh = bits / 2 + 1;
  uint64_t x = (uint64_t)i;
  do {
    x = (x ^ k0) & mask;
    x = (x * k2) & mask;
    x ^= x >> sh;
    x = (x ^ k1) & mask;
    x = (x * k3) & mask;
    x ^= x >> sh;
  } while (x >= (uint64_t)n);
  return (int64_t)x;
}

struct TrainShape {
  int64_t n;          // training points
  int B;              // batch
  int64_t spe;        // steps per epoch
  int bits;
  uint64_t seed;
  int nin, nout;
};

// Gather batch `step % spe` of epoch `step / spe` (rows of F and Y through the shuffle).
__global__ void mlp_gather_kernel(TrainShape s, const int64_t* __restrict__ step, const float* __restrict__ F,
                                  const float* __restrict__ Y, float* __restrict__ Xb, float* __restrict__ Yb) {
  const int64_t t = *step;
  const int64_t e = t / s.spe, bi = t % s.spe;
  const int row = blockIdx.x;
  const int64_t src = shuffle_index(bi * s.B + row, s.n, s.bits, s.seed, e);
  const float4* f4 = reinterpret_cast<const float4*>(F + src * s.nin);
  float4* x4 = reinterpret_cast<float4*>(Xb + (int64_t)row * s.nin);
  for (int i = threadIdx.x; i < s.nin / 4; i += blockDim.x) x4[i] = f4[i];
  for (int i = threadIdx.x; i < s.nout; i += blockDim.x) Yb[(int64_t)row * s.nout + i] = Y[src * s.nout + i];
}

// dOut = 2 (out - y) / (B nout); loss sum into loss_acc[epoch] (or loss_acc[0] without a counter).
__global__ void mlp_loss_kernel(const float* __restrict__ out, const float* __restrict__ y, int64_t total,
                                float scale, float* __restrict__ dout, const int64_t* __restrict__ step,
                                int64_t spe, double* __restrict__ loss_acc) {
  double part = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = out[i] - y[i];
    dout[i] = 2.0f * d * scale;
    part += (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    const int64_t e = step ? *step / spe : 0;
    atomicAdd(loss_acc + e, s * scale);
  }
}

// Bias gradient partials: gpart[s][boff + c] = sum over rows of split s of dZ[row, c].
__global__ void mlp_colsum_kernel(const float* __restrict__ dZ, int rows, int cols, int rows_per_split,
                                  float* __restrict__ gpart, int64_t nparam, int64_t boff) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (c >= cols) return;
  const int r0 = s * rows_per_split, r1 = min(rows, r0 + rows_per_split);
  float acc = 0.f;
  for (int r = r0; r < r1; ++r) acc += dZ[(int64_t)r * cols + c];
  gpart[(int64_t)s * nparam + boff + c] = acc;
}

struct AdamArgs {
  float* p;
  float* m;
  float* v;
  const float* gpart;
  int64_t nparam;
  int splits;
  const int64_t* step;
  double lr0, lr1;
  int64_t total_steps;
  float* grad_out;  // gradient-only mode: write the summed gradient, no update
};

__global__ void mlp_adam_kernel(AdamArgs a) {
  double lr = a.lr0;
  int64_t t = 1;
  if (a.step) {
    const int64_t st = *a.step;
    t = st + 1;
    const double f = a.total_steps > 1 ? (double)st / (double)(a.total_steps - 1) : 1.0;
    lr = a.lr1 + 0.5 * (a.lr0 - a.lr1) * (1.0 + cospi(fmin(f, 1.0)));
  }
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = (float)(1.0 / (1.0 - pow(0.9, (double)t)));
  const float c2 = (float)(1.0 / (1.0 - pow(0.999, (double)t)));
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.nparam; i += (int64_t)gridDim.x * blockDim.x) {
    float g = 0.f;
    for (int s = 0; s < a.splits; ++s) g += a.gpart[(int64_t)s * a.nparam + i];
    if (a.grad_out) {
      a.grad_out[i] = g;
      continue;
    }
    const float m = b1 * a.m[i] + (1.f - b1) * g;
    const float v = b2 * a.v[i] + (1.f - b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    a.p[i] -= (float)lr * (m * c1) / (sqrtf(v * c2) + 1e-8f);
  }
}

__global__ void mlp_step_advance_kernel(int64_t* step) { *step += 1; }

// Parameter initialisation: W ~ U(-a, a), a = sqrt(6 / (fan_in + fan_out)); b = 0.
__global__ void mlp_init_kernel(float* __restrict__ p, int64_t off, int64_t count, float amp, uint64_t seed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t r = splitmix64(seed ^ (uint64_t)(off + i) * 0xD1B54A32D192ED03ull);
    const float u = (float)((r >> 40) * (1.0 / 16777216.0));  // [0, 1)
    p[off + i] = amp * (2.f * u - 1.f);
  }
}

// Per-band mean and standard deviation of E (nout x n, double) -> mu, sc (FP32). One block per band.
__global__ void mlp_band_stats_kernel(const double* __restrict__ E, int nout, int64_t n, float* __restrict__ mu,
                                      float* __restrict__ sc) {
  const int b = blockIdx.x;
  double s = 0, s2 = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = E[i * nout + b];
    s += v;
    s2 += v * v;
  }
  __shared__ double r1[32], r2[32];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    r1[threadIdx.x >> 5] = s;
    r2[threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, a2 = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += r1[w];
      a2 += r2[w];
    }
    const double m = a / (double)n;
    const double var = fmax(a2 / (double)n - m * m, 0.0);
    mu[b] = (float)m;
    sc[b] = (float)(var > 0 ? sqrt(var) : 1.0);
  }
}

// Normalised targets Y[i, b] = (E[b, i] - mu_b) / sc_b.
__global__ void mlp_norm_targets_kernel(const double* __restrict__ E, int nout, int64_t n, const float* __restrict__ mu,
                                        const float* __restrict__ sc, float* __restrict__ Y) {
  const int64_t total = n * nout;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(i % nout);
    Y[i] = (float)((E[i] - (double)mu[b]) / (double)sc[b]);
  }
}

// Denormalised predictions E[b, j] = out[j, b] sc_b + mu_b (double).
__global__ void mlp_denorm_kernel(const float* __restrict__ out, int nout, int64_t n, const float* __restrict__ mu,
                                  const float* __restrict__ sc, double* __restrict__ E) {
  const int64_t total = n * nout;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(i % nout);
    E[i] = (double)out[i] * (double)sc[b] + (double)mu[b];
  }
}

// Max |pred - true| per band (non-negative doubles ordered as unsigned 64-bit integers).
__global__ void mlp_maxerr_kernel(const double* __restrict__ P, const double* __restrict__ T, int nout, int64_t n,
                                  unsigned long long* __restrict__ maxerr) {
  const int64_t total = n * nout;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const double d = fabs(P[i] - T[i]);
    atomicMax(maxerr + (i % nout), (unsigned long long)__double_as_longlong(d));
  }
}

static unsigned grid1d(epb_ctx* ctx, int64_t total, int threads = 256) {
  int64_t b = cdiv(total, threads);
  const int64_t cap = (int64_t)ctx->sm_count * 16;
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}

// ---- forward / backward drivers ------------------------------------------------------------------
// Activation buffers of a batch of B rows: X[0] = features (B x nin), X[l] (B x hidden) for
// l = 1..nhidden, Z[l] (B x hidden) pre-activations, out (B x nout), Y, two gradient buffers.
struct MlpBatchBufs {
  std::vector<float*> X, Z;
  float* out = nullptr;
  float* Y = nullptr;
  float* d0 = nullptr;
  float* d1 = nullptr;
  float* gpart = nullptr;
  double* loss = nullptr;
};

static size_t batch_bytes(const epb_mlp* m, int64_t B) {
  const int64_t H = m->hidden;
  size_t f = (size_t)B * m->nin + (size_t)B * H * m->nhidden * 2 + (size_t)B * m->nout * 2 +
             2 * (size_t)B * std::max<int64_t>(H, m->nout) + (size_t)MLP_SPLITS * m->nparam;
  return f * sizeof(float) + 64 * 1024;
}

static void carve(const epb_mlp* m, int64_t B, uint8_t* base, MlpBatchBufs& b) {
  auto take = [&](size_t floats) {
    float* p = (float*)base;
    base += ((floats * sizeof(float) + 255) / 256) * 256;
    return p;
  };
  const int64_t H = m->hidden;
  b.X.assign(m->nhidden + 1, nullptr);
  b.Z.assign(m->nhidden, nullptr);
  b.X[0] = take((size_t)B * m->nin);
  for (int l = 1; l <= m->nhidden; ++l) b.X[l] = take((size_t)B * H);
  for (int l = 0; l < m->nhidden; ++l) b.Z[l] = take((size_t)B * H);
  b.out = take((size_t)B * m->nout);
  b.Y = take((size_t)B * m->nout);
  b.d0 = take((size_t)B * std::max<int64_t>(H, m->nout));
  b.d1 = take((size_t)B * std::max<int64_t>(H, m->nout));
  b.gpart = take((size_t)MLP_SPLITS * m->nparam);
  b.loss = (double*)base;
}

// Forward on B rows of b.X[0]; keep_z stores the pre-activations for the backward pass.
static int mlp_forward(epb_ctx* ctx, const epb_mlp* m, MlpBatchBufs& b, int B, bool keep_z) {
  for (int l = 0; l <= m->nhidden; ++l) {
    SgemmArgs g{};
    g.A = b.X[l];
    g.lda = m->fan_in[l];
    g.B = m->params + m->w_off[l];
    g.ldb = m->fan_out[l];
    g.bias = m->params + m->b_off[l];
    g.M = B;
    g.N = m->fan_out[l];
    g.K = m->fan_in[l];
    g.ldc = m->fan_out[l];
    if (l < m->nhidden) {
      g.C = b.X[l + 1];
      g.Z = b.Z[l];
      if (keep_z)
        EPB_TRY((sgemm<false, false, EPI_HIDDEN>(ctx, g, 1)));
      else
        EPB_TRY((sgemm<false, false, EPI_HIDDEN_NOZ>(ctx, g, 1)));
    } else {
      g.C = b.out;
      EPB_TRY((sgemm<false, false, EPI_OUT>(ctx, g, 1)));
    }
  }
  return EPB_OK;
}

// Loss gradient and backward pass into b.gpart (MLP_SPLITS partial sums per parameter).
static int mlp_backward(epb_ctx* ctx, const epb_mlp* m, MlpBatchBufs& b, int B, const int64_t* step, int64_t spe,
                        double* loss_acc) {
  const int64_t tot = (int64_t)B * m->nout;
  mlp_loss_kernel<<<grid1d(ctx, tot), 256, 0, ctx->stream>>>(b.out, b.Y, tot, 1.0f / (float)tot, b.d0, step, spe,
                                                              loss_acc);
  EPB_LAUNCH_CHECK();
  const int rps = (int)cdiv(cdiv(B, MLP_SPLITS), 16) * 16;
  float* dz = b.d0;  // gradient w.r.t. the output of layer l (pre-activation for hidden layers)
  float* other = b.d1;
  for (int l = m->nhidden; l >= 0; --l) {
    const int fin = m->fan_in[l], fout = m->fan_out[l];
    // dW_l = X_l^T dZ_l, split over the batch
    SgemmArgs g{};
    g.A = b.X[l];
    g.lda = fin;
    g.B = dz;
    g.ldb = fout;
    g.C = b.gpart + m->w_off[l];
    g.ldc = fout;
    g.M = fin;
    g.N = fout;
    g.K = B;
    g.kps = rps;
    g.c_split = m->nparam;
    EPB_TRY((sgemm<true, false, EPI_STORE>(ctx, g, MLP_SPLITS)));
    // db_l
    mlp_colsum_kernel<<<dim3((unsigned)cdiv(fout, 128), MLP_SPLITS), 128, 0, ctx->stream>>>(
        dz, B, fout, rps, b.gpart, m->nparam, m->b_off[l]);
    EPB_LAUNCH_CHECK();
    if (l == 0) break;
    // dZ_{l-1} = (dZ_l W_l^T) * silu'(Z_{l-1})
    SgemmArgs d{};
    d.A = dz;
    d.lda = fout;
    d.B = m->params + m->w_off[l];
    d.ldb = fout;
    d.C = other;
    d.ldc = fin;
    d.Zp = b.Z[l - 1];
    d.M = B;
    d.N = fin;
    d.K = fout;
    EPB_TRY((sgemm<false, true, EPI_DACT>(ctx, d, 1)));
    std::swap(dz, other);
  }
  return EPB_OK;
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_mlp_create(epb_ctx* ctx, const int32_t* fvec_host, int64_t nf, int64_t hidden, int64_t nhidden,
                   int64_t nout, uint64_t seed, epb_mlp** out) {
  clear_error();
  EPB_CHECK_ARG(ctx && fvec_host && out, "epb_mlp_create: NULL argument");
  EPB_CHECK_ARG(nf >= 2 && nf <= 4096 && (2 * nf) % 4 == 0, "epb_mlp_create: nf=%lld must be even, 2..4096",
                (long long)nf);
  EPB_CHECK_ARG(hidden >= 4 && hidden <= 4096 && hidden % 4 == 0, "epb_mlp_create: hidden=%lld must be a multiple of 4",
                (long long)hidden);
  EPB_CHECK_ARG(nhidden >= 1 && nhidden <= 8, "epb_mlp_create: nhidden=%lld outside 1..8", (long long)nhidden);
  EPB_CHECK_ARG(nout >= 4 && nout <= 256 && nout % 4 == 0, "epb_mlp_create: nout=%lld must be a multiple of 4",
                (long long)nout);
  EPB_TRY(make_current(ctx));
  epb_mlp* m = new epb_mlp();
  m->ctx = ctx;
  m->nf = (int)nf;
  m->nin = (int)(2 * nf);
  m->hidden = (int)hidden;
  m->nhidden = (int)nhidden;
  m->nout = (int)nout;
  int64_t off = 0;
  for (int l = 0; l <= m->nhidden; ++l) {
    const int fin = l == 0 ? m->nin : m->hidden;
    const int fout = l == m->nhidden ? m->nout : m->hidden;
    m->fan_in.push_back(fin);
    m->fan_out.push_back(fout);
    m->w_off.push_back(off);
    off += (int64_t)fin * fout;
    m->b_off.push_back(off);
    off += fout;
    off = (off + 3) & ~int64_t(3);  // keep every block 16-byte aligned
  }
  m->nparam = off;
  std::vector<int4> fv(nf);
  for (int64_t i = 0; i < nf; ++i) fv[i] = make_int4(fvec_host[3 * i], fvec_host[3 * i + 1], fvec_host[3 * i + 2], 0);
  auto fail = [&](const char* what) {
    cudaGetLastError();
    cudaFree(m->fvec);
    cudaFree(m->params);
    cudaFree(m->step);
    delete m;
    set_error("epb_mlp_create: %s", what);
    return EPB_ERR_OOM;
  };
  const size_t pb = (size_t)m->nparam * sizeof(float);
  if (cudaMalloc(&m->fvec, nf * sizeof(int4)) != cudaSuccess) return fail("allocation failed");
  // params | adam m | adam v | mu | sc | margin
  if (cudaMalloc(&m->params, 3 * pb + 2 * 256 * sizeof(float) + 256 * sizeof(double) + 1024) != cudaSuccess)
    return fail("allocation failed");
  m->adam_m = m->params + m->nparam;
  m->adam_v = m->adam_m + m->nparam;
  m->y_mu = m->adam_v + m->nparam;
  m->y_sc = m->y_mu + 256;
  m->margin = (double*)(((uintptr_t)(m->y_sc + 256) + 15) & ~uintptr_t(15));
  if (cudaMalloc(&m->step, 64) != cudaSuccess) return fail("allocation failed");
  EPB_CUDA(cudaMemcpyAsync(m->fvec, fv.data(), nf * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(m->params, 0, 3 * pb, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(m->step, 0, 64, ctx->stream));
  std::vector<float> one(256, 1.0f);
  EPB_CUDA(cudaMemsetAsync(m->y_mu, 0, 256 * sizeof(float), ctx->stream));
  EPB_CUDA(cudaMemcpyAsync(m->y_sc, one.data(), 256 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(m->margin, 0, 256 * sizeof(double), ctx->stream));
  for (int l = 0; l <= m->nhidden; ++l) {
    const float amp = (float)std::sqrt(6.0 / (double)(m->fan_in[l] + m->fan_out[l]));
    const int64_t cnt = (int64_t)m->fan_in[l] * m->fan_out[l];
    mlp_init_kernel<<<grid1d(ctx, cnt), 256, 0, ctx->stream>>>(m->params, m->w_off[l], cnt, amp, seed);
    EPB_LAUNCH_CHECK();
  }
  m->margin_host.assign(nout, 0.0);
  m->tc_dirty = true;
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  *out = m;
  return EPB_OK;
}

int epb_mlp_destroy(epb_mlp* m) {
  if (!m) return EPB_OK;
  cudaFree(m->fvec);
  cudaFree(m->params);
  cudaFree(m->step);
  cudaFree(m->loss_acc);
  cudaFree(m->tc_image);
  delete m;
  return EPB_OK;
}

int epb_mlp_info(const epb_mlp* m, int64_t* nparam, int64_t* nin, int64_t* nout) {
  clear_error();
  EPB_CHECK_ARG(m, "epb_mlp_info: NULL model");
  if (nparam) *nparam = m->nparam;
  if (nin) *nin = m->nin;
  if (nout) *nout = m->nout;
  return EPB_OK;
}

int epb_mlp_get_params(epb_ctx* ctx, const epb_mlp* m, float* dst) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && dst, "epb_mlp_get_params: NULL argument");
  EPB_TRY(make_current(ctx));
  EPB_CUDA(cudaMemcpyAsync(dst, m->params, m->nparam * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  return EPB_OK;
}

int epb_mlp_set_params(epb_ctx* ctx, epb_mlp* m, const float* src) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && src, "epb_mlp_set_params: NULL argument");
  EPB_TRY(make_current(ctx));
  EPB_CUDA(cudaMemcpyAsync(m->params, src, m->nparam * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  m->calibrated = false;
  m->tc_dirty = true;
  return EPB_OK;
}

int epb_mlp_set_scaling(epb_ctx* ctx, epb_mlp* m, const double* mu_host, const double* sc_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && mu_host && sc_host, "epb_mlp_set_scaling: NULL argument");
  EPB_TRY(make_current(ctx));
  std::vector<float> mu(m->nout), sc(m->nout);
  for (int i = 0; i < m->nout; ++i) {
    EPB_CHECK_ARG(sc_host[i] > 0, "epb_mlp_set_scaling: scale %d must be positive", i);
    mu[i] = (float)mu_host[i];
    sc[i] = (float)sc_host[i];
  }
  EPB_CUDA(cudaMemcpyAsync(m->y_mu, mu.data(), m->nout * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  EPB_CUDA(cudaMemcpyAsync(m->y_sc, sc.data(), m->nout * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  m->scaled = true;
  m->calibrated = false;
  return EPB_OK;
}

int epb_mlp_get_scaling(epb_ctx* ctx, const epb_mlp* m, double* mu_host, double* sc_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && mu_host && sc_host, "epb_mlp_get_scaling: NULL argument");
  EPB_TRY(make_current(ctx));
  std::vector<float> mu(m->nout), sc(m->nout);
  EPB_CUDA(cudaMemcpyAsync(mu.data(), m->y_mu, m->nout * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaMemcpyAsync(sc.data(), m->y_sc, m->nout * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < m->nout; ++i) {
    mu_host[i] = mu[i];
    sc_host[i] = sc[i];
  }
  return EPB_OK;
}

int epb_mlp_features(epb_ctx* ctx, const epb_mlp* m, const double* x, int64_t n, float* feat) {
  clear_error();
  EPB_CHECK_ARG(ctx && m, "epb_mlp_features: NULL argument");
  EPB_CHECK_ARG(n >= 0 && (n == 0 || (x && feat)), "epb_mlp_features: bad arguments");
  if (n == 0) return EPB_OK;
  EPB_TRY(make_current(ctx));
  mlp_features_kernel<<<grid1d(ctx, n * m->nf), 256, 0, ctx->stream>>>(m->fvec, m->nf, x, nullptr, 1, nullptr, 0, n,
                                                                        feat);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_mlp_loss_grad(epb_ctx* ctx, epb_mlp* m, const double* x, const double* E, int64_t n, float* grad,
                      double* loss_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && x && E && grad, "epb_mlp_loss_grad: NULL argument");
  EPB_CHECK_ARG(n >= 4 && n <= 65536 && n % 4 == 0, "epb_mlp_loss_grad: n=%lld must be a multiple of 4 in 4..65536",
                (long long)n);
  EPB_TRY(make_current(ctx));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_MLP, batch_bytes(m, n), &ws));
  MlpBatchBufs b;
  carve(m, n, (uint8_t*)ws, b);
  prof_begin(ctx, EPB_PROF_MLP_TRAIN);
  mlp_features_kernel<<<grid1d(ctx, n * m->nf), 256, 0, ctx->stream>>>(m->fvec, m->nf, x, nullptr, 1, nullptr, 0, n,
                                                                        b.X[0]);
  EPB_LAUNCH_CHECK();
  mlp_norm_targets_kernel<<<grid1d(ctx, n * m->nout), 256, 0, ctx->stream>>>(E, m->nout, n, m->y_mu, m->y_sc, b.Y);
  EPB_LAUNCH_CHECK();
  EPB_CUDA(cudaMemsetAsync(b.loss, 0, sizeof(double), ctx->stream));
  EPB_TRY(mlp_forward(ctx, m, b, (int)n, true));
  EPB_TRY(mlp_backward(ctx, m, b, (int)n, nullptr, 1, b.loss));
  AdamArgs ad{};
  ad.gpart = b.gpart;
  ad.nparam = m->nparam;
  ad.splits = MLP_SPLITS;
  ad.grad_out = grad;
  mlp_adam_kernel<<<grid1d(ctx, m->nparam), 256, 0, ctx->stream>>>(ad);
  EPB_LAUNCH_CHECK();
  prof_end(ctx);
  if (loss_host) {
    EPB_CUDA(cudaMemcpyAsync(ctx->pinned, b.loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EPB_CUDA(cudaStreamSynchronize(ctx->stream));
    *loss_host = *(double*)ctx->pinned;
  }
  return EPB_OK;
}

int epb_mlp_train(epb_ctx* ctx, epb_mlp* m, const double* x, const double* E, int64_t n,
                  const epb_mlp_train_opts* opts, double* loss_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && x && E && opts, "epb_mlp_train: NULL argument");
  const int64_t B = opts->batch;
  EPB_CHECK_ARG(B >= 16 && B <= 65536 && B % 16 == 0, "epb_mlp_train: batch=%lld must be a multiple of 16 in 16..65536",
                (long long)B);
  EPB_CHECK_ARG(n >= B, "epb_mlp_train: n=%lld smaller than the batch", (long long)n);
  EPB_CHECK_ARG(opts->epochs >= 1 && opts->lr > 0 && opts->lr_final >= 0, "epb_mlp_train: bad schedule");
  EPB_TRY(make_current(ctx));
  const int64_t spe = n / B;
  const int64_t total = spe * opts->epochs;
  // workspace: batch buffers | all features (n x nin) | all normalised targets (n x nout)
  const size_t bb = batch_bytes(m, B);
  const size_t fb = ((size_t)n * m->nin * sizeof(float) + 255) & ~size_t(255);
  const size_t yb = ((size_t)n * m->nout * sizeof(float) + 255) & ~size_t(255);
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_MLP, bb + fb + yb, &ws));
  MlpBatchBufs b;
  carve(m, B, (uint8_t*)ws, b);
  float* Fall = (float*)((uint8_t*)ws + bb);
  float* Yall = (float*)((uint8_t*)ws + bb + fb);
  if (m->loss_cap < opts->epochs) {
    cudaFree(m->loss_acc);
    m->loss_acc = nullptr;
    if (cudaMalloc(&m->loss_acc, opts->epochs * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      m->loss_cap = 0;
      set_error("epb_mlp_train: loss buffer allocation failed");
      return EPB_ERR_OOM;
    }
    m->loss_cap = opts->epochs;
  }
  prof_begin(ctx, EPB_PROF_MLP_TRAIN);
  // target normalisation from the training set, features of every training point once
  mlp_band_stats_kernel<<<m->nout, 256, 0, ctx->stream>>>(E, m->nout, n, m->y_mu, m->y_sc);
  EPB_LAUNCH_CHECK();
  mlp_norm_targets_kernel<<<grid1d(ctx, n * m->nout), 256, 0, ctx->stream>>>(E, m->nout, n, m->y_mu, m->y_sc, Yall);
  EPB_LAUNCH_CHECK();
  mlp_features_kernel<<<grid1d(ctx, n * m->nf), 256, 0, ctx->stream>>>(m->fvec, m->nf, x, nullptr, 1, nullptr, 0, n,
                                                                        Fall);
  EPB_LAUNCH_CHECK();
  EPB_CUDA(cudaMemsetAsync(m->step, 0, sizeof(int64_t), ctx->stream));
  EPB_CUDA(cudaMemsetAsync(m->loss_acc, 0, opts->epochs * sizeof(double), ctx->stream));
  EPB_CUDA(cudaMemsetAsync(m->adam_m, 0, 2 * m->nparam * sizeof(float), ctx->stream));
  m->scaled = true;
  m->calibrated = false;
  m->tc_dirty = true;

  TrainShape ts{};
  ts.n = n;
  ts.B = (int)B;
  ts.spe = spe;
  ts.bits = 1;
  while ((int64_t(1) << ts.bits) < n) ++ts.bits;
  ts.seed = opts->seed;
  ts.nin = m->nin;
  ts.nout = m->nout;
  AdamArgs ad{};
  ad.p = m->params;
  ad.m = m->adam_m;
  ad.v = m->adam_v;
  ad.gpart = b.gpart;
  ad.nparam = m->nparam;
  ad.splits = MLP_SPLITS;
  ad.step = m->step;
  ad.lr0 = opts->lr;
  ad.lr1 = opts->lr_final;
  ad.total_steps = total;

  const int64_t launches0 = ctx->launches;
  auto one_step = [&]() -> int {
    mlp_gather_kernel<<<(unsigned)B, 64, 0, ctx->stream>>>(ts, m->step, Fall, Yall, b.X[0], b.Y);
    EPB_LAUNCH_CHECK();
    EPB_TRY(mlp_forward(ctx, m, b, (int)B, true));
    EPB_TRY(mlp_backward(ctx, m, b, (int)B, m->step, spe, m->loss_acc));
    mlp_adam_kernel<<<grid1d(ctx, m->nparam), 256, 0, ctx->stream>>>(ad);
    EPB_LAUNCH_CHECK();
    mlp_step_advance_kernel<<<1, 1, 0, ctx->stream>>>(m->step);
    EPB_LAUNCH_CHECK();
    return EPB_OK;
  };

  if (opts->use_graph) {
    // Capture one epoch and replay it `epochs` times. The legacy default stream cannot be captured:
    // then the graph runs on a private stream ordered after (and before) the context stream.
    cudaStream_t user = ctx->stream, cap = ctx->stream;
    const bool own = user == nullptr || user == cudaStreamLegacy;
    cudaEvent_t ev = nullptr;
    if (own) {
      EPB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      EPB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      EPB_CUDA(cudaEventRecord(ev, user));
      EPB_CUDA(cudaStreamWaitEvent(cap, ev, 0));
    }
    ctx->stream = cap;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int st = EPB_OK;
    cudaError_t ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      for (int64_t s = 0; s < spe && st == EPB_OK; ++s) st = one_step();
      ce = cudaStreamEndCapture(cap, &graph);
    }
    const int64_t per_epoch = ctx->launches - launches0;
    if (st == EPB_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    for (int64_t e = 0; st == EPB_OK && ce == cudaSuccess && e < opts->epochs; ++e) ce = cudaGraphLaunch(exec, cap);
    if (exec) cudaGraphExecDestroy(exec);
    ctx->launches = launches0 + (st == EPB_OK && ce == cudaSuccess ? per_epoch * opts->epochs : 0);
    ctx->stream = user;
    if (own) {
      cudaEventRecord(ev, cap);
      cudaStreamWaitEvent(user, ev, 0);
      cudaEventDestroy(ev);
      cudaStreamDestroy(cap);
    }
    if (st != EPB_OK) return st;
    if (ce != cudaSuccess) {
      cudaGetLastError();
      set_error("epb_mlp_train: CUDA graph capture/launch failed: %s", cudaGetErrorString(ce));
      return EPB_ERR_CUDA;
    }
  } else {
    for (int64_t t = 0; t < total; ++t) EPB_TRY(one_step());
  }
  prof_end(ctx);
  if (loss_host) {
    std::vector<double> l(opts->epochs);
    EPB_CUDA(cudaMemcpyAsync(l.data(), m->loss_acc, opts->epochs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EPB_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int64_t e = 0; e < opts->epochs; ++e) loss_host[e] = l[e] / (double)spe;  // mean batch loss
  } else {
    EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return EPB_OK;
}

}  // extern "C"

namespace epb {

// Normalised predictions of the n points given as coordinates (xb == null) or as pairs xa + xb
// (pair indices pidx, or pair0 + j): out (n x nout, FP32) in a caller buffer. Chunked internally.
bool mlp_tc_eligible(const epb_mlp* m);
int mlp_predict_tc(epb_ctx* ctx, const epb_mlp* m, const double* xa, const double* xb, int64_t nb, const int64_t* pidx,
                   int64_t pair0, int64_t n, float* out);
int mlp_tc_check(epb_ctx* ctx);

// The inference path of the model (tensor cores when eligible and selected, else the FP32 kernels);
// calibration and screening both go through here, so the margins match the path that screens.
int mlp_predict_norm(epb_ctx* ctx, const epb_mlp* m, const double* xa, const double* xb, int64_t nb,
                     const int64_t* pidx, int64_t pair0, int64_t n, float* out_all) {
  if (n == 0) return EPB_OK;
  if (mlp_tc_eligible(m)) return mlp_predict_tc(ctx, m, xa, xb, nb, pidx, pair0, n, out_all);
  const int64_t CH = 32768;
  void* ws = nullptr;
  const int64_t rows = std::min<int64_t>(cdiv(n, 4) * 4, CH);
  EPB_TRY(ws_get(ctx, EPB_WS_MLP, batch_bytes(m, rows), &ws));
  MlpBatchBufs b;
  carve(m, rows, (uint8_t*)ws, b);
  for (int64_t c0 = 0; c0 < n; c0 += CH) {
    const int64_t cn = std::min(CH, n - c0);
    const int64_t cr = cdiv(cn, 4) * 4;
    mlp_features_kernel<<<grid1d(ctx, cn * m->nf), 256, 0, ctx->stream>>>(
        m->fvec, m->nf, xb ? xa : xa + 3 * c0, xb, nb, pidx ? pidx + c0 : nullptr, pair0 + c0, cn, b.X[0]);
    EPB_LAUNCH_CHECK();
    if (cr > cn) EPB_CUDA(cudaMemsetAsync(b.X[0] + cn * m->nin, 0, (cr - cn) * m->nin * sizeof(float), ctx->stream));
    MlpBatchBufs bc = b;
    bc.out = out_all + c0 * m->nout;
    if (cr > cn) bc.out = b.out;  // ragged tail: compute into scratch, copy the valid rows
    EPB_TRY(mlp_forward(ctx, m, bc, (int)cr, false));
    if (cr > cn)
      EPB_CUDA(cudaMemcpyAsync(out_all + c0 * m->nout, b.out, cn * m->nout * sizeof(float), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  }
  return EPB_OK;
}

int mlp_screen_params(const epb_mlp* m, const float** mu, const float** sc, const double** margin, int* nout,
                      bool* calibrated) {
  *mu = m->y_mu;
  *sc = m->y_sc;
  *margin = m->margin;
  *nout = m->nout;
  *calibrated = m->calibrated;
  return EPB_OK;
}

}  // namespace epb

extern "C" {

int epb_mlp_predict(epb_ctx* ctx, const epb_mlp* m, const double* x, int64_t n, double* E) {
  clear_error();
  EPB_CHECK_ARG(ctx && m, "epb_mlp_predict: NULL argument");
  EPB_CHECK_ARG(n >= 0 && (n == 0 || (x && E)), "epb_mlp_predict: bad arguments");
  if (n == 0) return EPB_OK;
  EPB_TRY(make_current(ctx));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_MLP_OUT, (size_t)n * m->nout * sizeof(float) + 256, &ws));
  float* out = (float*)ws;
  prof_begin(ctx, EPB_PROF_MLP_INFER);
  EPB_TRY(mlp_predict_norm(ctx, m, x, nullptr, 1, nullptr, 0, n, out));
  mlp_denorm_kernel<<<grid1d(ctx, n * m->nout), 256, 0, ctx->stream>>>(out, m->nout, n, m->y_mu, m->y_sc, E);
  EPB_LAUNCH_CHECK();
  prof_end(ctx);
  return mlp_tc_eligible(m) ? mlp_tc_check(ctx) : EPB_OK;
}

int epb_mlp_set_inference(epb_mlp* m, int mode) {
  clear_error();
  EPB_CHECK_ARG(m && (mode == 0 || mode == 1), "epb_mlp_set_inference: mode must be 0 (FP32) or 1 (BF16 tensor cores)");
  if (m->infer_mode != mode) m->calibrated = false;  // margins belong to the path that was calibrated
  m->infer_mode = mode;
  return EPB_OK;
}

int epb_mlp_inference_path(const epb_mlp* m, int* path_host) {
  clear_error();
  EPB_CHECK_ARG(m && path_host, "epb_mlp_inference_path: NULL argument");
  *path_host = mlp_tc_eligible(m) ? 1 : 0;
  return EPB_OK;
}

int epb_mlp_calibrate(epb_ctx* ctx, epb_mlp* m, const double* x, const double* E, int64_t n, double safety,
                      double* margin_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && x && E, "epb_mlp_calibrate: NULL argument");
  EPB_CHECK_ARG(n >= 1, "epb_mlp_calibrate: empty held-out set");
  EPB_CHECK_ARG(safety >= 1.0, "epb_mlp_calibrate: safety factor %g < 1", safety);
  EPB_TRY(make_current(ctx));
  void* ws = nullptr;
  const size_t pb = ((size_t)n * m->nout * sizeof(double) + 255) & ~size_t(255);
  EPB_TRY(ws_get(ctx, EPB_WS_MLP_CAL, pb + 256 * sizeof(double), &ws));
  double* P = (double*)ws;
  unsigned long long* mx = (unsigned long long*)((uint8_t*)ws + pb);
  EPB_TRY(epb_mlp_predict(ctx, m, x, n, P));
  EPB_CUDA(cudaMemsetAsync(mx, 0, m->nout * sizeof(double), ctx->stream));
  mlp_maxerr_kernel<<<grid1d(ctx, n * m->nout), 256, 0, ctx->stream>>>(P, E, m->nout, n, mx);
  EPB_LAUNCH_CHECK();
  std::vector<double> h(m->nout);
  EPB_CUDA(cudaMemcpyAsync(h.data(), mx, m->nout * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < m->nout; ++i) {
    EPB_CHECK_ARG(std::isfinite(h[i]), "epb_mlp_calibrate: non-finite error on band %d", i);
    m->margin_host[i] = safety * h[i];
  }
  EPB_CUDA(cudaMemcpyAsync(m->margin, m->margin_host.data(), m->nout * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  m->calibrated = true;
  if (margin_host)
    for (int i = 0; i < m->nout; ++i) margin_host[i] = m->margin_host[i];
  return EPB_OK;
}

}  // extern "C"
