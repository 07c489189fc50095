// Shared infrastructure of the epb200 library: context, workspace, error reporting, complex math.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "epb200.h"

namespace epb {

// ---- error reporting ------------------------------------------------------------------------
void set_error(const char* fmt, ...);
void clear_error();

#define EPB_CHECK_ARG(cond, ...)          \
  do {                                    \
    if (!(cond)) {                        \
      ::epb::set_error(__VA_ARGS__);      \
      return EPB_ERR_ARG;                 \
    }                                     \
  } while (0)

#define EPB_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess) {                                                                \
      ::epb::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__,   \
                       __LINE__);                                                           \
      return EPB_ERR_CUDA;                                                                  \
    }                                                                                       \
  } while (0)

#define EPB_LAUNCH_CHECK()                                                                    \
  do {                                                                                        \
    ++ctx->launches;                                                                          \
    cudaError_t _e = cudaGetLastError();                                                      \
    if (_e != cudaSuccess) {                                                                  \
      ::epb::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(_e), __FILE__, \
                       __LINE__);                                                             \
      return EPB_ERR_CUDA;                                                                    \
    }                                                                                         \
  } while (0)

#define EPB_TRY(call)            \
  do {                           \
    int _s = (call);             \
    if (_s != EPB_OK) return _s; \
  } while (0)

}  // namespace epb

// ---- context --------------------------------------------------------------------------------
// Workspace slots: each entry point uses named slots so that nested calls do not alias.
enum epb_slot {
  EPB_WS_FOURIER = 0,
  EPB_WS_EIGH,
  EPB_WS_EPH_G,
  EPB_WS_EPH_T,
  EPB_WS_FLAGS,
  EPB_WS_SPLIT_A,
  EPB_WS_SPLIT_B,
  EPB_WS_PASS0,
  EPB_WS_PASS1,
  EPB_WS_PASS2,
  EPB_WS_PASS3,
  EPB_WS_PASS4,
  EPB_WS_PASS5,
  EPB_WS_PASS6,
  EPB_WS_PASS7,
  EPB_WS_MLP,
  EPB_WS_EIGH_BIG,
  EPB_WS_MLP_OUT,
  EPB_WS_MLP_CAL,
  EPB_WS_PAIR0,
  EPB_WS_PAIR1,
  EPB_WS_PAIR2,
  EPB_WS_PAIR3,
  EPB_WS_OQ0,  // outer-q loop: k and q states (whole run)
  EPB_WS_OQ1,  // outer-q loop: g(Re, q) of a q chunk
  EPB_WS_OQ2,  // outer-q loop: per k batch
  EPB_WS_NSLOTS
};

// Kernel families timed by the optional profiler (epb_profile_*).
enum epb_prof_id {
  EPB_PROF_FOURIER_F64 = 0,
  EPB_PROF_ZGEMM,
  EPB_PROF_EIGH,
  EPB_PROF_ROT,
  EPB_PROF_RR_ROT,
  EPB_PROF_UMMA_H,
  EPB_PROF_UMMA_KQ,
  EPB_PROF_UMMA_RR,
  EPB_PROF_SPLIT,
  EPB_PROF_OTHER,
  EPB_PROF_REFINE,
  EPB_PROF_TRIDIAG,
  EPB_PROF_MLP_TRAIN,
  EPB_PROF_MLP_INFER,
  EPB_PROF_PAIRS,
  EPB_PROF_N
};

struct epb_prof_rec {
  cudaEvent_t a, b;
  int id;
};

struct epb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  void* ws[EPB_WS_NSLOTS] = {};
  size_t ws_bytes[EPB_WS_NSLOTS] = {};
  int fail_alloc_nth = 0;  // test hook
  // Small pinned host scratch for scalar read-backs.
  int64_t* pinned = nullptr;
  // Device status words: [0] eigensolver non-convergence count, [1] eigensolver bad order count,
  // [2] tensor-core GEMM timeout flag, [3] iq-hash miss count.
  int* dstat = nullptr;
  // instrumentation
  int64_t launches = 0;          // kernels launched by the library on this context
  bool prof_on = false;
  std::vector<epb_prof_rec> prof;  // event pairs recorded while profiling
  size_t prof_used = 0;
  double prof_ms[EPB_PROF_N] = {};
  bool graph_mode = false;  // epb_eph_pass: capture and replay as a CUDA graph (epb_set_graph_mode)
  // autotuner results: shape key -> chosen parameter (epb_tune.cu lists the keys)
  std::vector<std::pair<std::string, int64_t>> tuned;
  int64_t prof_cnt[EPB_PROF_N] = {};
  // side stream of the mixed pass (the kR->kq GEMM runs beside the eigensolvers) and its events,
  // created on first use
  cudaStream_t side = nullptr;
  cudaEvent_t side_ev[5] = {};
  // the mixed pass's inner-batch pipeline (nw = 16, nm = 12): a second stream for the FP64 refinement and
  // the rotation of batch i while the caller's stream runs the H(k+q) GEMM and FP32 Jacobi of batch i + 1,
  // and its events (per buffer parity: H GEMM, Jacobi, kR->kq, refinement, rotation done), made on first use
  cudaStream_t tail = nullptr;
  cudaEvent_t pipe_ev[10] = {};
  // rotation kernel of the mixed pass for nw = 16, nm = 12: 0 = warp tensor cores (mma.sync),
  // 1 = FP32 CUDA cores; -1 = the tuning table's choice (timed when epb_eph_pass autotunes), else 0
  int rot_variant = -1;
  // the choices of the pass in progress (set by epb_eph_pass): rotation kernel, A-resident kR->kq GEMM
  int cur_rot = 0, cur_kq_ares = 1;
  // cuBLAS handle of the plain FP64 pass (its GEMMs are library ZGEMMs, as in the reference's GPU path),
  // created on first use
  void* cublas = nullptr;
};

struct epb_rset {
  epb_ctx* ctx = nullptr;
  int64_t nr = 0;
  int4* dev = nullptr;       // (R1, R2, R3, 0) per vector
  int lo[3] = {0, 0, 0};     // per-axis min
  int hi[3] = {0, 0, 0};     // per-axis max
  std::vector<int64_t> host;  // 3 x nr
};

// A model's hot-path operators (caller-owned device memory) plus the library's derived data.
// Arguments a captured pass was recorded with (a replay is valid only for the same buffers and sizes).
struct PassKey {
  const void* xk = nullptr;
  int64_t nk = 0;
  const void* xq = nullptr;
  int64_t nq = 0;
  int prec = -1;
  int64_t k_batch = 0, stride = 0;
  const void *ek = nullptr, *om = nullptr, *g2 = nullptr, *samp = nullptr;
  int rot = 0, kq = 1;  // rotation kernel and kR->kq form the graph was captured with
  bool operator==(const PassKey& o) const {
    return xk == o.xk && nk == o.nk && xq == o.xq && nq == o.nq && prec == o.prec && k_batch == o.k_batch &&
           stride == o.stride && ek == o.ek && om == o.om && g2 == o.g2 && samp == o.samp && rot == o.rot && kq == o.kq;
  }
};
struct PassGraph {
  PassKey key;
  bool warm = false;                 // one eager run with `key` has sized the workspaces
  cudaGraphExec_t exec = nullptr;    // the captured pass for `key`
  int64_t launches = 0;              // kernels in the graph
};

struct epb_model {
  epb_ctx* ctx = nullptr;
  int64_t nw = 0, nm = 0, nr_el = 0, nr_ph = 0, nr_ep = 0;
  const double2* ham = nullptr;   // (nw^2, nr_el)
  const double2* dyn = nullptr;   // (nm^2, nr_ph)
  const double* mass = nullptr;   // (nm)
  const double2* epmat = nullptr; // (nw^2 nm nr_ep, nr_el)
  epb_rset* rs_el = nullptr;
  epb_rset* rs_ph = nullptr;
  epb_rset* rs_ep = nullptr;
  // mixed-precision operand planes (owned), see epb_umma.cu
  void* mixed = nullptr;
  PassGraph graph;  // graph mode of epb_eph_pass
  double2* epmat_ph = nullptr;  // owned "ph"-layout copy of epmat (outer-q loop), made on first use
  uint8_t* epmat_ph_planes = nullptr;  // owned split-BF16 planes of epmat_ph (mixed outer-q loop)
};

namespace epb {

// Profiler brackets around a launch (no-ops unless epb_profile_enable was called).
void prof_begin(epb_ctx* ctx, int id);
int side_stream(epb_ctx* ctx);
int pipe_streams(epb_ctx* ctx);
void cublas_release(epb_ctx* ctx);
void prof_end(epb_ctx* ctx);

// Grow-only workspace slot; returns EPB_ERR_OOM on failure.
int ws_get(epb_ctx* ctx, int slot, size_t bytes, void** out);
int make_current(epb_ctx* ctx);

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ---- complex helpers (double2 / float2) -----------------------------------------------------
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// acc += a * b
__host__ __device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__host__ __device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__host__ __device__ __forceinline__ void cfma_conj(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
__host__ __device__ __forceinline__ void cfma_conj(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(-a.y, b.x, acc.y);
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two floats in one 64-bit register pair, FMA and
// multiply on both lanes with one instruction; every lane rounds as its scalar counterpart.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk(float x, float y) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ float2 upk(f32x2 v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ f32x2 pfma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f32x2 pmul(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 padd(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ float hsum(f32x2 v) {
  const float2 t = upk(v);
  return t.x + t.y;
}

template <typename T> struct cplx;
template <> struct cplx<double> { using type = double2; };
template <> struct cplx<float> { using type = float2; };

__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }

// R . x evaluated as (R1 x1 + R2 x2) + R3 x3 with every product and sum rounded separately (no FMA
// contraction), i.e. the same rounding as the reference's broadcast in fourier_phase!
// (src/wannier/batched_fourier_core.jl:26-28).
__device__ __forceinline__ double rdotx(int r1, int r2, int r3, double x1, double x2, double x3) {
  return __dadd_rn(__dadd_rn(__dmul_rn((double)r1, x1), __dmul_rn((double)r2, x2)), __dmul_rn((double)r3, x3));
}

// exp(2 pi i t) for a double t, with exact argument reduction t - rint(t) in [-1/2, 1/2].
__device__ __forceinline__ double2 cis2pi(double t) {
  double r = t - rint(t);
  double s, c;
  sincospi(2.0 * r, &s, &c);
  return make_double2(c, s);
}

}  // namespace epb
