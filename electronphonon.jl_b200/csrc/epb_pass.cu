// Whole e-ph pass over random k x random q (the arbitrary-q semantics of run_eph_over_k_and_q,
// src/calculator/run_eph_over_k_and_q.jl:251-330, batched the way the GPU outer-k loop batches,
// src/calculator/run_eph_over_k_and_kq.jl:792-892):
//
//   q side (once):  D(q) -> omega, u_ph;  P[p, q] = exp(2 pi i Rp . q)     (q convention)
//   per k batch:    H(k) -> e_k, u_k;  g(k, Rp) = RR->kR rotated by u_k
//                   H(k+q) -> e_kq, u_kq for every (k, q) pair of the batch
//                   g(k, q) = sum_p g(k, Rp) P[p, q];  ep = u_kq^dagger g u_ph;  g2 = |ep|^2 / (2 omega)
//
// The 5e10 g2 values of a full pass are never materialised: the rotation kernel consumes each
// (k, q) block in place, accumulating g2sum[nu, k] = sum_{m, n, q} g2 and writing the full block
// only for the sampled q (q % sample_stride == 0), which is what the parity checks read.
// The plain FP64 pass (the mixed pass's denominator) runs its dense algebra the way the reference's GPU
// path does, as library ZGEMMs (epb_f64blas.cu); the mixed pass is this project's kernels throughout.
#include <algorithm>
#include <vector>

#include "epb_common.cuh"



namespace epb {

int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                const double* xk, int64_t N, double2* out, int64_t ldo);
int eigh_async(epb_ctx* ctx, double2* A, int64_t n, int64_t batch, double* E, bool want_v,
               const double* mass, int prec);
int eigh_check(epb_ctx* ctx);
int mixed_pass(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double* xq, int64_t nq,
               const double2* uph, const double* omega, double* ek_out, double* g2sum, double* g2_sample,
               int64_t sample_stride, int64_t kbi_max, bool defer_checks);
int split_gemm_check(epb_ctx* ctx);
bool tune_lookup(const std::vector<std::pair<std::string, int64_t>>& kv, const std::string& key, int64_t* value);
void tune_store(std::vector<std::pair<std::string, int64_t>>& kv, const std::string& key, int64_t value);
int mixed_model_prepare(epb_ctx* ctx, epb_model* m);
void mixed_model_free(epb_model* m);

// x_{k+q} for every (k_local, q) pair, q fastest: xkq[:, kl * nq + q] = xk[:, kl] + xq[:, q]
__global__ void xkq_kernel(const double* __restrict__ xk, int64_t nkb, const double* __restrict__ xq,
                           int64_t nq, double* __restrict__ xkq) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nkb * nq) return;
  int64_t kl = idx / nq, q = idx % nq;
  xkq[3 * idx + 0] = xk[3 * kl + 0] + xq[3 * q + 0];
  xkq[3 * idx + 1] = xk[3 * kl + 1] + xq[3 * q + 1];
  xkq[3 * idx + 2] = xk[3 * kl + 2] + xq[3 * q + 2];
}

int launch_phase(epb_ctx* ctx, const epb_rset* rs, const double* xk, int64_t nk, double2* phase);
int zgemm_blas(epb_ctx* ctx, char ta, char tb, int64_t m, int64_t n, int64_t k, const double2* A, int64_t lda,
               const double2* B, int64_t ldb, double2* C, int64_t ldc);
int zgemm_blas_strided(epb_ctx* ctx, char ta, char tb, int64_t m, int64_t n, int64_t k, const double2* A,
                       int64_t lda, int64_t sa, const double2* B, int64_t ldb, int64_t sb, double2* C, int64_t ldc,
                       int64_t sc, int64_t batch);
int fourier_zgemm(epb_ctx* ctx, const double2* op_r, int64_t ndata, int64_t ld_op, const epb_rset* rs,
                  const double* x, int64_t npts, double2* phase_scratch, double2* out, int64_t ldo);
int g2_fold_f64(epb_ctx* ctx, const double2* ep, const double* omega, int nw, int nm, int64_t nq, double* g2sum,
                double* sample, int64_t stride);

}  // namespace epb

using namespace epb;

extern "C" {

int epb_model_create(epb_ctx* ctx, const double* ham_op, int64_t nw, const int64_t* irvec_el_host,
                     int64_t nr_el, const double* dyn_op, const double* mass, int64_t nm,
                     const int64_t* irvec_ph_host, int64_t nr_ph, const double* epmat_op,
                     const int64_t* irvec_ep_host, int64_t nr_ep, int flags, epb_model** out) {
  clear_error();
  EPB_CHECK_ARG(ctx && out && ham_op && irvec_el_host && dyn_op && mass && irvec_ph_host && epmat_op &&
                    irvec_ep_host,
                "epb_model_create: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nw <= 32 && nm >= 1 && nm <= 32 && nr_el >= 1 && nr_ph >= 1 && nr_ep >= 1,
                "epb_model_create: unsupported sizes (nw=%lld nm=%lld)", (long long)nw, (long long)nm);
  EPB_TRY(make_current(ctx));
  epb_model* m = new epb_model();
  m->ctx = ctx;
  m->nw = nw;
  m->nm = nm;
  m->nr_el = nr_el;
  m->nr_ph = nr_ph;
  m->nr_ep = nr_ep;
  m->ham = (const double2*)ham_op;
  m->dyn = (const double2*)dyn_op;
  m->mass = mass;
  m->epmat = (const double2*)epmat_op;
  int st = epb_rset_create(ctx, irvec_el_host, nr_el, &m->rs_el);
  if (st == EPB_OK) st = epb_rset_create(ctx, irvec_ph_host, nr_ph, &m->rs_ph);
  if (st == EPB_OK) st = epb_rset_create(ctx, irvec_ep_host, nr_ep, &m->rs_ep);
  if (st == EPB_OK && (flags & 1)) st = mixed_model_prepare(ctx, m);
  if (st != EPB_OK) {
    epb_model_destroy(m);
    return st;
  }
  *out = m;
  return EPB_OK;
}

int epb_model_destroy(epb_model* m) {
  if (!m) return EPB_OK;
  if (m->ctx) make_current(m->ctx);
  mixed_model_free(m);
  epb_rset_destroy(m->rs_el);
  epb_rset_destroy(m->rs_ph);
  epb_rset_destroy(m->rs_ep);
  if (m->graph.exec) cudaGraphExecDestroy(m->graph.exec);
  if (m->epmat_ph) cudaFree(m->epmat_ph);
  if (m->epmat_ph_planes) cudaFree(m->epmat_ph_planes);
  delete m;
  return EPB_OK;
}

static int eph_pass_run(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double* xq, int64_t nq,
                        int prec, int64_t k_batch, int64_t sample_stride, double* ek_out, double* omega_out,
                        double* g2sum_out, double* g2_sample, int64_t* stats_host, bool defer_checks = false);

// Choices of one pass: inner k batch, rotation kernel of the mixed pass (0 warp tensor cores, 1 FP32 CUDA
// cores) and kR->kq GEMM form (1 A-resident, 0 streamed operands). The mixed pass reads the last two from
// ctx->cur_rot / ctx->cur_kq_ares.
struct PassChoice {
  int64_t kb = 16;
  int rot = 0;
  int kq = 1;
};

static std::string pass_key(const char* what, const epb_model* m, int64_t nq, int prec) {
  char key[128];
  snprintf(key, sizeof(key), "pass_%s/%lld/%lld/%lld/%d", what, (long long)m->nw, (long long)m->nm, (long long)nq,
           prec);
  return key;
}
// the mixed pass has a second rotation kernel only for the register-tiled shape, and an A-resident kR->kq
// only for K' = 2 round_up(nr_ep, 8) <= 256
static bool rot_alternatives(const epb_model* m, int prec) { return prec == EPB_PREC_MIXED && m->nw == 16 && m->nm == 12; }
static bool kq_alternatives(const epb_model* m, int prec) { return prec == EPB_PREC_MIXED && m->nr_ep <= 128; }

// The choices from the context's table, else the defaults (a forced rotation kernel wins).
static PassChoice pass_choice(const epb_ctx* ctx, const epb_model* m, int64_t nq, int prec, int64_t k_batch) {
  PassChoice c;
  int64_t v;
  c.kb = k_batch > 0 ? k_batch : (tune_lookup(ctx->tuned, pass_key("kb", m, nq, prec), &v) ? v : 16);
  c.rot = ctx->rot_variant >= 0 ? ctx->rot_variant : (tune_lookup(ctx->tuned, pass_key("rot", m, nq, prec), &v) ? (int)v : 0);
  c.kq = tune_lookup(ctx->tuned, pass_key("kq", m, nq, prec), &v) ? (int)v : 1;
  return c;
}

// Autotuner of the pass (k_batch <= 0): times the candidates on the first min(nk, 64) k against the
// caller's q list (CUDA events on the context stream, one untimed run before each timed one) and keeps the
// fastest per (nw, nm, nq, prec) in the context's table: first the inner k batch (4, 8, 16, 32) -- the
// k+q eigensolve / kR->kq / rotation batch --, then with it the rotation kernel (unless one is forced) and
// the kR->kq GEMM form. Choices already in the table (measured earlier or loaded with epb_tune_import) are
// not timed again. The trial passes write the caller's outputs for those k; the real pass rewrites them.
static int tune_pass(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double* xq, int64_t nq, int prec,
                     double* ek_out, double* omega_out, double* g2sum_out, PassChoice* out) {
  PassChoice c = pass_choice(ctx, m, nq, prec, 0);
  int64_t v;
  const std::string kkb = pass_key("kb", m, nq, prec), krot = pass_key("rot", m, nq, prec),
                    kkq = pass_key("kq", m, nq, prec);
  const bool need_kb = !tune_lookup(ctx->tuned, kkb, &v);
  const bool need_rot = ctx->rot_variant < 0 && rot_alternatives(m, prec) && !tune_lookup(ctx->tuned, krot, &v);
  const bool need_kq = kq_alternatives(m, prec) && !tune_lookup(ctx->tuned, kkq, &v);
  if (need_kb || need_rot || need_kq) {
    const int64_t ns = std::min<int64_t>(nk, 64);
    cudaEvent_t e0, e1;
    EPB_CUDA(cudaEventCreate(&e0));
    EPB_CUDA(cudaEventCreate(&e1));
    // time one candidate; <0 when it does not fit (out of memory), the error status otherwise
    auto trial = [&](const PassChoice& t, float* ms) -> int {
      ctx->cur_rot = t.rot;
      ctx->cur_kq_ares = t.kq;
      int st = eph_pass_run(ctx, m, xk, ns, xq, nq, prec, t.kb, 1, ek_out, omega_out, g2sum_out, nullptr, nullptr);
      if (st == EPB_OK) {
        cudaEventRecord(e0, ctx->stream);
        st = eph_pass_run(ctx, m, xk, ns, xq, nq, prec, t.kb, 1, ek_out, omega_out, g2sum_out, nullptr, nullptr);
        cudaEventRecord(e1, ctx->stream);
      }
      if (st != EPB_OK) return st;
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(ms, e0, e1);
      return EPB_OK;
    };
    int st = EPB_OK;
    if (need_kb) {
      const int64_t cands[4] = {4, 8, 16, 32};
      float best = 1e30f;
      for (int64_t kb : cands) {
        if (kb > ns && kb != cands[0]) continue;
        PassChoice t = c;
        t.kb = kb;
        float ms = 0.f;
        st = trial(t, &ms);
        if (st == EPB_ERR_OOM) {  // a larger batch does not fit: the smaller ones stand
          clear_error();
          st = EPB_OK;
          break;
        }
        if (st != EPB_OK) break;
        if (ms < best) {
          best = ms;
          c.kb = kb;
        }
      }
      if (st == EPB_OK) tune_store(ctx->tuned, kkb, c.kb);
    }
    if (st == EPB_OK && need_rot) {
      float best = 1e30f;
      for (int r : {0, 1}) {
        PassChoice t = c;
        t.rot = r;
        float ms = 0.f;
        if ((st = trial(t, &ms)) != EPB_OK) break;
        if (ms < best) {
          best = ms;
          c.rot = r;
        }
      }
      if (st == EPB_OK) tune_store(ctx->tuned, krot, c.rot);
    }
    if (st == EPB_OK && need_kq) {
      float best = 1e30f;
      for (int f : {1, 0}) {
        PassChoice t = c;
        t.kq = f;
        float ms = 0.f;
        if ((st = trial(t, &ms)) != EPB_OK) break;
        if (ms < best) {
          best = ms;
          c.kq = f;
        }
      }
      if (st == EPB_OK) tune_store(ctx->tuned, kkq, c.kq);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != EPB_OK) return st;
  }
  *out = c;
  return EPB_OK;
}

int epb_eph_pass(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double* xq, int64_t nq,
                 int prec, int64_t k_batch, int64_t sample_stride, double* ek_out, double* omega_out,
                 double* g2sum_out, double* g2_sample, int64_t* stats_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && xk && xq && ek_out && omega_out && g2sum_out, "epb_eph_pass: NULL argument");
  EPB_CHECK_ARG(nk >= 1 && nq >= 1, "epb_eph_pass: bad sizes");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_pass: bad prec");
  EPB_CHECK_ARG(prec != EPB_PREC_MIXED || m->mixed, "epb_eph_pass: model was created without mixed planes");
  EPB_TRY(make_current(ctx));
  PassChoice ch = pass_choice(ctx, m, nq, prec, k_batch);
  if (k_batch <= 0) EPB_TRY(tune_pass(ctx, m, xk, nk, xq, nq, prec, ek_out, omega_out, g2sum_out, &ch));
  k_batch = ch.kb;
  ctx->cur_rot = ch.rot;
  ctx->cur_kq_ares = ch.kq;
  const bool capturable = ctx->graph_mode && !ctx->prof_on && ctx->stream != nullptr && ctx->stream != cudaStreamLegacy;
  auto report = [&](int64_t* sh) {  // stats: elements, inner k batch, rotation kernel, kR->kq form
    if (!sh) return;
    sh[0] = nk * nq * m->nw * m->nw * m->nm;
    sh[1] = k_batch;
    sh[2] = prec == EPB_PREC_MIXED ? ch.rot : -1;
    sh[3] = prec == EPB_PREC_MIXED ? ch.kq : -1;
  };
  if (!capturable) {
    int st = eph_pass_run(ctx, m, xk, nk, xq, nq, prec, k_batch, sample_stride, ek_out, omega_out, g2sum_out, g2_sample,
                          stats_host);
    if (st == EPB_OK) report(stats_host);
    return st;
  }
  // Graph mode: the first call with these arguments runs eagerly (sizing every workspace), the
  // second captures the pass (status checks left out of the graph), later ones replay it.
  PassGraph& pg = m->graph;
  const PassKey key{xk, nk, xq, nq, prec, k_batch, sample_stride, ek_out, omega_out, g2sum_out, g2_sample, ch.rot, ch.kq};
  if (pg.exec && pg.key == key) {
    EPB_CUDA(cudaGraphLaunch(pg.exec, ctx->stream));
    ctx->launches += pg.launches;
  } else if (pg.warm && pg.key == key) {
    if (pg.exec) {
      cudaGraphExecDestroy(pg.exec);
      pg.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    const int64_t l0 = ctx->launches;
    EPB_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int st = eph_pass_run(ctx, m, xk, nk, xq, nq, prec, k_batch, sample_stride, ek_out, omega_out, g2sum_out, g2_sample,
                          nullptr, true);
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    pg.launches = ctx->launches - l0;
    ctx->launches = l0;
    if (st != EPB_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    EPB_CUDA(ce);
    ce = cudaGraphInstantiate(&pg.exec, graph, 0);
    cudaGraphDestroy(graph);
    EPB_CUDA(ce);
    EPB_CUDA(cudaGraphLaunch(pg.exec, ctx->stream));
    ctx->launches += pg.launches;
  } else {
    int st = eph_pass_run(ctx, m, xk, nk, xq, nq, prec, k_batch, sample_stride, ek_out, omega_out, g2sum_out, g2_sample,
                          nullptr);
    if (st != EPB_OK) return st;
    pg.key = key;
    pg.warm = true;
  }
  EPB_TRY(eigh_check(ctx));
  if (prec == EPB_PREC_MIXED) EPB_TRY(split_gemm_check(ctx));
  report(stats_host);
  return EPB_OK;
}

int epb_set_rotation_variant(epb_ctx* ctx, int variant) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_set_rotation_variant: NULL ctx");
  EPB_CHECK_ARG(variant >= -1 && variant <= 1, "epb_set_rotation_variant: variant must be -1, 0 or 1");
  ctx->rot_variant = variant;
  return EPB_OK;
}

int epb_set_graph_mode(epb_ctx* ctx, int on) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_set_graph_mode: NULL ctx");
  ctx->graph_mode = on != 0;
  return EPB_OK;
}

static int eph_pass_run(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double* xq, int64_t nq,
                        int prec, int64_t k_batch, int64_t sample_stride, double* ek_out, double* omega_out,
                        double* g2sum_out, double* g2_sample, int64_t* stats_host, bool defer_checks) {
  EPB_CHECK_ARG(k_batch >= 1, "epb_eph_pass: bad k batch");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_pass: bad prec");
  EPB_CHECK_ARG(!g2_sample || sample_stride >= 1, "epb_eph_pass: sample_stride must be >= 1");
  EPB_CHECK_ARG(prec != EPB_PREC_MIXED || m->mixed, "epb_eph_pass: model was created without mixed planes");
  EPB_TRY(make_current(ctx));
  const int64_t nw = m->nw, nm = m->nm, nr_ep = m->nr_ep;
  const int64_t nw2 = nw * nw;
  if (k_batch > nk) k_batch = nk;
  // ---- workspace layout ----------------------------------------------------------------------
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_dq = carve(16ull * nm * nm * nq);
  const size_t o_ph = carve(16ull * nr_ep * nq);
  const bool f64 = prec == EPB_PREC_FP64;
  const size_t o_hk = carve(16ull * nw2 * k_batch);
  const size_t o_G = carve(f64 ? 16ull * nw2 * nm * nr_ep * k_batch : 0);
  const size_t o_xkq = carve(f64 ? 24ull * k_batch * nq : 0);
  const size_t o_hkq = carve(f64 ? 16ull * nw2 * k_batch * nq : 0);
  const size_t o_g = carve(f64 ? 16ull * nw2 * nm * nq : 0);
  const size_t o_t = carve(f64 ? 16ull * nw2 * nm * nq : 0);                   // u_kq^H g per q
  const size_t o_pkq = carve(f64 ? 16ull * m->nr_el * k_batch * nq : 0);      // phases of the k+q points
  void* base = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS0, off, &base));
  char* b = (char*)base;
  double2* Dq = (double2*)(b + o_dq);
  double2* P = (double2*)(b + o_ph);
  double2* Hk = (double2*)(b + o_hk);
  double2* G = (double2*)(b + o_G);
  double* Xkq = (double*)(b + o_xkq);
  double2* Hkq = (double2*)(b + o_hkq);
  double2* gb = (double2*)(b + o_g);
  double2* Tb = (double2*)(b + o_t);
  double2* Pkq = (double2*)(b + o_pkq);
  EPB_CUDA(cudaMemsetAsync(g2sum_out, 0, sizeof(double) * nm * nk, ctx->stream));
  const int64_t nsamp = g2_sample ? (nq + sample_stride - 1) / sample_stride : 0;
  int64_t stats[4] = {0, 0, 0, 0};

  // ---- q side --------------------------------------------------------------------------------
  EPB_TRY(fourier_f64(ctx, m->dyn, nm * nm, nm * nm, m->rs_ph, xq, nq, Dq, nm * nm));
  EPB_TRY(eigh_async(ctx, Dq, nm, nq, omega_out, true, m->mass, EPB_PREC_FP64));
  EPB_TRY(launch_phase(ctx, m->rs_ep, xq, nq, P));

  // ---- k batches -----------------------------------------------------------------------------
  if (prec == EPB_PREC_MIXED) {
    EPB_TRY(mixed_pass(ctx, m, xk, nk, xq, nq, Dq, omega_out, ek_out, g2sum_out, g2_sample, sample_stride, k_batch,
                       defer_checks));
  }
  for (int64_t k0 = 0; prec == EPB_PREC_FP64 && k0 < nk; k0 += k_batch) {
    const int64_t nkb = nk - k0 < k_batch ? nk - k0 : k_batch;
    const double* xkb = xk + 3 * k0;
    // electrons at k: FP64 in both modes (2048 points; the k side is not the bulk of the work)
    EPB_TRY(fourier_f64(ctx, m->ham, nw2, nw2, m->rs_el, xkb, nkb, Hk, nw2));
    EPB_TRY(eigh_async(ctx, Hk, nw, nkb, ek_out + nw * k0, true, nullptr, EPB_PREC_FP64));
    // x_{k+q}
    xkq_kernel<<<(unsigned)cdiv(nkb * nq, 256), 256, 0, ctx->stream>>>(xkb, nkb, xq, nq, Xkq);
    EPB_LAUNCH_CHECK();
    EPB_TRY(epb_eph_RR_to_kR(ctx, (const double*)m->epmat, nw, nm, nr_ep, m->rs_el, xkb, nkb,
                             (const double*)Hk, nw, nullptr, (double*)G, EPB_PREC_FP64));
    // H(k+q) of every pair of the batch: phase matrix and one ZGEMM (the reference's fourier_batched!)
    prof_begin(ctx, EPB_PROF_FOURIER_F64);
    EPB_TRY(fourier_zgemm(ctx, m->ham, nw2, nw2, m->rs_el, Xkq, nkb * nq, Pkq, Hkq, nw2));
    prof_end(ctx);
    EPB_TRY(eigh_async(ctx, Hkq, nw, nkb * nq, nullptr, true, nullptr, EPB_PREC_FP64));
    const int64_t ndata = nw2 * nm;
    for (int64_t kl = 0; kl < nkb; ++kl) {
      // g(k, q) = g(k, Rp) P (ZGEMM), then per q: T = u_kq^H g (nw x nw nm), ep = T u_ph (nw^2 x nm), two
      // strided-batched ZGEMMs as in the reference's eph_apply_rotations!; ep overwrites g
      prof_begin(ctx, EPB_PROF_ZGEMM);
      EPB_TRY(zgemm_blas(ctx, 'N', 'N', ndata, nq, nr_ep, G + kl * ndata * nr_ep, ndata, P, nr_ep, gb, ndata));
      prof_end(ctx);
      prof_begin(ctx, EPB_PROF_ROT);
      EPB_TRY(zgemm_blas_strided(ctx, 'C', 'N', nw, nw * nm, nw, Hkq + kl * nq * nw2, nw, nw2, gb, nw, ndata, Tb, nw,
                                 ndata, nq));
      EPB_TRY(zgemm_blas_strided(ctx, 'N', 'N', nw2, nm, nm, Tb, nw2, ndata, Dq, nm, nm * nm, gb, nw2, ndata, nq));
      EPB_TRY(g2_fold_f64(ctx, gb, omega_out, (int)nw, (int)nm, nq, g2sum_out + nm * (k0 + kl),
                          g2_sample ? g2_sample + (k0 + kl) * nsamp * nw2 * nm : nullptr, sample_stride));
      prof_end(ctx);
    }
  }
  if (!defer_checks) EPB_TRY(eigh_check(ctx));
  if (stats_host) {
    stats_host[0] = nk * nq * nw2 * nm;  // g elements produced (all bands)
    stats_host[1] = stats[1];
    stats_host[2] = stats[2];
    stats_host[3] = stats[3];
  }
  return EPB_OK;
}

}  // extern "C"
