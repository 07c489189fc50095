// Calculator-facing device hooks of the batched e-ph loop: the window scatter of |g|^2 / omega into a
// device-resident calculator buffer (eph_window_scatter!, src/calculator/calculator_utils.jl:36-50,
// CUDA method ext/ElectronPhononCUDAExt.jl:280-313) and the Boltzmann window accumulation of the
// scattering-out / scattering-in increments (bte_window_accumulate!,
// src/boltzmann/boltzmann_calculator.jl:336-362, CUDA method ext/ElectronPhononCUDAExt.jl:323-372,
// increments of src/boltzmann/bte_scattering_core.jl:9-84).
//
// Conventions are the reference's: arrays column-major, state indices 1-based with 0 = out of window,
// index maps Int64, g2vals (nbandkq, nbandk, nm, nq_batch), omega (nm, nq_batch), imap_f (ld, nkq),
// ikqs 1-based columns of imap_f.
#include <algorithm>

#include "epb_common.cuh"

namespace epb {

// One thread per (m, n, nu, j); targets lin = nu + nm (i - i0 - 1) + nm ni_stride (f - 1) (1-based) are
// unique across a run, so no atomics.
__global__ void window_scatter_kernel(double* __restrict__ g2_out, double* __restrict__ om_out,
                                      const double* __restrict__ g2vals, const int64_t* __restrict__ imap_i,
                                      const int64_t* __restrict__ imap_f, int64_t ld_f, const int64_t* __restrict__ ikqs,
                                      const double* __restrict__ om, int64_t nbkq, int64_t nbk, int64_t nm, int64_t nqb,
                                      int64_t ni_stride, int64_t i0) {
  const int64_t N = nbkq * nbk * nm * nqb;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = e % nbkq, n = (e / nbkq) % nbk, nu = (e / (nbkq * nbk)) % nm, j = e / (nbkq * nbk * nm);
    const int64_t i = imap_i[n];
    const int64_t f = imap_f[m + ld_f * (ikqs[j] - 1)];
    if (i > 0 && f > 0) {
      const int64_t lin = nu + nm * (i - i0 - 1) + nm * ni_stride * (f - 1);  // 0-based
      g2_out[lin] = g2vals[e];
      om_out[lin] = om[nu + nm * j];
    }
  }
}

__device__ __forceinline__ double c_occ_fd(double e, double t) { return 1.0 / (exp(e / t) + 1.0); }
__device__ __forceinline__ double c_occ_fd_deriv(double e, double t) {
  return -1.0 / (2.0 + exp(e / t) + exp(-e / t)) / t;
}
__device__ __forceinline__ double c_occ_boson(double e, double t) { return e == 0.0 ? 0.0 : 1.0 / expm1(e / t); }

// (s_out, s_in) of one (k, k+q, mode) triple with Gaussian smearing eta.
__device__ void bte_increments(int method, double ek, double ekq, double wq, double g2, double wtq, double mu, double t,
                               double eta, double& so, double& si) {
  const double d1 = 0.5641895835477563 / eta * exp(-((ek - ekq + wq) / eta) * ((ek - ekq + wq) / eta));
  const double d2 = 0.5641895835477563 / eta * exp(-((ek - ekq - wq) / eta) * ((ek - ekq - wq) / eta));
  so = si = 0.0;
  if (d1 == 0.0 && d2 == 0.0) return;
  const double nq = c_occ_boson(wq, t);
  const double fk = c_occ_fd(ek - mu, t), fkq = c_occ_fd(ekq - mu, t);
  double f1o, f2o, f1i, f2i;
  switch (method) {
    case 1:
      f1o = nq + fkq;
      f2o = nq + 1 - fkq;
      f1i = nq + fk;
      f2i = nq + 1 - fk;
      break;
    case 2: {
      const double po = fkq * (1 - fkq) / (fk * (1 - fk)), pi = fk * (1 - fk) / (fkq * (1 - fkq));
      f1o = po * (nq + 1 - fk);
      f2o = po * (nq + fk);
      f1i = pi * (nq + 1 - fkq);
      f2i = pi * (nq + fkq);
      break;
    }
    case 3: {
      const double po = (1 - fkq) / (1 - fk), pi = (1 - fk) / (1 - fkq);
      f1o = po * nq;
      f2o = po * (nq + 1);
      f1i = pi * nq;
      f2i = pi * (nq + 1);
      break;
    }
    case 4: {
      const double po = fkq / fk, pi = fk / fkq;
      f1o = po * (nq + 1);
      f2o = po * nq;
      f1i = pi * (nq + 1);
      f2i = pi * nq;
      break;
    }
    case 5: {
      const double dfk = c_occ_fd_deriv(ek - mu, t), dfkq = c_occ_fd_deriv(ekq - mu, t);
      f1o = f2o = sqrt(nq * (nq + 1) * dfkq / dfk);
      f1i = f2i = sqrt(nq * (nq + 1) * dfk / dfkq);
      break;
    }
    default: {
      const double ndo = c_occ_boson(ekq - ek, t), ndi = c_occ_boson(ek - ekq, t);
      f1o = ndo + fkq;
      f2o = -(ndo + fkq);
      f1i = ndi + fk;
      f2i = -(ndi + fk);
    }
  }
  const double pref = 2.0 * 3.141592653589793 * wtq * g2;
  so = ((d1 == 0.0 ? 0.0 : d1 * f1o) + (d2 == 0.0 ? 0.0 : d2 * f2o)) * pref;
  si = ((d2 == 0.0 ? 0.0 : d2 * f1i) + (d1 == 0.0 ? 0.0 : d1 * f2i)) * pref;
}

struct AccArgs {
  double* sout;        // (n_i, nT)
  int64_t ld_sout;     // n_i
  double* sin;         // (ni_tile, n_f, nT)
  int64_t ld_sin_i, ld_sin_f;
  const double* g2vals;
  const double* om;    // (nm, nq_batch)
  const int64_t* imap_i;
  const int64_t* imap_f;
  int64_t ld_f;
  const int64_t* ikqs;
  const double* e_i;
  const double* e_f;
  const double* wf;
  const double* mus;
  const double* ts;
  const double* etas;
  int64_t nT;
  int method;
  double omega_cutoff;
  int64_t nbkq, nbk, nm, nqb, i0;
};

// One thread per (m, n, j): S_out[i, T] += sum_nu s_out (atomic: many (m, j) share an i),
// S_in[i - i0, f, T] = sum_nu s_in (each (i, f) written by one thread of the run).
__global__ void bte_window_accumulate_kernel(AccArgs a) {
  const int64_t N = a.nbkq * a.nbk * a.nqb;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = e % a.nbkq, n = (e / a.nbkq) % a.nbk, j = e / (a.nbkq * a.nbk);
    const int64_t i = a.imap_i[n];
    if (i <= 0) continue;
    const int64_t f = a.imap_f[m + a.ld_f * (a.ikqs[j] - 1)];
    if (f <= 0) continue;
    const double ek = a.e_i[i - 1], ekq = a.e_f[f - 1], wtq = a.wf[f - 1];
    const int64_t il = i - a.i0;
    for (int64_t iT = 0; iT < a.nT; ++iT) {
      double so = 0.0, si = 0.0;
      for (int64_t nu = 0; nu < a.nm; ++nu) {
        const double wq = a.om[nu + a.nm * j];
        if (wq < a.omega_cutoff) continue;
        double o, in;
        bte_increments(a.method, ek, ekq, wq, a.g2vals[m + a.nbkq * (n + a.nbk * (nu + a.nm * j))], wtq, a.mus[iT],
                       a.ts[iT], a.etas[iT], o, in);
        so += o;
        si += in;
      }
      atomicAdd(a.sout + (i - 1) + a.ld_sout * iT, so);
      if (a.sin) a.sin[(il - 1) + a.ld_sin_i * ((f - 1) + a.ld_sin_f * iT)] = si;
    }
  }
}

static unsigned grid_n(epb_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)ctx->sm_count * 32));
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_eph_window_scatter(epb_ctx* ctx, double* g2_out, double* omega_out, const double* g2vals,
                           const int64_t* imap_i_col, const int64_t* imap_f, int64_t ld_imap_f, const int64_t* ikqs,
                           const double* omega, int64_t nbandkq, int64_t nbandk, int64_t nm, int64_t nq_batch,
                           int64_t ni_stride, int64_t i0) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_eph_window_scatter: NULL ctx");
  EPB_CHECK_ARG(nbandkq >= 0 && nbandk >= 0 && nm >= 0 && nq_batch >= 0 && ni_stride >= 0 && i0 >= 0 &&
                    ld_imap_f >= nbandkq,
                "epb_eph_window_scatter: bad sizes");
  const int64_t N = nbandkq * nbandk * nm * nq_batch;
  if (N == 0) return EPB_OK;
  EPB_CHECK_ARG(g2_out && omega_out && g2vals && imap_i_col && imap_f && ikqs && omega,
                "epb_eph_window_scatter: NULL buffer");
  EPB_TRY(make_current(ctx));
  prof_begin(ctx, EPB_PROF_OTHER);
  window_scatter_kernel<<<grid_n(ctx, N), 256, 0, ctx->stream>>>(g2_out, omega_out, g2vals, imap_i_col, imap_f, ld_imap_f,
                                                                  ikqs, omega, nbandkq, nbandk, nm, nq_batch, ni_stride,
                                                                  i0);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_bte_window_accumulate(epb_ctx* ctx, double* sout, int64_t n_i, double* sin, int64_t ni_tile, int64_t n_f,
                              const double* g2vals, const double* omega, const int64_t* imap_i_at_k,
                              const int64_t* imap_f, int64_t ld_imap_f, const int64_t* ikqs, const double* e_i,
                              const double* e_f, const double* wf, const double* mus, const double* ts,
                              const double* etas, int64_t nT, int method, double omega_cutoff, int64_t nbandkq,
                              int64_t nbandk, int64_t nmodes, int64_t nq_batch, int64_t i0) {
  clear_error();
  EPB_CHECK_ARG(ctx, "epb_bte_window_accumulate: NULL ctx");
  EPB_CHECK_ARG(method >= 1 && method <= 6, "epb_bte_window_accumulate: method %d outside 1..6", method);
  EPB_CHECK_ARG(nbandkq >= 0 && nbandk >= 0 && nmodes >= 0 && nq_batch >= 0 && nT >= 1 && ld_imap_f >= nbandkq &&
                    n_i >= 0 && i0 >= 0,
                "epb_bte_window_accumulate: bad sizes");
  const int64_t N = nbandkq * nbandk * nq_batch;
  if (N == 0) return EPB_OK;
  EPB_CHECK_ARG(sout && g2vals && omega && imap_i_at_k && imap_f && ikqs && e_i && e_f && wf && mus && ts && etas,
                "epb_bte_window_accumulate: NULL buffer");
  EPB_CHECK_ARG(!sin || (ni_tile >= 1 && n_f >= 1), "epb_bte_window_accumulate: S_in tile sizes");
  EPB_TRY(make_current(ctx));
  AccArgs a{};
  a.sout = sout;
  a.ld_sout = n_i;
  a.sin = sin;
  a.ld_sin_i = ni_tile;
  a.ld_sin_f = n_f;
  a.g2vals = g2vals;
  a.om = omega;
  a.imap_i = imap_i_at_k;
  a.imap_f = imap_f;
  a.ld_f = ld_imap_f;
  a.ikqs = ikqs;
  a.e_i = e_i;
  a.e_f = e_f;
  a.wf = wf;
  a.mus = mus;
  a.ts = ts;
  a.etas = etas;
  a.nT = nT;
  a.method = method;
  a.omega_cutoff = omega_cutoff;
  a.nbkq = nbandkq;
  a.nbk = nbandk;
  a.nm = nmodes;
  a.nqb = nq_batch;
  a.i0 = i0;
  prof_begin(ctx, EPB_PROF_OTHER);
  bte_window_accumulate_kernel<<<grid_n(ctx, N), 256, 0, ctx->stream>>>(a);
  prof_end(ctx);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

}  // extern "C"
