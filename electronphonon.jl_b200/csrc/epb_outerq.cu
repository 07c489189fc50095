// Outer-q e-ph loop: g(Re, q) = sum_Rp e^{2 pi i q.Rp} g(Re, Rp) rotated into the phonon eigenmode basis
// (get_eph_RR_to_Rq!, src/wannier_to_bloch.jl:277-300), then for a list of k
// g(k, q) = sum_Re e^{2 pi i k.Re} g(Re, q) and ep[m, n, nu, k] = sum_{iw, jw} conj(ukq[iw, m, k])
// g[iw, jw, nu, k] uk[jw, n, k] (get_eph_Rq_to_kq_batched! / eph_apply_rotations_rqkq!,
// src/wannier_to_bloch_batched.jl:317-377, fused CUDA method ext/ElectronPhononCUDAExt.jl:206-258),
// plus the conversion of the e-ph matrix from the "el" layout (rows (i, j, nu, Rp), columns Re) to
// the "ph" layout (rows (i, j, nu, Re), columns Rp) (src/model.jl:80-81,293-296, src/model_new.jl:551-565).
#include <algorithm>

#include "epb_common.cuh"

namespace epb {

int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* xk,
                int64_t N, double2* out, int64_t ldo);

static unsigned grid_oq(epb_ctx* ctx, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)ctx->sm_count * 32));
}

// out[b, ir, q] (b = (i, j) pair, ir = Re) with the mode index rotated:
// out[(ij, nu), ir, q] = sum_mu g[(ij, mu), ir, q] uph[mu, nu, q].
__global__ void rq_mode_rotate_kernel(const double2* __restrict__ g, const double2* __restrict__ uph, int64_t nb,
                                      int64_t nm, int64_t nr, int64_t nq, double2* __restrict__ out) {
  const int64_t total = nb * nm * nr * nq;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e % nb, nu = (e / nb) % nm, rq = e / (nb * nm);  // rq = ir + nr q
    const int64_t q = rq / nr;
    const double2* gp = g + rq * nb * nm + b;
    const double2* up = uph + q * nm * nm + nu * nm;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t mu = 0; mu < nm; ++mu) cfma(acc, gp[mu * nb], up[mu]);
    out[e] = acc;
  }
}

// One thread per (m, n, k): ep[m, n, nu, k] for all nu; g2 = |ep|^2 / (2 omega_nu) when requested.
__global__ void rqkq_rot_kernel(const double2* __restrict__ g, const double2* __restrict__ uks,
                                const double2* __restrict__ ukqs, const double* __restrict__ omega,
                                double2* __restrict__ ep, double* __restrict__ g2, int nw, int nbkq, int nbk, int nm,
                                int64_t nk) {
  const int64_t total = (int64_t)nbkq * nbk * nk;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(t % nbkq);
    const int n = (int)((t / nbkq) % nbk);
    const int64_t k = t / ((int64_t)nbkq * nbk);
    const double2* uq = ukqs + (k * nbkq + m) * nw;
    const double2* uk = uks + (k * nbk + n) * nw;
    for (int nu = 0; nu < nm; ++nu) {
      const double2* gk = g + ((k * nm + nu) * nw) * nw;
      double2 acc = make_double2(0.0, 0.0);
      for (int jw = 0; jw < nw; ++jw) {
        double2 tv = make_double2(0.0, 0.0);
        for (int iw = 0; iw < nw; ++iw) cfma_conj(tv, uq[iw], gk[iw + jw * nw]);
        cfma(acc, tv, uk[jw]);
      }
      const int64_t o = m + (int64_t)nbkq * (n + (int64_t)nbk * (nu + (int64_t)nm * k));
      if (ep) ep[o] = acc;
      if (g2) g2[o] = (acc.x * acc.x + acc.y * acc.y) / (2.0 * omega[nu]);
    }
  }
}

// "el" layout (nb nr_ep rows, nr_el columns) -> "ph" layout (nb nr_el rows, nr_ep columns), nb = nw^2 nm.
__global__ void epmat_el_to_ph_kernel(const double2* __restrict__ in, int64_t nb, int64_t nr_el, int64_t nr_ep,
                                      double2* __restrict__ out) {
  const int64_t total = nb * nr_el * nr_ep;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e % nb, re = (e / nb) % nr_el, rp = e / (nb * nr_el);  // out element (b, re, rp)
    out[e] = in[b + nb * (rp + nr_ep * re)];
  }
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_epmat_el_to_ph(epb_ctx* ctx, const double* epmat_el, int64_t nw, int64_t nm, int64_t nr_el, int64_t nr_ep,
                       double* epmat_ph) {
  clear_error();
  EPB_CHECK_ARG(ctx && epmat_el && epmat_ph, "epb_epmat_el_to_ph: NULL argument");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nr_el >= 1 && nr_ep >= 1, "epb_epmat_el_to_ph: bad sizes");
  EPB_CHECK_ARG(epmat_el != epmat_ph, "epb_epmat_el_to_ph: in-place conversion is not supported");
  EPB_TRY(make_current(ctx));
  const int64_t nb = nw * nw * nm;
  epmat_el_to_ph_kernel<<<grid_oq(ctx, nb * nr_el * nr_ep), 256, 0, ctx->stream>>>(
      (const double2*)epmat_el, nb, nr_el, nr_ep, (double2*)epmat_ph);
  EPB_LAUNCH_CHECK();
  return EPB_OK;
}

int epb_eph_RR_to_Rq(epb_ctx* ctx, const double* epmat_ph, int64_t nw, int64_t nm, int64_t nr_el,
                     const epb_rset* rset_ph, const double* xq, int64_t nq, const double* uph, double* out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset_ph, "epb_eph_RR_to_Rq: NULL ctx or rset");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nr_el >= 1 && nq >= 0, "epb_eph_RR_to_Rq: bad sizes");
  EPB_CHECK_ARG(nq == 0 || (epmat_ph && xq && uph && out), "epb_eph_RR_to_Rq: NULL buffer");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_RR_to_Rq: bad prec");
  EPB_TRY(make_current(ctx));
  if (nq == 0) return EPB_OK;
  const int64_t nb = nw * nw, ndata = nb * nm * nr_el;
  // chunk over q so that the Fourier intermediate stays below ~2 GiB
  const int64_t qc = std::max<int64_t>(1, std::min<int64_t>(nq, ((int64_t)2 << 30) / (16 * ndata)));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EPH_G, 16 * ndata * qc, &ws));
  double2* g = (double2*)ws;
  for (int64_t q0 = 0; q0 < nq; q0 += qc) {
    const int64_t qn = std::min(qc, nq - q0);
    EPB_TRY(fourier_f64(ctx, (const double2*)epmat_ph, ndata, ndata, rset_ph, xq + 3 * q0, qn, g, ndata));
    prof_begin(ctx, EPB_PROF_RR_ROT);
    rq_mode_rotate_kernel<<<grid_oq(ctx, ndata * qn), 256, 0, ctx->stream>>>(
        g, (const double2*)uph + q0 * nm * nm, nb, nm, nr_el, qn, (double2*)out + q0 * ndata);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

int epb_eph_Rq_to_kq(epb_ctx* ctx, const double* g_Rq, int64_t nw, int64_t nm, const epb_rset* rset_el, const double* xk,
                     int64_t nk, const double* uks, int64_t nbk, const double* ukqs, int64_t nbkq, const double* omega,
                     double* ep_out, double* g2_out, int prec) {
  clear_error();
  EPB_CHECK_ARG(ctx && rset_el, "epb_eph_Rq_to_kq: NULL ctx or rset");
  EPB_CHECK_ARG(nw >= 1 && nm >= 1 && nk >= 0 && nbk >= 1 && nbk <= nw && nbkq >= 1 && nbkq <= nw,
                "epb_eph_Rq_to_kq: bad sizes");
  EPB_CHECK_ARG(nk == 0 || (g_Rq && xk && uks && ukqs && (ep_out || g2_out)), "epb_eph_Rq_to_kq: NULL buffer");
  EPB_CHECK_ARG(!g2_out || omega, "epb_eph_Rq_to_kq: g2_out requires omega");
  EPB_CHECK_ARG(prec == EPB_PREC_FP64 || prec == EPB_PREC_MIXED, "epb_eph_Rq_to_kq: bad prec");
  EPB_TRY(make_current(ctx));
  if (nk == 0) return EPB_OK;
  const int64_t ndata = nw * nw * nm;
  const int64_t kc = std::max<int64_t>(1, std::min<int64_t>(nk, ((int64_t)1 << 30) / (16 * ndata)));
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_EPH_T, 16 * ndata * kc, &ws));
  double2* g = (double2*)ws;
  for (int64_t k0 = 0; k0 < nk; k0 += kc) {
    const int64_t kn = std::min(kc, nk - k0);
    EPB_TRY(fourier_f64(ctx, (const double2*)g_Rq, ndata, ndata, rset_el, xk + 3 * k0, kn, g, ndata));
    const int64_t o = nbkq * nbk * nm * k0;
    prof_begin(ctx, EPB_PROF_ROT);
    rqkq_rot_kernel<<<grid_oq(ctx, nbkq * nbk * kn), 256, 0, ctx->stream>>>(
        g, (const double2*)uks + k0 * nw * nbk, (const double2*)ukqs + k0 * nw * nbkq, omega,
        ep_out ? (double2*)ep_out + o : nullptr, g2_out ? g2_out + o : nullptr, (int)nw, (int)nbkq, (int)nbk, (int)nm, kn);
    prof_end(ctx);
    EPB_LAUNCH_CHECK();
  }
  return EPB_OK;
}

}  // extern "C"
