// SERTA Boltzmann consumer over commensurate k = q grids (epb_bte_serta).
//
// Reference: the batched k / k+q loop (src/calculator/run_eph_over_k_and_kq.jl:792-892) feeding the
// Boltzmann calculator (src/boltzmann/boltzmann_calculator.jl:336-362, bte_window_accumulate!, the
// increments of src/boltzmann/bte_scattering_core.jl:9-84 with Gaussian smearing,
// src/common/smearing.jl:29-57) and the SERTA conductivity (src/boltzmann/electron_lbte.jl:43-49,
// 153-185). Grid order k fastest (src/common/kpoints.jl:135-153): ik = (i1 ng + i2) ng + i3.
//
// Steps (one call):
//  1. electron states on the whole grid (H(k) FP64 Fourier sum, FP64 eigensolve, energies and
//     eigenvectors kept in HBM: k+q of every pair is a grid point), energy window per k and the kept
//     list (fused compaction), the widest window W;
//  2. phonons on the same grid (D(q) Fourier sum, mass-scaled eigensolve);
//  3. band velocities of the kept states: dH/dk_a = sum_R i R_cart,a H(R) e^{2 pi i x.R} (three
//     Fourier sums), v_n = Re u_n^H dH_a u_n;
//  4. per batch of kept k: g(k, Rp) (FP64 Fourier sum, or the split-BF16 tensor-core GEMM in the mixed
//     mode, the largest contraction of the consumer) for a fixed band slice of width W containing the window
//     (offset o_k = min(band_min - 1, nw - W)); the pairs (k, q) whose k+q window is non-empty
//     (grid-hash flags + compaction, one count read-back per batch); per k: q phases, g(k,q) =
//     g(k,Rp) P (ZGEMM), rotations by u_{k+q} (its band slice) and u_ph with |g|^2 / (2 omega), and
//     the fused accumulation of the out-scattering rates S_out[k, n] over (q, m, nu);
//  5. SERTA: sigma = (spin / V) sum_{k, n in window} (1/N) (-f'(e - mu) / S_out) v v^T.
#include <algorithm>
#include <vector>

#include "epb_common.cuh"

namespace epb {

int fourier_f64(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs, const double* xk,
                int64_t N, double2* out, int64_t ldo);
int eigh_async(epb_ctx* ctx, double2* A, int64_t n, int64_t batch, double* E, bool want_v, const double* mass,
               int prec);
int eigh_check(epb_ctx* ctx);
int window_filter(epb_ctx* ctx, const double* E, int64_t nw, int64_t nk, double wmin, double wmax, int32_t* bmin,
                  int32_t* bmax, int32_t* keep_idx, int64_t* nkeep, double* nbelow);
int launch_phase(epb_ctx* ctx, const epb_rset* rs, const double* xk, int64_t nk, double2* phase);
int fourier_zgemm(epb_ctx* ctx, const double2* op_r, int64_t ndata, int64_t ld_op, const epb_rset* rs,
                  const double* x, int64_t npts, double2* phase_scratch, double2* out, int64_t ldo);
int zgemm_nn(epb_ctx* ctx, const double2* A, int64_t lda, const double2* B, int64_t ldb, double2* C, int64_t ldc,
             int64_t M, int64_t N, int64_t K);
int eph_rotations_f64(epb_ctx* ctx, const double2* g, int64_t ldg, int nw, int nbk, int nm, int64_t nq,
                      const double2* ukq, int nbkq, const double2* uph, const double* omega, double2* ep, double* g2);
int mixed_rr_to_kR(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double2* uk, int nband,
                   double2* out);
int split_gemm_check(epb_ctx* ctx);
int eph_rotations_c64(epb_ctx* ctx, const float2* g, int64_t ldg, int nw, int nbk, int nm, int64_t nq,
                      const double2* ukq, int nbkq, const double2* uph, const double* omega, double2* ep, double* g2);
int64_t bte_a2_bytes(epb_model* m, int64_t nk, int64_t nband);
int64_t bte_b_bytes(epb_model* m, int64_t ncols);
int bte_pack_kR(epb_ctx* ctx, epb_model* m, const double* xk, int64_t nk, const double2* uk, int nband, uint8_t* a2);
int bte_kq_grouped(epb_ctx* ctx, epb_model* m, const uint8_t* a2, int64_t nk_a2, int nband, const double* x,
                   int64_t ncols, const int64_t* grp, const int64_t* grp_a, int64_t ngrp, uint8_t* bmem, float2* C,
                   int64_t ldc);

static unsigned gsz(epb_ctx* ctx, int64_t total) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(total, 256), (int64_t)ctx->sm_count * 16));
}

__device__ __forceinline__ int64_t grid_index(int64_t i1, int64_t i2, int64_t i3, int64_t ng) {
  return (i1 * ng + i2) * ng + i3;
}

__global__ void bte_grid_points_kernel(int64_t ng, double* __restrict__ x) {
  const int64_t N = ng * ng * ng;
  for (int64_t ik = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ik < N; ik += (int64_t)gridDim.x * blockDim.x) {
    x[3 * ik] = (double)(ik / (ng * ng)) / (double)ng;
    x[3 * ik + 1] = (double)((ik / ng) % ng) / (double)ng;
    x[3 * ik + 2] = (double)(ik % ng) / (double)ng;
  }
}

struct Lattice {
  double a[9];  // column-major: column d = lattice vector a_d (Cartesian)
};

// dop[a][:, r] = i R_cart,a op[:, r], R_cart = A R.
__global__ void bte_deriv_op_kernel(const double2* __restrict__ op, int64_t nd, const int4* __restrict__ rv, int64_t nr,
                                    Lattice L, double2* __restrict__ dop) {
  const int64_t total = nd * nr;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / nd;
    const int4 R = rv[r];
    const double2 v = op[e];
    for (int a = 0; a < 3; ++a) {
      const double rc = L.a[a] * R.x + L.a[3 + a] * R.y + L.a[6 + a] * R.z;
      dop[(int64_t)a * total + e] = make_double2(-rc * v.y, rc * v.x);  // i rc (x + i y)
    }
  }
}

// v[(kk * 3 + a) * nw + n] = Re u_n^H dH_a u_n for the kept point kk (grid point keep[kk]).
__global__ void bte_velocity_kernel(const double2* __restrict__ dH, int64_t nkb, const double2* __restrict__ U,
                                    const int32_t* __restrict__ keep, int64_t k0, int nw, double* __restrict__ v) {
  const int64_t total = nkb * 3 * nw;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int n = (int)(e % nw);
    const int a = (int)((e / nw) % 3);
    const int64_t kk = e / (3 * nw);
    const double2* u = U + (int64_t)keep[k0 + kk] * nw * nw + (int64_t)n * nw;
    const double2* h = dH + ((int64_t)a * nkb + kk) * nw * nw;
    double acc = 0.0;
    // (H u)_i = sum_j h_ij u_j ; acc = Re sum_i conj(u_i) (H u)_i
    for (int i = 0; i < nw; ++i) {
      double2 hu = make_double2(0.0, 0.0);
      for (int j = 0; j < nw; ++j) cfma(hu, h[i + j * nw], u[j]);
      acc += u[i].x * hu.x + u[i].y * hu.y;
    }
    v[(k0 + kk) * 3 * nw + a * nw + n] = acc;
  }
}

__global__ void bte_gather_x_kernel(const double* __restrict__ xg, const int32_t* __restrict__ keep, int64_t k0,
                                    int64_t n, double* __restrict__ x) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) x[3 * j + d] = xg[3 * (int64_t)keep[k0 + j] + d];
}

// Stable compaction kernels (epb_pairs.cu).
__global__ void cmp_count_kernel(const int32_t* __restrict__ flag, int64_t n, int32_t* __restrict__ bcount);
__global__ void cmp_scan_kernel(int32_t* __restrict__ bcount, int64_t nblocks, int64_t* __restrict__ running,
                                int64_t* __restrict__ boff);
__global__ void cmp_scatter_kernel(const int32_t* __restrict__ flag, int64_t n, const int64_t* __restrict__ boff,
                                   const int64_t* __restrict__ pidx, int64_t base, int64_t* __restrict__ out,
                                   const int32_t* __restrict__ bmin, const int32_t* __restrict__ bmax,
                                   int32_t* __restrict__ omin, int32_t* __restrict__ omax, int64_t cap);

// Band-slice offset of a grid point with a non-empty window: o = min(band_min - 1, nw - W).
__device__ __forceinline__ int slice_offset(int bmin, int nw, int W) { return min(bmin - 1, nw - W); }

// uk slice of the kept points keep[k0 .. k0 + nkb): out (nw x W x nkb).
__global__ void bte_gather_uk_kernel(const double2* __restrict__ U, const int32_t* __restrict__ keep, int64_t k0,
                                     int64_t nkb, const int32_t* __restrict__ bmin, int nw, int W,
                                     double2* __restrict__ out) {
  const int64_t total = nkb * nw * W;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nw);
    const int c = (int)((e / nw) % W);
    const int64_t kk = e / ((int64_t)nw * W);
    const int64_t ik = keep[k0 + kk];
    const int o = slice_offset(bmin[ik], nw, W);
    out[e] = U[ik * nw * nw + (int64_t)(o + c) * nw + i];
  }
}

// flag[kk * N + iq] = window of k+q non-empty, for the kept points of the batch.
__global__ void bte_pair_flags_kernel(const int32_t* __restrict__ keep, int64_t k0, int64_t nkb, int64_t ng,
                                      const int32_t* __restrict__ bmin, int32_t* __restrict__ flag) {
  const int64_t N = ng * ng * ng, total = nkb * N;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t iq = e % N, ik = keep[k0 + e / N];
    const int64_t ikq = grid_index((ik / (ng * ng) + iq / (ng * ng)) % ng, ((ik / ng) % ng + (iq / ng) % ng) % ng,
                                   (ik % ng + iq % ng) % ng, ng);
    flag[e] = bmin[ikq] > 0;
  }
}

// seg[kk] = first position of pairs of batch point kk in the ascending pair list (lower bound).
__global__ void bte_segments_kernel(const int64_t* __restrict__ pairs, int64_t np, int64_t N, int64_t nkb,
                                    int64_t* __restrict__ seg) {
  for (int64_t kk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; kk <= nkb; kk += (int64_t)gridDim.x * blockDim.x) {
    const int64_t key = kk * N;
    int64_t lo = 0, hi = np;
    while (lo < hi) {
      const int64_t mid = (lo + hi) / 2;
      if (pairs[mid] < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    seg[kk] = lo;
  }
}

// q-side data of the pairs pairs[s0 .. s0 + n) of batch point kk (grid point ik): x_q, the k+q band
// slice of U, u_ph, omega, and the k+q grid index.
__global__ void bte_gather_q_kernel(const int64_t* __restrict__ pairs, int64_t n, int64_t ik, int64_t ng,
                                    const double* __restrict__ xgrid, const double2* __restrict__ U,
                                    const int32_t* __restrict__ bmin, int nw, int W, const double2* __restrict__ uph_g,
                                    const double* __restrict__ om_g, int nm, double* __restrict__ xq,
                                    double2* __restrict__ ukq, double2* __restrict__ uph, double* __restrict__ om,
                                    int32_t* __restrict__ ikq_out) {
  const int64_t N = ng * ng * ng;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t iq = pairs[j] % N;
    const int64_t ikq = grid_index((ik / (ng * ng) + iq / (ng * ng)) % ng, ((ik / ng) % ng + (iq / ng) % ng) % ng,
                                   (ik % ng + iq % ng) % ng, ng);
    ikq_out[j] = (int32_t)ikq;
    for (int d = 0; d < 3; ++d) xq[3 * j + d] = xgrid[3 * iq + d];
    const int o = slice_offset(bmin[ikq], nw, W);
    for (int c = 0; c < W; ++c)
      for (int i = 0; i < nw; ++i) ukq[(j * W + c) * nw + i] = U[ikq * nw * nw + (int64_t)(o + c) * nw + i];
    for (int e = 0; e < nm * nm; ++e) uph[j * nm * nm + e] = uph_g[iq * nm * nm + e];
    for (int e = 0; e < nm; ++e) om[j * nm + e] = om_g[iq * nm + e];
  }
}

struct BteParams {
  double mu, temp, eta, omega_cutoff, wtq;
  int method;
};

__device__ __forceinline__ double occ_fd(double e, double t) { return 1.0 / (exp(e / t) + 1.0); }
__device__ __forceinline__ double occ_fd_deriv(double e, double t) { return -1.0 / (2.0 + exp(e / t) + exp(-e / t)) / t; }
__device__ __forceinline__ double occ_boson(double e, double t) { return e == 0.0 ? 0.0 : 1.0 / expm1(e / t); }
__device__ __forceinline__ double gauss(double de, double eta) {
  return 0.5641895835477563 / eta * exp(-(de / eta) * (de / eta));  // 1/sqrt(pi)
}

// Out-scattering increment of one (k, k+q, mode) triple (bte_scattering_core.jl:9-84).
__device__ double bte_out_increment(const BteParams& p, double ek, double ekq, double wq, double g2) {
  const double d1 = gauss(ek - ekq + wq, p.eta), d2 = gauss(ek - ekq - wq, p.eta);
  if (d1 == 0.0 && d2 == 0.0) return 0.0;
  const double nq = occ_boson(wq, p.temp);
  const double fk = occ_fd(ek - p.mu, p.temp), fkq = occ_fd(ekq - p.mu, p.temp);
  double f1, f2;
  switch (p.method) {
    case 1:
      f1 = nq + fkq;
      f2 = nq + 1 - fkq;
      break;
    case 2: {
      const double pre = fkq * (1 - fkq) / (fk * (1 - fk));
      f1 = pre * (nq + 1 - fk);
      f2 = pre * (nq + fk);
      break;
    }
    case 3: {
      const double pre = (1 - fkq) / (1 - fk);
      f1 = pre * nq;
      f2 = pre * (nq + 1);
      break;
    }
    case 4: {
      const double pre = fkq / fk;
      f1 = pre * (nq + 1);
      f2 = pre * nq;
      break;
    }
    case 5: {
      const double dfk = occ_fd_deriv(ek - p.mu, p.temp), dfkq = occ_fd_deriv(ekq - p.mu, p.temp);
      f1 = sqrt(nq * (nq + 1) * dfkq / dfk);
      f2 = f1;
      break;
    }
    default: {
      const double nd = occ_boson(ekq - ek, p.temp);
      f1 = nd + fkq;
      f2 = -(nd + fkq);
    }
  }
  const double so = (d1 == 0.0 ? 0.0 : d1 * f1) + (d2 == 0.0 ? 0.0 : d2 * f2);
  return so * 2.0 * 3.141592653589793 * p.wtq * g2;
}

// S_out[kk_glob * W + n] += sum over (pair j, m, nu) of the increments; one thread per (j, n).
__global__ void bte_accumulate_kernel(const double* __restrict__ g2, int64_t n, int W, int nm,
                                      const double* __restrict__ E, int nw, int64_t ik,
                                      const int32_t* __restrict__ ikq, const int32_t* __restrict__ bmin,
                                      const int32_t* __restrict__ bmax, const double* __restrict__ om, BteParams p,
                                      double* __restrict__ sout) {
  const int bmin_k = bmin[ik], bmax_k = bmax[ik];
  const int ok_ = slice_offset(bmin_k, nw, W);
  const int64_t total = n * W;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int nb = (int)(e % W);
    const int64_t j = e / W;
    const int bk = ok_ + nb;  // 0-based band at k
    if (bk < bmin_k - 1 || bk > bmax_k - 1) continue;
    const int64_t f = ikq[j];
    const int bmf = bmin[f], bxf = bmax[f];
    const int okq = slice_offset(bmf, nw, W);
    const double ek = E[ik * nw + bk];
    double acc = 0.0;
    for (int m = 0; m < W; ++m) {
      const int bq = okq + m;
      if (bq < bmf - 1 || bq > bxf - 1) continue;
      const double ekq = E[f * nw + bq];
      for (int nu = 0; nu < nm; ++nu) {
        const double wq = om[j * nm + nu];
        if (wq < p.omega_cutoff) continue;
        acc += bte_out_increment(p, ek, ekq, wq, g2[((j * nm + nu) * W + nb) * W + m]);
      }
    }
    if (acc != 0.0) atomicAdd(sout + nb, acc);
  }
}

// Columns of the grouped tensor-core kR->kq: group g (tiles [grp[g], grp[g+1]) of 128 columns) holds the
// pairs plist[grp_p0[g] + j], j < grp_n[g], of the batch's kept k number grp_a[g]; the rest of its columns
// are padding (zero u_{k+q}, so their g2 is zero, and ikq = -1). Per column: q, u_{k+q} slice, u_ph, omega.
__global__ void bte_cols_kernel(const int64_t* __restrict__ grp, const int64_t* __restrict__ grp_a,
                                const int64_t* __restrict__ grp_p0, const int64_t* __restrict__ grp_n, int64_t ngrp,
                                int64_t ncols, const int64_t* __restrict__ plist, const int32_t* __restrict__ keep,
                                int64_t b0, int64_t ng, const double* __restrict__ xgrid, const double2* __restrict__ U,
                                const int32_t* __restrict__ bmin, int nw, int W, const double2* __restrict__ uph_g,
                                const double* __restrict__ om_g, int nm, double* __restrict__ xq,
                                double2* __restrict__ ukq, double2* __restrict__ uph, double* __restrict__ om,
                                int32_t* __restrict__ ikq_out, int32_t* __restrict__ kk_out) {
  const int64_t N = ng * ng * ng;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t tile = c / 128;
    int64_t lo = 0, hi = ngrp;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (grp[mid] <= tile) lo = mid; else hi = mid;
    }
    const int64_t j = c - grp[lo] * 128;
    if (j >= grp_n[lo]) {
      for (int d = 0; d < 3; ++d) xq[3 * c + d] = 0.0;
      for (int e = 0; e < W * nw; ++e) ukq[c * W * nw + e] = make_double2(0.0, 0.0);
      for (int e = 0; e < nm * nm; ++e) uph[c * nm * nm + e] = make_double2(0.0, 0.0);
      for (int e = 0; e < nm; ++e) om[c * nm + e] = 1.0;
      ikq_out[c] = -1;
      kk_out[c] = -1;
      continue;
    }
    const int64_t kk = grp_a[lo];
    const int64_t ik = keep[b0 + kk];
    const int64_t iq = plist[grp_p0[lo] + j] % N;
    const int64_t ikq = grid_index((ik / (ng * ng) + iq / (ng * ng)) % ng, ((ik / ng) % ng + (iq / ng) % ng) % ng,
                                   (ik % ng + iq % ng) % ng, ng);
    ikq_out[c] = (int32_t)ikq;
    kk_out[c] = (int32_t)kk;
    for (int d = 0; d < 3; ++d) xq[3 * c + d] = xgrid[3 * iq + d];
    const int o = slice_offset(bmin[ikq], nw, W);
    for (int b = 0; b < W; ++b)
      for (int i = 0; i < nw; ++i) ukq[(c * W + b) * nw + i] = U[ikq * nw * nw + (int64_t)(o + b) * nw + i];
    for (int e = 0; e < nm * nm; ++e) uph[c * nm * nm + e] = uph_g[iq * nm * nm + e];
    for (int e = 0; e < nm; ++e) om[c * nm + e] = om_g[iq * nm + e];
  }
}

// Light column map for narrow windows (W <= 4): the phase point x_q of every column (for the packed B
// operand) and the column's kept k (local), q and k+q grid indices (-1 for padding).
__global__ void bte_cols_meta_kernel(const int64_t* __restrict__ grp, const int64_t* __restrict__ grp_a,
                                     const int64_t* __restrict__ grp_p0, const int64_t* __restrict__ grp_n,
                                     int64_t ngrp, int64_t ncols, const int64_t* __restrict__ plist,
                                     const int32_t* __restrict__ keep, int64_t b0, int64_t ng,
                                     const double* __restrict__ xgrid, double* __restrict__ xq,
                                     int32_t* __restrict__ kk_out, int32_t* __restrict__ iq_out,
                                     int32_t* __restrict__ ikq_out) {
  const int64_t N = ng * ng * ng;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t tile = c / 128;
    int64_t lo = 0, hi = ngrp;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (grp[mid] <= tile) lo = mid; else hi = mid;
    }
    const int64_t j = c - grp[lo] * 128;
    if (j >= grp_n[lo]) {
      for (int d = 0; d < 3; ++d) xq[3 * c + d] = 0.0;
      kk_out[c] = iq_out[c] = ikq_out[c] = -1;
      continue;
    }
    const int64_t kk = grp_a[lo], ik = keep[b0 + kk];
    const int64_t iq = plist[grp_p0[lo] + j] % N;
    kk_out[c] = (int32_t)kk;
    iq_out[c] = (int32_t)iq;
    ikq_out[c] = (int32_t)grid_index((ik / (ng * ng) + iq / (ng * ng)) % ng, ((ik / ng) % ng + (iq / ng) % ng) % ng,
                                     (ik % ng + iq % ng) % ng, ng);
    for (int d = 0; d < 3; ++d) xq[3 * c + d] = xgrid[3 * iq + d];
  }
}

// Rotation, |g|^2 fold and out-scattering accumulation, one column per 16-lane group (narrow windows,
// W <= 4), two columns per warp:
//   T[m, n, jm] = sum_iw conj(ukq[iw, m]) g[iw, n, jm],  ep[m, n, nu] = sum_jm T[m, n, jm] uph[jm, nu],
//   g2 = |ep|^2 / (2 omega_nu), and S_out[n at k] += the method's increments over m, nu
// (eph_rot_kernel + bte_accumulate_kernel in one pass). g(k, q) and u_ph are read straight from global
// memory (each lane a contiguous run), u_{k+q} by grid index into a small shared slice; the per-column
// sums over (m, nu) are reduced across the group, one atomic per state.
constexpr int BTE_GROUPS = 16;  // 16-lane groups per block (256 threads)
__global__ void __launch_bounds__(16 * BTE_GROUPS, 4) bte_rot_acc_kernel(
    const float2* __restrict__ C, int64_t ldc, int64_t ncols, const int32_t* __restrict__ kk_col,
    const int32_t* __restrict__ iq_col, const int32_t* __restrict__ ikq_col, const int32_t* __restrict__ keep,
    int64_t b0, const double2* __restrict__ U, const int32_t* __restrict__ bmin, const int32_t* __restrict__ bmax,
    const double* __restrict__ E, const double2* __restrict__ uph_g, const double* __restrict__ om_g, int nw, int W,
    int nm, BteParams p, double* __restrict__ sout) {
  extern __shared__ __align__(16) unsigned char bte_smem[];
  const int grp = threadIdx.x >> 4, l = threadIdx.x & 15;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const int nt = W * W * nm;
  double2* su = reinterpret_cast<double2*>(bte_smem) + (size_t)grp * (nw * W + nt);  // ukq slice (nw x W)
  double2* st = su + nw * W;                                                          // T (W, W, nm), m fastest
  const int64_t gid = (int64_t)blockIdx.x * BTE_GROUPS + grp, ngroups = (int64_t)gridDim.x * BTE_GROUPS;
  const int64_t iters = (ncols + ngroups - 1) / ngroups;  // same trip count in both halves of a warp
  for (int64_t it = 0; it < iters; ++it) {
    const int64_t c = gid + it * ngroups;
    const int32_t f = c < ncols ? ikq_col[c] : -1;
    const bool valid = f >= 0;
    int64_t kk = 0, ik = 0, iq = 0;
    int bmin_k = 0, bmax_k = -1, bmf = 0, bxf = -1, ok_ = 0, oq = 0;
    if (valid) {
      kk = kk_col[c];
      iq = iq_col[c];
      ik = keep[b0 + kk];
      bmin_k = bmin[ik];
      bmax_k = bmax[ik];
      bmf = bmin[f];
      bxf = bmax[f];
      ok_ = slice_offset(bmin_k, nw, W);
      oq = slice_offset(bmf, nw, W);
      for (int e = l; e < nw * W; e += 16) su[e] = U[(int64_t)f * nw * nw + (int64_t)oq * nw + e];
    }
    __syncwarp(hmask);
    if (valid) {
      const float2* gc = C + c * ldc;
      for (int e = l; e < nt; e += 16) {  // e = m + W (n + W jm)
        const int m = e % W, r = e / W;   // r = n + W jm
        const float2* gr = gc + (int64_t)r * nw;
        double2 acc = make_double2(0.0, 0.0);
        for (int iw = 0; iw < nw; ++iw) {
          const float2 gv = gr[iw];
          cfma_conj(acc, su[m * nw + iw], make_double2(gv.x, gv.y));
        }
        st[e] = acc;
      }
    }
    __syncwarp(hmask);
    for (int n = 0; n < W; ++n) {
      double part = 0.0;
      const int bk = ok_ + n;
      if (valid && bk >= bmin_k - 1 && bk <= bmax_k - 1) {
        const double ek = E[ik * nw + bk];
        for (int e = l; e < W * nm; e += 16) {
          const int m = e % W, nu = e / W;
          const int bq = oq + m;
          if (bq < bmf - 1 || bq > bxf - 1) continue;
          const double wq = om_g[iq * nm + nu];
          if (wq < p.omega_cutoff) continue;
          const double2* up = uph_g + iq * nm * nm + (int64_t)nu * nm;
          double2 v = make_double2(0.0, 0.0);
          for (int jm = 0; jm < nm; ++jm) cfma(v, st[m + W * (n + W * jm)], up[jm]);
          const double g2 = (v.x * v.x + v.y * v.y) / (2.0 * wq);
          part += bte_out_increment(p, ek, E[(int64_t)f * nw + bq], wq, g2);
        }
      }
      for (int o = 8; o > 0; o >>= 1) part += __shfl_xor_sync(hmask, part, o);
      if (l == 0 && part != 0.0) atomicAdd(sout + (b0 + kk) * W + n, part);
    }
    __syncwarp(hmask);
  }
}

// bte_accumulate_kernel over columns of several kept k (column c belongs to kept k b0 + kk_c; padding skipped).
__global__ void bte_accumulate_cols_kernel(const double* __restrict__ g2, int64_t n, int W, int nm,
                                           const double* __restrict__ E, int nw, const int32_t* __restrict__ keep,
                                           int64_t b0, const int32_t* __restrict__ kk_col,
                                           const int32_t* __restrict__ ikq, const int32_t* __restrict__ bmin,
                                           const int32_t* __restrict__ bmax, const double* __restrict__ om, BteParams p,
                                           double* __restrict__ sout) {
  const int64_t total = n * W;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int nb = (int)(e % W);
    const int64_t j = e / W;
    if (ikq[j] < 0) continue;
    const int64_t kk = kk_col[j], ik = keep[b0 + kk];
    const int bmin_k = bmin[ik], bmax_k = bmax[ik];
    const int bk = slice_offset(bmin_k, nw, W) + nb;  // 0-based band at k
    if (bk < bmin_k - 1 || bk > bmax_k - 1) continue;
    const int64_t f = ikq[j];
    const int bmf = bmin[f], bxf = bmax[f];
    const int okq = slice_offset(bmf, nw, W);
    const double ek = E[ik * nw + bk];
    double acc = 0.0;
    for (int m = 0; m < W; ++m) {
      const int bq = okq + m;
      if (bq < bmf - 1 || bq > bxf - 1) continue;
      const double ekq = E[f * nw + bq];
      for (int nu = 0; nu < nm; ++nu) {
        const double wq = om[j * nm + nu];
        if (wq < p.omega_cutoff) continue;
        acc += bte_out_increment(p, ek, ekq, wq, g2[((j * nm + nu) * W + nb) * W + m]);
      }
    }
    if (acc != 0.0) atomicAdd(sout + (b0 + kk) * W + nb, acc);
  }
}

// sigma (9, column-major) += (1/N) (-f'(e - mu) / S_out) v v^T over the kept states; inv_tau listed.
__global__ void bte_serta_kernel(const int32_t* __restrict__ keep, int64_t nkeep, const int32_t* __restrict__ bmin,
                                 const int32_t* __restrict__ bmax, const double* __restrict__ E, int nw, int W,
                                 const double* __restrict__ sout, const double* __restrict__ v, double mu, double temp,
                                 double wk, double* __restrict__ sigma) {
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nkeep * W; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t kk = e / W;
    const int nb = (int)(e % W);
    const int64_t ik = keep[kk];
    const int b = slice_offset(bmin[ik], nw, W) + nb;
    if (b < bmin[ik] - 1 || b > bmax[ik] - 1) continue;
    const double it = sout[e];
    if (!(it > 0.0)) continue;
    const double df = -occ_fd_deriv(E[ik * nw + b] - mu, temp) / it;
    const double va[3] = {v[kk * 3 * nw + b], v[kk * 3 * nw + nw + b], v[kk * 3 * nw + 2 * nw + b]};
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) s[a + 3 * c] += wk * df * va[a] * va[c];
  }
  for (int i = 0; i < 9; ++i) {
    double x = s[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(sigma + i, x);
  }
}

// inv_tau of the kept states in order (kept k ascending, band ascending), up to cap.
__global__ void bte_list_states_kernel(const int32_t* __restrict__ keep, int64_t nkeep, const int32_t* __restrict__ bmin,
                                       const int32_t* __restrict__ bmax, int nw, int W, const double* __restrict__ sout,
                                       const int64_t* __restrict__ state_off, double* __restrict__ out, int64_t cap) {
  for (int64_t kk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; kk < nkeep; kk += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ik = keep[kk];
    const int o = slice_offset(bmin[ik], nw, W);
    int64_t pos = state_off[kk];
    for (int b = bmin[ik] - 1; b <= bmax[ik] - 1; ++b, ++pos)
      if (pos < cap) out[pos] = sout[kk * W + (b - o)];
  }
}

__global__ void bte_width_kernel(const int32_t* __restrict__ keep, int64_t nkeep, const int32_t* __restrict__ bmin,
                                 const int32_t* __restrict__ bmax, int* __restrict__ wmax, int64_t* __restrict__ nstates) {
  int w = 0;
  long long c = 0;
  for (int64_t kk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; kk < nkeep; kk += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ik = keep[kk];
    const int d = bmax[ik] - bmin[ik] + 1;
    w = max(w, d);
    c += d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(wmax, w);
    atomicAdd((unsigned long long*)nstates, (unsigned long long)c);
  }
}

// state_off[kk] = number of window states of the kept points before kk (exclusive scan, one block).
__global__ void bte_state_offsets_kernel(const int32_t* __restrict__ keep, int64_t nkeep, const int32_t* __restrict__ bmin,
                                         const int32_t* __restrict__ bmax, int64_t* __restrict__ off) {
  __shared__ int64_t carry;
  __shared__ int64_t buf[1024];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nkeep; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < nkeep ? (int64_t)(bmax[keep[i]] - bmin[keep[i]] + 1) : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const int64_t t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nkeep) off[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += buf[1023];
    __syncthreads();
  }
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_bte_serta(epb_ctx* ctx, epb_model* m, const epb_bte_params* prm, double* sigma_host, double* inv_tau,
                  int64_t inv_tau_cap, int64_t* stats_host) {
  clear_error();
  EPB_CHECK_ARG(ctx && m && prm && sigma_host, "epb_bte_serta: NULL argument");
  const int64_t ng = prm->ngrid;
  EPB_CHECK_ARG(ng >= 1 && ng <= 128, "epb_bte_serta: ngrid %lld outside 1..128", (long long)ng);
  EPB_CHECK_ARG(prm->temperature > 0 && prm->smearing > 0 && prm->volume > 0, "epb_bte_serta: bad physical parameters");
  EPB_CHECK_ARG(prm->method >= 1 && prm->method <= 6, "epb_bte_serta: method %d outside 1..6", prm->method);
  EPB_CHECK_ARG(prm->prec == EPB_PREC_FP64 || prm->prec == EPB_PREC_MIXED, "epb_bte_serta: unknown precision %d",
                prm->prec);
  EPB_CHECK_ARG(prm->prec == EPB_PREC_FP64 || m->mixed,
                "epb_bte_serta: EPB_PREC_MIXED needs a model created with the mixed operand planes");
  EPB_CHECK_ARG(inv_tau_cap == 0 || inv_tau, "epb_bte_serta: NULL inv_tau with a capacity");
  EPB_TRY(make_current(ctx));
  const int nw = (int)m->nw, nm = (int)m->nm;
  const int64_t N = ng * ng * ng, nw2 = (int64_t)nw * nw, nr_ep = m->nr_ep;
  // 128 kept k per batch by default: the RR->kR GEMM's column tile is 128 points wide
  const int64_t KB = std::max<int64_t>(1, std::min<int64_t>(prm->k_batch > 0 ? prm->k_batch : 128, 256));
  EPB_CHECK_ARG(prm->pair_chunk <= 0 || prm->pair_chunk % 128 == 0, "epb_bte_serta: pair_chunk must be a multiple of 128");
  EPB_CHECK_ARG(prm->shard_count <= 1 || (prm->shard_rank >= 0 && prm->shard_rank < prm->shard_count),
                "epb_bte_serta: shard_rank %lld outside 0..%lld", (long long)prm->shard_rank,
                (long long)prm->shard_count - 1);
  const int64_t QCH = prm->pair_chunk > 0 ? prm->pair_chunk : 65536;  // pairs per rotation launch

  // ---- persistent buffers (whole grid) ----
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_x = take(24 * N), o_U = take(16 * nw2 * N), o_E = take(8 * nw * N), o_bmin = take(4 * N),
               o_bmax = take(4 * N), o_keep = take(4 * std::max<int64_t>(N, 1)), o_nkeep = take(64),
               o_uph = take(16 * (int64_t)nm * nm * N), o_om = take(8 * (int64_t)nm * N), o_sig = take(9 * 8),
               o_w = take(64);
  void* ws = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS2, off + 256, &ws));
  uint8_t* base = (uint8_t*)ws;
  double* xg = (double*)(base + o_x);
  double2* U = (double2*)(base + o_U);
  double* E = (double*)(base + o_E);
  int32_t* bmin = (int32_t*)(base + o_bmin);
  int32_t* bmax = (int32_t*)(base + o_bmax);
  int32_t* keep = (int32_t*)(base + o_keep);
  int64_t* nkeep_d = (int64_t*)(base + o_nkeep);
  double2* uph = (double2*)(base + o_uph);
  double* om = (double*)(base + o_om);
  double* sig_d = (double*)(base + o_sig);
  int* wmax_d = (int*)(base + o_w);
  int64_t* nst_d = (int64_t*)(base + o_w + 8);

  // 1. electrons on the grid
  bte_grid_points_kernel<<<gsz(ctx, N), 256, 0, ctx->stream>>>(ng, xg);
  EPB_LAUNCH_CHECK();
  const int64_t HC = 65536;
  // H(k) of the grid as a phase matrix times H(R) (one cuBLAS ZGEMM per chunk of 65536 points, the phase
  // chunk in a workspace): the FP64 Fourier sum at library-GEMM rate
  void* phs = nullptr;
  EPB_TRY(ws_get(ctx, EPB_WS_PASS6, (size_t)m->rs_el->nr * std::min(HC, N) * sizeof(double2) + 256, &phs));
  for (int64_t k0 = 0; k0 < N; k0 += HC) {
    const int64_t kn = std::min(HC, N - k0);
    prof_begin(ctx, EPB_PROF_FOURIER_F64);
    EPB_TRY(fourier_zgemm(ctx, m->ham, nw2, nw2, m->rs_el, xg + 3 * k0, kn, (double2*)phs, U + k0 * nw2, nw2));
    prof_end(ctx);
    // the mixed mode solves in FP32 and refines in FP64 (eigenvalues to the FP64 level, vectors to ~1e-12)
    EPB_TRY(eigh_async(ctx, U + k0 * nw2, nw, kn, E + k0 * nw, true, nullptr, prm->prec));
  }
  EPB_TRY(window_filter(ctx, E, nw, N, prm->wmin, prm->wmax, bmin, bmax, keep, nkeep_d, nullptr));
  // 2. phonons on the grid
  for (int64_t q0 = 0; q0 < N; q0 += HC) {
    const int64_t qn = std::min(HC, N - q0);
    EPB_TRY(fourier_f64(ctx, m->dyn, (int64_t)nm * nm, (int64_t)nm * nm, m->rs_ph, xg + 3 * q0, qn,
                        uph + q0 * nm * nm, (int64_t)nm * nm));
    EPB_TRY(eigh_async(ctx, uph + q0 * nm * nm, nm, qn, om + q0 * nm, true, m->mass, prm->prec));
  }
  EPB_TRY(eigh_check(ctx));
  int64_t hk[2];
  EPB_CUDA(cudaMemcpyAsync(hk, nkeep_d, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(wmax_d, 0, 16, ctx->stream));
  EPB_CUDA(cudaMemsetAsync(sig_d, 0, 9 * 8, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  const int64_t nkeep = hk[0];
  int W = 0;
  int64_t nstates = 0;
  if (nkeep > 0) {
    bte_width_kernel<<<gsz(ctx, nkeep), 256, 0, ctx->stream>>>(keep, nkeep, bmin, bmax, wmax_d, nst_d);
    EPB_LAUNCH_CHECK();
    EPB_CUDA(cudaMemcpyAsync(&W, wmax_d, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    EPB_CUDA(cudaMemcpyAsync(&nstates, nst_d, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  int64_t npairs_total = 0;
  // this shard's contiguous range [ks, ke) of the kept k (the reference's mpi_comm_k split)
  int64_t ks = 0, ke = nkeep;
  if (prm->shard_count > 1) {
    const int64_t base_n = nkeep / prm->shard_count, extra = nkeep % prm->shard_count, r = prm->shard_rank;
    ks = r * base_n + std::min(r, extra);
    ke = ks + base_n + (r < extra ? 1 : 0);
  }
  if (nkeep > 0 && ke > ks && prm->shard_count > 1) {  // states of this shard
    EPB_CUDA(cudaMemsetAsync(wmax_d, 0, 16, ctx->stream));
    bte_width_kernel<<<gsz(ctx, ke - ks), 256, 0, ctx->stream>>>(keep + ks, ke - ks, bmin, bmax, wmax_d, nst_d);
    EPB_LAUNCH_CHECK();
    EPB_CUDA(cudaMemcpyAsync(&nstates, nst_d, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  } else if (ke <= ks) {
    nstates = 0;
  }
  if (nkeep > 0 && ke > ks) {
    // ---- kept-state buffers ----
    size_t off2 = 0;
    auto take2 = [&](size_t bytes) {
      size_t o = off2;
      off2 += (bytes + 255) & ~size_t(255);
      return o;
    };
    const int64_t VB = std::min<int64_t>(nkeep, 16384);  // velocity batch
    const size_t o_dop = take2(16 * 3 * nw2 * m->nr_el), o_dH = take2(16 * 3 * nw2 * VB),
                 o_v = take2(8 * 3 * nw * nkeep), o_so = take2(8 * W * nkeep), o_so_off = take2(8 * (nkeep + 1)),
                 o_uk = take2(16 * nw * W * KB), o_kR = take2(16 * (int64_t)nw * W * nm * nr_ep * KB),
                 o_fl = take2(4 * KB * N), o_pr = take2(8 * KB * N), o_seg = take2(8 * (KB + 1)),
                 o_bc = take2(4 * (cdiv(KB * N, 1024) + 1)), o_bo = take2(8 * (cdiv(KB * N, 1024) + 1)),
                 o_cnt = take2(64), o_xq = take2(24 * QCH), o_ukq = take2(16 * nw * W * QCH),
                 o_uphq = take2(16 * (int64_t)nm * nm * QCH), o_omq = take2(8 * nm * QCH), o_ikq = take2(4 * QCH),
                 o_P = take2(16 * nr_ep * QCH), o_g = take2(16 * (int64_t)nw * W * nm * QCH),
                 o_g2 = take2(8 * (int64_t)W * W * nm * QCH), o_xkb = take2(24 * std::max(VB, KB));
    const bool mixed = prm->prec == EPB_PREC_MIXED;
    const int64_t MAXG = QCH / 128 + 1;  // groups of one column chunk
    const size_t o_a2 = mixed ? take2(bte_a2_bytes(m, KB, W) + 1024) : 0, o_bq = mixed ? take2(bte_b_bytes(m, QCH) + 1024) : 0,
                 o_grp = mixed ? take2(8 * 4 * (MAXG + 1)) : 0, o_kkc = mixed ? take2(4 * QCH) : 0,
                 o_iqc = mixed ? take2(4 * QCH) : 0;
    void* ws2 = nullptr;
    EPB_TRY(ws_get(ctx, EPB_WS_PASS3, off2 + 256, &ws2));
    uint8_t* b2 = (uint8_t*)ws2;
    double2* dop = (double2*)(b2 + o_dop);
    double2* dH = (double2*)(b2 + o_dH);
    double* vel = (double*)(b2 + o_v);
    double* sout = (double*)(b2 + o_so);
    int64_t* st_off = (int64_t*)(b2 + o_so_off);
    double2* ukb = (double2*)(b2 + o_uk);
    double2* kR = (double2*)(b2 + o_kR);
    int32_t* pflag = (int32_t*)(b2 + o_fl);
    int64_t* plist = (int64_t*)(b2 + o_pr);
    int64_t* seg = (int64_t*)(b2 + o_seg);
    int32_t* bcount = (int32_t*)(b2 + o_bc);
    int64_t* boff = (int64_t*)(b2 + o_bo);
    int64_t* pcount = (int64_t*)(b2 + o_cnt);
    double* xq = (double*)(b2 + o_xq);
    double2* ukq = (double2*)(b2 + o_ukq);
    double2* uphq = (double2*)(b2 + o_uphq);
    double* omq = (double*)(b2 + o_omq);
    int32_t* ikq = (int32_t*)(b2 + o_ikq);
    double2* P = (double2*)(b2 + o_P);
    double2* g = (double2*)(b2 + o_g);
    double* g2 = (double*)(b2 + o_g2);
    double* xkb = (double*)(b2 + o_xkb);
    uint8_t* a2 = mixed ? (uint8_t*)(((uintptr_t)(b2 + o_a2) + 1023) & ~uintptr_t(1023)) : nullptr;
    uint8_t* bq = mixed ? (uint8_t*)(((uintptr_t)(b2 + o_bq) + 1023) & ~uintptr_t(1023)) : nullptr;
    int64_t* grp_d = (int64_t*)(b2 + o_grp);
    int32_t* kkc = (int32_t*)(b2 + o_kkc);
    int32_t* iqc = (int32_t*)(b2 + o_iqc);
    const bool narrow = W <= 4;
    const size_t rot_smem = (size_t)BTE_GROUPS * 16 * (nw * W + W * W * nm);
    if (mixed && narrow && rot_smem > 48 * 1024)
      EPB_CUDA(cudaFuncSetAttribute(bte_rot_acc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rot_smem));
    std::vector<int64_t> grp_h(4 * (MAXG + 1));
    EPB_CUDA(cudaMemsetAsync(sout, 0, 8 * W * nkeep, ctx->stream));

    // 3. velocities of the kept points
    Lattice L;
    for (int i = 0; i < 9; ++i) L.a[i] = prm->lattice[i];
    bte_deriv_op_kernel<<<gsz(ctx, nw2 * m->nr_el), 256, 0, ctx->stream>>>(m->ham, nw2, m->rs_el->dev, m->nr_el, L, dop);
    EPB_LAUNCH_CHECK();
    for (int64_t k0 = ks; k0 < ke; k0 += VB) {
      const int64_t kn = std::min(VB, ke - k0);
      bte_gather_x_kernel<<<gsz(ctx, kn), 256, 0, ctx->stream>>>(xg, keep, k0, kn, xkb);
      EPB_LAUNCH_CHECK();
      for (int a = 0; a < 3; ++a)
        EPB_TRY(fourier_f64(ctx, dop + (int64_t)a * nw2 * m->nr_el, nw2, nw2, m->rs_el, xkb, kn, dH + (int64_t)a * nw2 * kn,
                            nw2));
      bte_velocity_kernel<<<gsz(ctx, kn * 3 * nw), 256, 0, ctx->stream>>>(dH, kn, U, keep, k0, nw, vel);
      EPB_LAUNCH_CHECK();
    }
    std::vector<int32_t> keep_h(nkeep);
    EPB_CUDA(cudaMemcpyAsync(keep_h.data(), keep, 4 * nkeep, cudaMemcpyDeviceToHost, ctx->stream));

    // 4. batches of kept k
    BteParams bp{prm->mu, prm->temperature, prm->smearing, prm->omega_cutoff, 1.0 / (double)N, prm->method};
    const int64_t Mrows = (int64_t)nw * W * nm;
    const int64_t outk = Mrows * nr_ep;
    std::vector<int64_t> seg_h(KB + 1);
    for (int64_t b0 = ks; b0 < ke; b0 += KB) {
      const int64_t nkb = std::min(KB, ke - b0);
      bte_gather_x_kernel<<<gsz(ctx, nkb), 256, 0, ctx->stream>>>(xg, keep, b0, nkb, xkb);
      EPB_LAUNCH_CHECK();
      bte_gather_uk_kernel<<<gsz(ctx, nkb * nw * W), 256, 0, ctx->stream>>>(U, keep, b0, nkb, bmin, nw, W, ukb);
      EPB_LAUNCH_CHECK();
      if (mixed)
        EPB_TRY(bte_pack_kR(ctx, m, xkb, nkb, ukb, W, a2));
      else
        EPB_TRY(epb_eph_RR_to_kR(ctx, (const double*)m->epmat, nw, nm, nr_ep, m->rs_el, xkb, nkb, (const double*)ukb, W,
                                 nullptr, (double*)kR, EPB_PREC_FP64));
      // pairs (kk, q) with a non-empty window at k+q, ascending
      const int64_t nf = nkb * N, nb = cdiv(nf, 1024);
      bte_pair_flags_kernel<<<gsz(ctx, nf), 256, 0, ctx->stream>>>(keep, b0, nkb, ng, bmin, pflag);
      EPB_LAUNCH_CHECK();
      EPB_CUDA(cudaMemsetAsync(pcount, 0, sizeof(int64_t), ctx->stream));
      cmp_count_kernel<<<(unsigned)nb, 1024, 0, ctx->stream>>>(pflag, nf, bcount);
      EPB_LAUNCH_CHECK();
      cmp_scan_kernel<<<1, 1024, 0, ctx->stream>>>(bcount, nb, pcount, boff);
      EPB_LAUNCH_CHECK();
      cmp_scatter_kernel<<<(unsigned)nb, 1024, 0, ctx->stream>>>(pflag, nf, boff, nullptr, 0, plist, nullptr, nullptr,
                                                                   nullptr, nullptr, nf);
      EPB_LAUNCH_CHECK();
      int64_t np = 0;
      EPB_CUDA(cudaMemcpyAsync(&np, pcount, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
      EPB_CUDA(cudaStreamSynchronize(ctx->stream));
      bte_segments_kernel<<<gsz(ctx, nkb + 1), 256, 0, ctx->stream>>>(plist, np, N, nkb, seg);
      EPB_LAUNCH_CHECK();
      EPB_CUDA(cudaMemcpyAsync(seg_h.data(), seg, 8 * (nkb + 1), cudaMemcpyDeviceToHost, ctx->stream));
      EPB_CUDA(cudaStreamSynchronize(ctx->stream));
      npairs_total += np;
      if (mixed) {
        // grouped tensor-core kR->kq: column chunks of at most QCH columns, each kept k's pairs padded to 128
        int64_t kk = 0, off = 0;  // next pair of kept k kk not yet placed: seg_h[kk] + off
        while (kk < nkb) {
          int64_t ng_ = 0, tiles = 0;
          int64_t* g_t = grp_h.data();          // tile prefix (ngrp + 1)
          int64_t* g_a = g_t + (MAXG + 1);      // kept k of the group
          int64_t* g_p = g_a + (MAXG + 1);      // first pair (index into plist)
          int64_t* g_n = g_p + (MAXG + 1);      // pairs in the group
          while (kk < nkb && ng_ < MAXG - 1) {
            const int64_t left = seg_h[kk + 1] - seg_h[kk] - off;
            if (left <= 0) {
              ++kk;
              off = 0;
              continue;
            }
            const int64_t room = QCH / 128 - tiles;
            if (room <= 0) break;
            const int64_t take = std::min(left, room * 128);
            g_t[ng_] = tiles;
            g_a[ng_] = kk;
            g_p[ng_] = seg_h[kk] + off;
            g_n[ng_] = take;
            tiles += cdiv(take, 128);
            ++ng_;
            off += take;
          }
          if (ng_ == 0) break;
          g_t[ng_] = tiles;
          const int64_t ncols = tiles * 128;
          EPB_CUDA(cudaMemcpyAsync(grp_d, grp_h.data(), 8 * 4 * (MAXG + 1), cudaMemcpyHostToDevice, ctx->stream));
          const int64_t* gt_d = grp_d;
          const int64_t* ga_d = grp_d + (MAXG + 1);
          if (narrow) {  // fused rotation + accumulation, grid arrays read by index
            bte_cols_meta_kernel<<<gsz(ctx, ncols), 256, 0, ctx->stream>>>(
                gt_d, ga_d, grp_d + 2 * (MAXG + 1), grp_d + 3 * (MAXG + 1), ng_, ncols, plist, keep, b0, ng, xg, xq, kkc,
                iqc, ikq);
            EPB_LAUNCH_CHECK();
            EPB_TRY(bte_kq_grouped(ctx, m, a2, nkb, W, xq, ncols, gt_d, ga_d, ng_, bq, (float2*)g, Mrows));
            const unsigned grid = (unsigned)std::max<int64_t>(
                1, std::min<int64_t>(cdiv(ncols, BTE_GROUPS), (int64_t)ctx->sm_count * 8));
            prof_begin(ctx, EPB_PROF_ROT);
            bte_rot_acc_kernel<<<grid, 16 * BTE_GROUPS, rot_smem, ctx->stream>>>(
                (const float2*)g, Mrows, ncols, kkc, iqc, ikq, keep, b0, U, bmin, bmax, E, uph, om, nw, W, nm, bp, sout);
            prof_end(ctx);
            EPB_LAUNCH_CHECK();
            continue;
          }
          bte_cols_kernel<<<gsz(ctx, ncols), 256, 0, ctx->stream>>>(
              gt_d, ga_d, grp_d + 2 * (MAXG + 1), grp_d + 3 * (MAXG + 1), ng_, ncols, plist, keep, b0, ng, xg, U, bmin, nw,
              W, uph, om, nm, xq, ukq, uphq, omq, ikq, kkc);
          EPB_LAUNCH_CHECK();
          EPB_TRY(bte_kq_grouped(ctx, m, a2, nkb, W, xq, ncols, gt_d, ga_d, ng_, bq, (float2*)g, Mrows));
          EPB_TRY(eph_rotations_c64(ctx, (const float2*)g, Mrows, nw, W, nm, ncols, ukq, W, uphq, omq, nullptr, g2));
          bte_accumulate_cols_kernel<<<gsz(ctx, ncols * W), 256, 0, ctx->stream>>>(g2, ncols, W, nm, E, nw, keep, b0, kkc,
                                                                                ikq, bmin, bmax, omq, bp, sout);
          EPB_LAUNCH_CHECK();  // the next chunk's table upload is ordered after these kernels on the stream
        }
        continue;
      }
      for (int64_t kk = 0; kk < nkb; ++kk) {
        const int64_t s0 = seg_h[kk], nk_pairs = seg_h[kk + 1] - s0, ik = keep_h[b0 + kk];
        for (int64_t c0 = 0; c0 < nk_pairs; c0 += QCH) {
          const int64_t cn = std::min(QCH, nk_pairs - c0);
          bte_gather_q_kernel<<<gsz(ctx, cn), 256, 0, ctx->stream>>>(plist + s0 + c0, cn, ik, ng, xg, U, bmin, nw, W, uph,
                                                                     om, nm, xq, ukq, uphq, omq, ikq);
          EPB_LAUNCH_CHECK();
          EPB_TRY(launch_phase(ctx, m->rs_ep, xq, cn, P));
          EPB_TRY(zgemm_nn(ctx, kR + kk * outk, Mrows, P, nr_ep, g, Mrows, Mrows, cn, nr_ep));
          EPB_TRY(eph_rotations_f64(ctx, g, Mrows, nw, W, nm, cn, ukq, W, uphq, omq, nullptr, g2));
          bte_accumulate_kernel<<<gsz(ctx, cn * W), 256, 0, ctx->stream>>>(g2, cn, W, nm, E, nw, ik, ikq, bmin, bmax,
                                                                           omq, bp, sout + (b0 + kk) * W);
          EPB_LAUNCH_CHECK();
        }
      }
    }
    // 5. SERTA conductivity and the per-state rates
    const int64_t nsh = ke - ks;
    bte_serta_kernel<<<gsz(ctx, nsh * W), 256, 0, ctx->stream>>>(keep + ks, nsh, bmin, bmax, E, nw, W, sout + ks * W,
                                                                  vel + ks * 3 * nw, prm->mu, prm->temperature,
                                                                  1.0 / (double)N, sig_d);
    EPB_LAUNCH_CHECK();
    if (inv_tau_cap > 0) {
      bte_state_offsets_kernel<<<1, 1024, 0, ctx->stream>>>(keep + ks, nsh, bmin, bmax, st_off);
      EPB_LAUNCH_CHECK();
      bte_list_states_kernel<<<gsz(ctx, nsh), 256, 0, ctx->stream>>>(keep + ks, nsh, bmin, bmax, nw, W, sout + ks * W,
                                                                     st_off, inv_tau, inv_tau_cap);
      EPB_LAUNCH_CHECK();
    }
  }
  if (prm->prec == EPB_PREC_MIXED) EPB_TRY(split_gemm_check(ctx));
  double sh[9];
  EPB_CUDA(cudaMemcpyAsync(sh, sig_d, 9 * 8, cudaMemcpyDeviceToHost, ctx->stream));
  EPB_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 9; ++i) sigma_host[i] = sh[i] * prm->spin_degeneracy / prm->volume;
  if (stats_host) {
    stats_host[0] = nkeep;
    stats_host[1] = nstates;
    stats_host[2] = npairs_total;
    stats_host[3] = W;
  }
  return EPB_OK;
}

}  // extern "C"
