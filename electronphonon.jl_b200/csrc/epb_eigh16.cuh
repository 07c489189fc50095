// Arguments of the batched 16x16 (n <= 16) Hermitian eigensolver, shared by its kernels (one half-warp per
// matrix) and by the general eigensolver's dispatch, which routes the small orders to it.
#pragma once

#include "epb_common.cuh"

namespace epb {

struct Eigh16Args {
  const double2* A;   // c128 input (n x n per matrix, upper triangle), or null
  const float* Hp;    // packed FP32 Hermitian input (n*n per matrix), or null
  double2* U64;       // c128 eigenvector output (may alias A), or null
  float2* U32;        // c64 eigenvector output, or null
  double* E;          // eigenvalues (n per matrix), or null
  const double* mass; // phonon mode: scale by 1/sqrt(m_i m_j), omega = sign sqrt, u /= sqrt(m)
  int n;
  int64_t batch;
  int max_sweeps;
  int* nonconv;
  int refine;         // FP64 refinement iterations (mixed only)
  int64_t* flag_list; // if non-null: matrices with a near-degenerate pair are listed, not written
  int* flag_count;
  float2* V32;        // FP32 eigenvector workspace between the Jacobi and refinement kernels
  float angle_stop;   // mixed: the FP32 sweeps end after a sweep whose rotation angles all stay below it
  // complex64 refinement: matrices whose smallest eigenvalue gap lies in [1e-6, gap_rel) * max |lambda| are
  // listed (gap_list[0 .. gap_cap), count in *gap_count) for the FP64 re-solve of eigh16_fixup_launch; a
  // count above gap_cap leaves the excess with their mixed-precision vectors
  int64_t* gap_list;
  int* gap_count;
  int gap_cap;
  float gap_rel;
};

int eigh16_launch(epb_ctx* ctx, Eigh16Args& a, bool mixed);

// FP64 re-solve of the matrices listed by the complex64 refinement: H(x) = sum_R H(R) exp(2 pi i R.x) formed
// in FP64 at x = xk[b / nq] + xq[b % nq] for each listed matrix b, FP64 one-sided Jacobi, the sorted
// eigenvectors written over U32 (16 x 16 per matrix). The list count is read on the device.
int eigh16_fixup_launch(epb_ctx* ctx, const int64_t* list, const int* count, int cap, const double2* ham,
                        const int4* rv, int64_t nr, const double* xk, const double* xq, int64_t nq, float2* U32,
                        double2* hbuf);

}  // namespace epb
