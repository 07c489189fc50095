/*
 * epb200 -- B200 (sm_100a) Wannier->Bloch electron-phonon interpolation, C ABI.
 *
 * Every entry point replaces one generic function of ElectronPhonon.jl that its CUDA package
 * extension (ext/ElectronPhononCUDAExt.jl) overrides by dispatch on CuArray, or one batched driver
 * of src/wannier_to_bloch_batched.jl; the citation next to each declaration names it (paths are
 * relative to the reference project root).
 *
 * Conventions
 *  - Arrays are column-major (Julia layout). "c128" is interleaved (re, im) double pairs, the
 *    bytes of a Julia ComplexF64 / cuDoubleComplex array. Band, mode and k indices stored in
 *    integer outputs are 1-based where the reference's are (band ranges); list indices are 0-based.
 *  - Pointers are DEVICE pointers unless the parameter name ends in `_host`.
 *  - The caller owns every input and output buffer; the library allocates only its own workspace
 *    inside the context (grown on demand, released by epb_destroy).
 *  - All work is stream-ordered on the context's stream; nothing synchronises unless stated. The
 *    caller synchronises (the reference's `synchronize(backend)`, src/common/gpu_utils.jl:60).
 *  - Every function returns an int status (EPB_OK == 0) and never aborts or throws across the ABI;
 *    epb_last_error() gives a message for the calling thread's last failure.
 *  - Threading: one context per host thread, no internal locking (the reference's batched loop is
 *    single-threaded, src/boltzmann/boltzmann_calculator.jl:332-334).
 */
#ifndef EPB200_H
#define EPB200_H

#include <stdint.h>

#if defined(__GNUC__)
#define EPB_API __attribute__((visibility("default")))
#else
#define EPB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------------- */
#define EPB_OK              0
#define EPB_ERR_ARG         1   /* bad shape, null pointer, unsupported size               */
#define EPB_ERR_OOM         2   /* workspace allocation failed                             */
#define EPB_ERR_CUDA        3   /* a CUDA runtime call or kernel launch failed             */
#define EPB_ERR_TIMEOUT     4   /* a bounded device-side wait gave up                      */
#define EPB_ERR_UNSUPPORTED 5   /* feature not available (e.g. wrong GPU architecture)     */
#define EPB_ERR_NOCONVERGE  6   /* eigensolver hit its sweep limit (results still written) */

/* ---- precision modes ----------------------------------------------------------------------- */
#define EPB_PREC_FP64   0  /* plain FP64 everywhere                                            */
#define EPB_PREC_MIXED  1  /* split-BF16 tcgen05 contractions (FP32 accumulate), FP32 eigensolve
                              with one FP64 Rayleigh-Ritz refinement                           */

typedef struct epb_ctx epb_ctx;
typedef struct epb_rset epb_rset;

/* ---- context ------------------------------------------------------------------------------- */
/* Create a context on `device`, ordering work on `stream` (a cudaStream_t; NULL = legacy default).
   Replaces: gpu_backend() (ext/ElectronPhononCUDAExt.jl:34) and the CUDA.jl handle state. */
EPB_API int epb_create(epb_ctx** ctx, int device, void* stream);
EPB_API int epb_destroy(epb_ctx* ctx);
EPB_API int epb_set_stream(epb_ctx* ctx, void* stream);
/* Free device memory as seen by the library. Replaces: free_bytes(::GPUBackend) (ext:36). */
EPB_API int epb_free_bytes(epb_ctx* ctx, uint64_t* free_host, uint64_t* total_host);
/* Block until the context's stream is idle. Replaces: synchronize(::GPUBackend) (ext:37). */
EPB_API int epb_synchronize(epb_ctx* ctx);
/* Message of the calling thread's last failure ("" if none). */
EPB_API const char* epb_last_error(void);
EPB_API int epb_version(void);
/* Bytes of workspace currently held by the context. */
EPB_API int epb_workspace_bytes(epb_ctx* ctx, uint64_t* bytes_host);
/* Number of kernels this context has launched so far (instrumentation). */
EPB_API int epb_launch_count(epb_ctx* ctx, int64_t* count_host);
/* Per-kernel-family CUDA-event timing on the context stream (the reference's @timing /
   TimerOutputs instrumentation, src/common/timer.jl:5-24). Families, in order: fourier_f64, zgemm,
   eigh, rotation, rr_rotation, umma_h, umma_kq, umma_rr, split, other, eigh_refine, tridiag,
   mlp_train, mlp_infer, pairs. epb_profile_read synchronises, returns total ms and launch counts for
   the first n families, optionally resets. eigh_refine is the FP64 refinement stage of the mixed
   eigensolver; tridiag the Householder/Sturm eigenvalue path; mlp_* the surrogate's kernels; pairs
   the (k, q) pair filter's compaction kernels. */
EPB_API int epb_profile_enable(epb_ctx* ctx, int on);
EPB_API int epb_profile_read(epb_ctx* ctx, double* ms_host, int64_t* count_host, int n, int reset);
/* Test hook: make the N-th next workspace allocation fail (N = 0 disables). Drives the
   out-of-memory path without exhausting a GPU (src/calculator/eph_device_staging.jl:33-37). */
EPB_API int epb_debug_fail_alloc(epb_ctx* ctx, int nth);

/* ---- lattice-vector sets ------------------------------------------------------------------- */
/* Upload an R-vector list (host int64 3 x nr, i.e. Julia's Vector{Vec3{Int}} bytes). Replaces:
   _irvec_to_device_matrix (src/wannier/WannierObject.jl:148-152) inside BatchedFourierCore
   (src/wannier/batched_fourier_core.jl:68-79). |R_d| must be <= 1023. */
EPB_API int epb_rset_create(epb_ctx* ctx, const int64_t* irvec_host, int64_t nr, epb_rset** rset);
EPB_API int epb_rset_destroy(epb_rset* rset);

/* ---- Fourier transform --------------------------------------------------------------------- */
/* phase[ir, j] = exp(2 pi i R_ir . x_j), c128 (nr x nk). xk: f64 (3 x nk).
   Replaces: fourier_phase! (src/wannier/batched_fourier_core.jl:24-30). */
EPB_API int epb_fourier_phase(epb_ctx* ctx, const epb_rset* rset, const double* xk, int64_t nk,
                      double* phase);

/* The same phase from the reference method's own arguments, fourier_phase!(phase, irvec_mat, xkmat)
   (src/wannier/batched_fourier_core.jl:24-30): irvec_mat f64 (nr x 3, column-major, leading dimension
   ld_r >= nr, the device matrix of _irvec_to_device_matrix, src/wannier/WannierObject.jl:148-152),
   xkmat f64 (3 x nk, column stride ld_x >= 3), phase c128 (nr x nk, column stride ld_p >= nr); strided
   column views such as P_mk[:, 1:nk_batch] (src/calculator/run_eph_over_k_and_kq.jl:821) pass their
   parent's leading dimension. R . x is rounded as the reference's broadcast, (R1 x1 + R2 x2) + R3 x3. */
EPB_API int epb_fourier_phase_mat(epb_ctx* ctx, const double* irvec_mat, int64_t ld_r, int64_t nr,
                                  const double* xkmat, int64_t ld_x, int64_t nk, double* phase, int64_t ld_p);

/* out[i, j] = sum_r op_r[i, r] exp(2 pi i R_r . x_j) for i < ndata; op_r c128 with leading
   dimension ld_op >= ndata; out c128 (ndata x nk). The phase is generated on the fly.
   Replaces: fourier_batched! / get_fourier_batched! (src/wannier/batched_fourier_core.jl:117-139,
   src/wannier/batched_interpolator.jl:200-214), i.e. the cuBLAS ZGEMM of ext/ElectronPhononCUDAExt.jl.
   prec: EPB_PREC_FP64 or EPB_PREC_MIXED (split-BF16 tensor cores, FP32 accumulate). */
EPB_API int epb_fourier(epb_ctx* ctx, const double* op_r, int64_t ld_op, int64_t ndata,
                const epb_rset* rset, const double* xk, int64_t nk, double* out, int prec);

/* ---- batched Hermitian eigensolve ---------------------------------------------------------- */
/* A: c128 (n x n x batch), Hermitian (upper triangle read), destroyed; with jobz = 'V' it is
   overwritten by the eigenvectors. E: f64 (n x batch), ascending.
   Replaces: eigvals_batched / eigen_batched (ext/ElectronPhononCUDAExt.jl:80-115; CPU method
   src/wannier_to_bloch_batched.jl:30-65). No EPW gauge fix, as in the reference's batched path.
   Returns EPB_ERR_NOCONVERGE if any matrix hit the sweep limit (outputs are still written). */
EPB_API int epb_eigh_batched(epb_ctx* ctx, double* A, int64_t n, int64_t batch, double* E, char jobz,
                     int prec);

/* Uneven batch: matrix b has order n[b] (1..96) and starts at complex element a_offset[b] of A;
   its eigenvalues go to E + e_offset[b]. All index arrays are device arrays. Same semantics. In mixed
   precision the first call of a context times the candidate kernels of each size class on a copy of the
   batch's first 32768 matrices (two workspace copies of that sample) and records the faster in the
   tuning table (eigh_varlen/...), unless the table already holds it. */
EPB_API int epb_eigh_varlen(epb_ctx* ctx, double* A, const int64_t* a_offset, const int32_t* n,
                    int64_t batch, double* E, const int64_t* e_offset, char jobz, int prec);

/* The same uneven batch with no host synchronisation and no read-back (every size-class kernel is
   launched; each takes its class from the whole batch): the call is stream-ordered and can be captured
   in a CUDA graph once an eager call of the same size has sized the context's workspace. Status
   (matrices at the sweep limit, orders outside 0..96) accumulates in the context until epb_eigh_status,
   which synchronises the context stream and returns EPB_ERR_NOCONVERGE / EPB_ERR_ARG / EPB_OK (and
   clears it). Replaces: the chunked heevjBatched loop of eigen_batched (ext/ElectronPhononCUDAExt.jl:78-115)
   for ragged batches. */
EPB_API int epb_eigh_varlen_async(epb_ctx* ctx, double* A, const int64_t* a_offset, const int32_t* n,
                                  int64_t batch, double* E, const int64_t* e_offset, char jobz, int prec);
EPB_API int epb_eigh_status(epb_ctx* ctx);

/* Phonon eigenmodes from D(q): D c128 (nm x nm x nq) is scaled by 1/sqrt(m_i m_j), diagonalised,
   and overwritten by u with u[i, :] /= sqrt(m_i); omega f64 (nm x nq) = sign(l) sqrt|l|.
   mass: f64 (nm). Replaces: the device phonon branch of compute_phonon_states
   (src/compute_states.jl:293-300) with solve_eigen_ph! semantics (src/diagonalize.jl:104-127). */
EPB_API int epb_ph_eigen_batched(epb_ctx* ctx, double* D, const double* mass, int64_t nm, int64_t nq,
                         double* omega, int prec);

/* ---- electron-phonon chain ----------------------------------------------------------------- */
/* out[iw, n, (nu, p), k] = sum_jw g(k)[iw, jw, (nu, p)] uk[jw, n, k] (* add_phase[p, k]) with
   g(k) = sum_Re epmat[:, Re] exp(2 pi i Re . x_k). epmat c128 ((nw^2 nm nr_ep) x nr_el), "el"
   layout; uk c128 (nw x nband x nk); add_phase c128 (nr_ep x nk) or NULL; out c128
   ((nw nband nm) x nr_ep x nk). Replaces: get_eph_RR_to_kR_batched!
   (src/wannier_to_bloch_batched.jl:178-205). */
EPB_API int epb_eph_RR_to_kR(epb_ctx* ctx, const double* epmat, int64_t nw, int64_t nm, int64_t nr_ep,
                     const epb_rset* rset_el, const double* xk, int64_t nk, const double* uk,
                     int64_t nband, const double* add_phase, double* out, int prec);

/* ep[m, n, nu, q] = sum_{iw, jm} conj(ukq[iw, m, q]) g[iw, n, jm, q] uph[jm, nu, q] and
   g2 = |ep|^2 / (2 omega[nu, q]). g c128 (nw x nbk x nm x nq) with column stride ldg >= nw*nbk*nm
   between q; ukq c128 (nw x nbkq x nq); uph c128 (nm x nm x nq); omega f64 (nm x nq) or NULL;
   ep_out c128 (nbkq x nbk x nm x nq) or NULL; g2_out f64 (same) or NULL.
   Replaces: eph_apply_rotations! (ext/ElectronPhononCUDAExt.jl:177-201,
   src/wannier_to_bloch_batched.jl:442-455). */
EPB_API int epb_eph_apply_rotations(epb_ctx* ctx, const double* g, int64_t ldg, int64_t nw, int64_t nbk,
                            int64_t nm, int64_t nq, const double* ukq, int64_t nbkq,
                            const double* uph, const double* omega, double* ep_out,
                            double* g2_out);

/* Strided-batched complex FP64 GEMM: C_b = op(transA, A_b) * op(transB, B_b) for b < batch (alpha = 1,
   beta = 0), op 'N' (X), 'T' (transpose) or 'C' (adjoint); A_b = A + b * strideA (c128 elements),
   column-major with leading dimension lda (likewise B, C); C_b is m x n, the inner dimension k.
   Replaces: batched_gemm! (src/common/gpu_utils.jl:71-78; CUDA method ext/ElectronPhononCUDAExt.jl:122-126,
   CUBLAS.gemm_strided_batched!). */
EPB_API int epb_batched_zgemm(epb_ctx* ctx, char transA, char transB, int64_t m, int64_t n, int64_t k,
                              const double* A, int64_t lda, int64_t strideA, const double* B, int64_t ldb,
                              int64_t strideB, double* C, int64_t ldc, int64_t strideC, int64_t batch);

/* g(k, q) = ep_kR . phase (Fourier over Rp) followed by the rotations above. ep_kR c128
   ((nw nbk nm) x nr_ep) with leading dimension ld; phase c128 (nr_ep x nq).
   Replaces: get_eph_kR_to_kq_batched! (src/wannier_to_bloch_batched.jl:245-273). */
EPB_API int epb_eph_kR_to_kq(epb_ctx* ctx, const double* ep_kR, int64_t ld, int64_t nw, int64_t nbk,
                     int64_t nm, int64_t nr_ep, const double* phase, int64_t nq,
                     const double* ukq, int64_t nbkq, const double* uph, const double* omega,
                     double* ep_out, double* g2_out, int prec);

/* ---- energy window ------------------------------------------------------------------------- */
/* For each k: band range [band_min, band_max] (1-based, inclusive; 0/0 if empty) of sorted E
   (f64 nw x nk) inside [wmin, wmax] (searchsortedfirst/last, both ends inclusive), and the
   ascending list of kept k (0-based) compacted into keep_idx (capacity nk); *nkeep_dev receives
   the count (device int64). nbelow (f64 nk or NULL) = number of bands below the window.
   Replaces: inside_window + the device branch of _filter_kpoints (src/filter.jl:19,40-72). */
EPB_API int epb_window_filter(epb_ctx* ctx, const double* E, int64_t nw, int64_t nk, double wmin,
                      double wmax, int32_t* band_min, int32_t* band_max, int32_t* keep_idx,
                      int64_t* nkeep_dev, double* nbelow);

/* FilteredStates of the window filter's band ranges on the device (src/band_states.jl:85-121): states
   ordered by k, then band; iks[i], ibands[i] (int64, 1-based; i < capacity written, either may be NULL) and
   the index map in the physical-band form the device calculators read, indmap[b - 1, k] = i + 1 for the
   states and 0 elsewhere (int64, nw x nk; _indmap_to_device, band_states.jl:283-287, builds it on the host
   and uploads it). band_min / band_max as written by epb_window_filter (0 = k not kept). counts_dev
   (device int64[3]): number of states, nband_ignore and nband of the compact FilteredStates map (the
   band_extent of k is band_min[k]:band_max[k]). Stream-ordered, no host synchronisation. */
EPB_API int epb_filtered_states(epb_ctx* ctx, const int32_t* band_min, const int32_t* band_max, int64_t nw,
                                int64_t nk, int64_t* indmap, int64_t* iks, int64_t* ibands, int64_t capacity,
                                int64_t* counts_dev);

/* The same window filter, allocating nothing: no counterpart in the reference. For callers that
   cannot let a library allocate device memory (their memory is owned by a caching allocator such as
   a Julia CUDA.jl or PyTorch pool, or a hot loop must not pay an allocation's latency or risk its
   failure). Takes a plain cudaStream_t instead of an epb_ctx. Its only scratch is a fixed 64 KB
   device array held by every GPU that loads the library until exit: nk <= 16,777,216, larger nk
   returns EPB_ERR_ARG. Calls share that array, so calls that overlap on the GPU race; calls on one
   stream are safe. The first call on a device resolves the array's address with that device
   current and should come before any stream capture; that address is kept for the life of the process,
   so after a cudaDeviceReset of a device do not call it on that device again. Results equal
   epb_window_filter's. */
EPB_API int epb_window_filter_noalloc(void* stream, const double* E, int64_t nw, int64_t nk, double wmin,
                                      double wmax, int32_t* band_min, int32_t* band_max, int32_t* keep_idx,
                                      int64_t* nkeep_dev, double* nbelow);

/* iq index (1-based) of x_{k+q} - x_k on a commensurate grid: for each j < nkq,
   iqs[j] = dense_hash_to_iq[((c1 ng2) + c2) ng3 + c3] with c = wrap(xkq_int[:, j] - xk_int).
   xkq_int int64 (3 x nkq), xk_int int64 (3), dense_hash_to_iq int64 (ng1 ng2 ng3).
   A miss (0) makes the call return EPB_ERR_ARG after the kernel (one sync). Replaces: _fill_iqs!
   (src/calculator/run_eph_over_k_and_kq.jl:565-582) and _ik_from_hash (src/common/kpoints.jl:643). */
EPB_API int epb_fill_iqs(epb_ctx* ctx, const int64_t* xkq_int, int64_t nkq, const int64_t* xk_int_host,
                 int64_t ng1, int64_t ng2, int64_t ng3, const int64_t* dense_hash_to_iq,
                 int64_t* iqs);

/* ---- band energies, energy windows and the learned pre-filter ------------------------------ */
typedef struct epb_bands epb_bands;
typedef struct epb_mlp epb_mlp;

/* Counters of one window call (host struct). tested: points (k) or pairs (k, q) considered;
   culled: pairs removed by the surrogate; evaluated: points given the plain evaluation; rechecked:
   points re-evaluated in FP64 by the mixed path's guard; kept: points / pairs with a non-empty
   window; audited: culled pairs re-evaluated by the plain path as a check of the surrogate (one in
   64 per chunk); violations: audited pairs whose window was not empty; fallback_chunks: chunks
   that, after a violation, were evaluated entirely by the plain path; screened: pairs given to the
   surrogate (the screen stops once 2^20 screened pairs have culled under a fifth of them, where
   inference costs more than it saves; the rest go to the plain evaluation directly). */
typedef struct {
  int64_t tested, culled, evaluated, rechecked, kept, audited, violations, fallback_chunks, screened;
} epb_window_stats;

/* Bind an electron Hamiltonian H(R) (c128, (nw^2, nr), caller-owned; irvec int64 3 x nr, host)
   for band-energy and window queries; builds its tensor-core operand planes once.
   Replaces: the el_ham interpolator of compute_electron_states (src/electron_state.jl:118-150). */
EPB_API int epb_bands_create(epb_ctx* ctx, const double* ham_op, int64_t nw, const int64_t* irvec_host,
                             int64_t nr, epb_bands** out);
EPB_API int epb_bands_destroy(epb_bands* bands);

/* Ascending band energies E (nw x nk) at the points xk (3 x nk): H(x) by the Fourier sum (FP64, or
   split-BF16 tensor cores for EPB_PREC_MIXED), Householder tridiagonalisation and bisection in
   FP64 (order <= 32). Replaces: get_el_eigen_valueonly_batched
   (src/wannier_to_bloch_batched.jl:75-88) for eigenvalue-only callers. */
EPB_API int epb_bands_eigvals(epb_ctx* ctx, const epb_bands* bands, const double* xk, int64_t nk, double* E,
                              int prec);

/* Energy of one band (1-based `band`) at every point of xk (3 x nk): FP64 tridiagonalisation, then
   one bisection per point. E has nk entries. */
EPB_API int epb_bands_band_energy(epb_ctx* ctx, const epb_bands* bands, const double* xk, int64_t nk, int64_t band,
                                  double* E, int prec);

/* Energy window of every point of xk (3 x nk): band_min / band_max (int32, 1-based, 0 / 0 when
   empty) = searchsortedfirst(e, wmin) / searchsortedlast(e, wmax) from Sturm counts on the
   tridiagonal, and the ascending 0-based list of kept points keep_idx (capacity nk) with its count
   in *nkeep_host (synchronises). prec FP64: exact FP64 evaluation; MIXED: tensor-core H, FP32
   counts at wmin -/+ guard and wmax -/+ guard, FP64 re-evaluation of points whose counts differ
   across a guard interval (guard in Ry, > 0). Replaces: _filter_kpoints (src/filter.jl:40-72)
   without the eigenvalue download. */
EPB_API int epb_bands_window(epb_ctx* ctx, const epb_bands* bands, const double* xk, int64_t nk, double wmin,
                             double wmax, int prec, double guard, int32_t* band_min, int32_t* band_max,
                             int32_t* keep_idx, int64_t* nkeep_host, epb_window_stats* stats_host);

/* (k, q) pair window: for every pair of the k list xk (3 x nk, normally the kept k) and the q list
   xq (3 x nq), the band range at x_k + x_q; kept pairs (non-empty range) are written in ascending
   pair order as pair index p = ik * nq + iq (int64) with band_min / band_max, up to `capacity`;
   *npairs_host = the number of kept pairs (EPB_ERR_ARG, with the count, if it exceeds capacity).
   mlp (may be NULL): a calibrated surrogate; pairs whose predicted bands all lie outside
   [wmin - margin_n, wmax + margin_n] are culled before the plain evaluation. The kept set is the
   same with and without the surrogate whenever its margins hold. Synchronises.
   Replaces: the window skip of the pair loop (src/calculator/run_eph_over_k_and_q.jl:303-307) and
   filter_qpoints (src/filter.jl:109-133). */
EPB_API int epb_pair_window(epb_ctx* ctx, const epb_bands* bands, const double* xk, int64_t nk, const double* xq,
                            int64_t nq, double wmin, double wmax, const epb_mlp* mlp, int prec, double guard,
                            int64_t* pairs, int32_t* band_min, int32_t* band_max, int64_t capacity,
                            int64_t* npairs_host, epb_window_stats* stats_host);

/* Learned band-energy surrogate (no counterpart in the reference): an MLP on Fourier features
   [cos 2 pi f.k, sin 2 pi f.k] of nf integer vectors f (int32 3 x nf, host), nhidden SiLU layers of
   width `hidden`, nout linear outputs (normalised band energies). Parameters FP32, flat layout: per
   layer W (in x out, row-major) then b (out), each block padded to a multiple of 4 floats.
   Initialised from `seed` (uniform Glorot). */
EPB_API int epb_mlp_create(epb_ctx* ctx, const int32_t* fvec_host, int64_t nf, int64_t hidden, int64_t nhidden,
                           int64_t nout, uint64_t seed, epb_mlp** out);
EPB_API int epb_mlp_destroy(epb_mlp* mlp);
EPB_API int epb_mlp_info(const epb_mlp* mlp, int64_t* nparam_host, int64_t* nin_host, int64_t* nout_host);
EPB_API int epb_mlp_get_params(epb_ctx* ctx, const epb_mlp* mlp, float* params);
EPB_API int epb_mlp_set_params(epb_ctx* ctx, epb_mlp* mlp, const float* params);
/* Target normalisation: output b predicts (E_b - mu_b) / sc_b (host arrays of nout). */
EPB_API int epb_mlp_set_scaling(epb_ctx* ctx, epb_mlp* mlp, const double* mu_host, const double* sc_host);
EPB_API int epb_mlp_get_scaling(epb_ctx* ctx, const epb_mlp* mlp, double* mu_host, double* sc_host);
/* Feature rows (n x 2 nf, FP32) of the points x (3 x n). */
EPB_API int epb_mlp_features(epb_ctx* ctx, const epb_mlp* mlp, const double* x, int64_t n, float* feat);
/* Gradient of L = sum (y_pred - (E - mu) / sc)^2 / (n nout) over the n points x (3 x n) with band
   energies E (nout x n), with respect to every parameter (FP32, nparam), and L itself (host, may be
   NULL). n a multiple of 4, at most 65536. */
EPB_API int epb_mlp_loss_grad(epb_ctx* ctx, epb_mlp* mlp, const double* x, const double* E, int64_t n, float* grad,
                              double* loss_host);
typedef struct {
  int64_t epochs;     /* passes over the training set                                        */
  int64_t batch;      /* rows per step, multiple of 16                                        */
  double lr;          /* Adam learning rate at step 0 (cosine decay to lr_final)              */
  double lr_final;
  uint64_t seed;      /* shuffle seed                                                        */
  int32_t use_graph;  /* 1: capture one epoch as a CUDA graph and replay it                  */
  int32_t reserved;
} epb_mlp_train_opts;
/* Train on n points x (3 x n) with band energies E (nout x n): per-band normalisation from E, then
   epochs x floor(n / batch) Adam steps. loss_host (epochs entries, may be NULL): mean batch loss of
   each epoch. Synchronises. */
EPB_API int epb_mlp_train(epb_ctx* ctx, epb_mlp* mlp, const double* x, const double* E, int64_t n,
                          const epb_mlp_train_opts* opts, double* loss_host);
/* Inference path: 1 (default) = BF16 tensor cores (tcgen05; layer widths multiples of 64 up to 256,
   nout a multiple of 16 up to 256, nf a multiple of 4), 0 = the FP32 kernels used in training.
   Changing it clears the calibration. epb_mlp_inference_path reports the path in use (1 or 0). */
EPB_API int epb_mlp_set_inference(epb_mlp* mlp, int mode);
EPB_API int epb_mlp_inference_path(const epb_mlp* mlp, int* path_host);
/* Predicted band energies E (nout x n, FP64) at the points x (3 x n). */
EPB_API int epb_mlp_predict(epb_ctx* ctx, const epb_mlp* mlp, const double* x, int64_t n, double* E);
/* Culling margins: margin_b = safety * max over the held-out points x (3 x n) of
   |predicted - E| for band b (E nout x n); stored in the model and returned in margin_host (nout,
   may be NULL). safety >= 1. Synchronises. */
EPB_API int epb_mlp_calibrate(epb_ctx* ctx, epb_mlp* mlp, const double* x, const double* E, int64_t n, double safety,
                              double* margin_host);

/* ---- whole e-ph pass ---------------------------------------------------------------------- */
typedef struct epb_model epb_model;

/* Bind a model's device operators (the reference's Model fields el_ham, ph_dyn, mass, epmat in the
   "el" layout; src/model.jl:24-85, src/model_new.jl:551-565) and upload the three R-vector sets.
   The operators stay caller-owned and must outlive the model. flags bit 0: also build the
   split-BF16 operand planes used by EPB_PREC_MIXED (one-time cost, like to_device,
   ext/ElectronPhononCUDAExt.jl:51-53). */
EPB_API int epb_model_create(epb_ctx* ctx, const double* ham_op, int64_t nw, const int64_t* irvec_el_host,
                             int64_t nr_el, const double* dyn_op, const double* mass, int64_t nm,
                             const int64_t* irvec_ph_host, int64_t nr_ph, const double* epmat_op,
                             const int64_t* irvec_ep_host, int64_t nr_ep, int flags, epb_model** out);
EPB_API int epb_model_destroy(epb_model* model);

/* Full-band e-ph pass over random k x random q in the q convention: electrons at k and k+q,
   phonons at q, g(k,q) = ukq^dagger g u_ph, g2 = |g|^2/(2 omega). Outputs: ek (nw x nk),
   omega (nm x nq), g2sum (nm x nk) = sum over bands and q of g2, and, if g2_sample != NULL, the full
   g2 block (nw x nw x nm) of every q with q % sample_stride == 0, laid out
   (nw, nw, nm, nsamp, nk) with nsamp = ceil(nq / sample_stride). k_batch: k per inner batch, or
   <= 0 to let the autotuner pick it (candidates 4, 8, 16, 32 timed on the first 64 k with this q list,
   then the rotation kernel and the kR->kq GEMM form; kept in the context's tuning table per (nw, nm, nq,
   prec)). stats_host (4 int64, may be NULL): [0] = g elements produced, [1] = k batch used, [2] = rotation
   kernel (0 tensor cores, 1 FP32; -1 for FP64), [3] = kR->kq form (1 A-resident, 0 streamed; -1). Replaces: the per-(k, q) loop of run_eph_over_k_and_q
   (src/calculator/run_eph_over_k_and_q.jl:251-330) run the batched way of
   _loop_eph_over_k_and_kq_batched (src/calculator/run_eph_over_k_and_kq.jl:792-892). */
/* Graph mode (off by default): epb_eph_pass runs the first call with a given argument set eagerly,
   captures the second as a CUDA graph and replays it on later calls with the same buffers and sizes
   (the production loop refills the same device buffers). Ignored on the legacy default stream and
   while profiling. */
EPB_API int epb_set_graph_mode(epb_ctx* ctx, int on);
/* Rotation kernel of the mixed pass for nw = 16, nm = 12 (the fused rotation of
   ext/ElectronPhononCUDAExt.jl:146-201 and its two-GEMM fallback): 0 = warp-level tensor cores,
   1 = FP32 CUDA cores, -1 (default) = the tuning table's choice, timed when epb_eph_pass autotunes
   (k_batch <= 0), else 0. Both give |g|^2 within the mixed path's 1e-5 per-block bar of the FP64 pass. */
EPB_API int epb_set_rotation_variant(epb_ctx* ctx, int variant);

/* ---- tuning table -------------------------------------------------------------------------- */
/* The autotuner's measured choices, keyed by shape, replacing the reference's fixed crossovers
   _FUSED_ROT_MAX_NWNM (src/wannier_to_bloch_batched.jl:406) and _FUSED_RQKQ_MAX_NW2NM
   (ext/ElectronPhononCUDAExt.jl:214) with timings on the caller's shapes. Keys (all per nw, nm, nq,
   prec): pass_kb/... inner k batch of epb_eph_pass, pass_rot/... rotation kernel (0 tensor cores,
   1 FP32), pass_kq/... kR->kq GEMM form (1 A-resident, 0 streamed); eigh_varlen/<lo>/<hi>/<prec>: the
   kernel of a mixed uneven-eigensolve size class (lo, hi] (1 the L2-scratch instance for the class, 0 the
   shared-memory or 512-thread solver), timed by the first epb_eigh_varlen call of a context on a copy of
   the first 32768 matrices of its batch (epb_eigh_varlen_async only reads the table). A table is host memory only; its
   text form is one "key value" pair per line ('#' comment lines allowed). epb_tune_export copies a
   context's choices into a table, epb_tune_import loads a table's choices into a context (later calls
   of those shapes then use them without timing). get: *found = 0 when the key is absent. serialize:
   *len = text length; EPB_ERR_ARG (nothing written) when cap <= *len. parse: a malformed line rejects
   the whole text, the table unchanged. */
typedef struct epb_tune_table epb_tune_table;
EPB_API int epb_tune_table_create(epb_tune_table** table);
EPB_API int epb_tune_table_destroy(epb_tune_table* table);
EPB_API int epb_tune_table_set(epb_tune_table* table, const char* key, int64_t value);
EPB_API int epb_tune_table_get(const epb_tune_table* table, const char* key, int64_t* value, int* found);
EPB_API int epb_tune_table_size(const epb_tune_table* table, int64_t* n);
EPB_API int epb_tune_table_serialize(const epb_tune_table* table, char* buf, int64_t cap, int64_t* len);
EPB_API int epb_tune_table_parse(epb_tune_table* table, const char* text);
EPB_API int epb_tune_export(epb_ctx* ctx, epb_tune_table* table);
EPB_API int epb_tune_import(epb_ctx* ctx, const epb_tune_table* table);
EPB_API int epb_eph_pass(epb_ctx* ctx, epb_model* model, const double* xk, int64_t nk, const double* xq,
                         int64_t nq, int prec, int64_t k_batch, int64_t sample_stride, double* ek_out,
                         double* omega_out, double* g2sum_out, double* g2_sample, int64_t* stats_host);

/* ---- outer-q loop ----------------------------------------------------------------------------- */
/* "el" layout (nw^2 nm nr_ep rows (i, j, nu, Rp), nr_el columns Re) -> "ph" layout (nw^2 nm nr_el rows
   (i, j, nu, Re), nr_ep columns Rp), c128: permutedims [1,2,3,5,4] of src/model.jl:80-81,293-296. */
EPB_API int epb_epmat_el_to_ph(epb_ctx* ctx, const double* epmat_el, int64_t nw, int64_t nm, int64_t nr_el,
                               int64_t nr_ep, double* epmat_ph);
/* g(Re, q) for each q of xq (3 x nq): the Fourier sum over Rp of the "ph"-layout epmat_ph, then the mode
   rotation by uph (nm x nm x nq); out (nw^2 nm x nr_el x nq), rows (i, j, nu). Replaces:
   get_eph_RR_to_Rq! (src/wannier_to_bloch.jl:277-300) for a list of q. */
EPB_API int epb_eph_RR_to_Rq(epb_ctx* ctx, const double* epmat_ph, int64_t nw, int64_t nm, int64_t nr_el,
                             const epb_rset* rset_ph, const double* xq, int64_t nq, const double* uph, double* out,
                             int prec);
/* For one q: g(k, q) = sum_Re e^{2 pi i k.Re} g(Re, q) at each k of xk (3 x nk) (g_Rq from
   epb_eph_RR_to_Rq, rset_el its Re set), then ep[m, n, nu, k] = sum conj(ukq[iw, m, k]) g[iw, jw, nu, k]
   uk[jw, n, k] (uks (nw, nbk, nk), ukqs (nw, nbkq, nk)); outputs ep (nbkq, nbk, nm, nk) and/or
   g2 = |ep|^2 / (2 omega_nu) (omega: nm values of this q). Replaces: get_eph_Rq_to_kq_batched! +
   eph_apply_rotations_rqkq! (src/wannier_to_bloch_batched.jl:317-377, ext:206-258). */
EPB_API int epb_eph_Rq_to_kq(epb_ctx* ctx, const double* g_Rq, int64_t nw, int64_t nm, const epb_rset* rset_el,
                             const double* xk, int64_t nk, const double* uks, int64_t nbk, const double* ukqs,
                             int64_t nbkq, const double* omega, double* ep_out, double* g2_out, int prec);

/* Outer-q batched loop (src/calculator/run_eph_over_q_and_k.jl:428-613): for each q, g(Re, q) from the
   "ph"-layout epmat (made once per model from the "el" layout) and the phonon eigenmodes at q; then per
   batch of kept k (k with a non-empty window_k range; eigenvectors zero outside it): H(k+q), its eigen,
   eigenvector columns outside window_kq set to zero, ep = ukq^H g(k, q) uk, and the calculators'
   run_batch with the EPDataKBatched payload (src/EPData.jl:76-114). A_out[iq] (optional, host) receives
   the gauge-invariant record sum_k wtk sum_{m, n, nu} |ep|^2. */
typedef struct epb_outer_q_params {
  double wmin_k, wmax_k;    /* k window (window_k) */
  double wmin_kq, wmax_kq;  /* k+q window (window_kq) */
  int64_t k_batch;          /* kept k per batch; <= 0: min(nk kept, 4096) (nk_batch_max) */
  int64_t q_chunk;          /* q per RR->Rq launch; <= 0: as many as fit 1 GiB of g(Re, q) */
  int prec;                 /* EPB_PREC_FP64, or EPB_PREC_MIXED (FP32 + FP64-refined eigensolves, split-BF16
                               Fourier over Re) */
  int phonon_basis;         /* 0 eigenmode, 1 Cartesian (u_ph = identity) (eph_phonon_basis) */
} epb_outer_q_params;

/* EPDataKBatched (src/EPData.jl:76-114) plus the batch position; device pointers valid until run_batch
   returns; work that reads them must be ordered on `stream` (the context's). */
typedef struct epb_kbatch_payload {
  int64_t iq, k0, nk;  /* q index, first kept-k index of the batch, batch width */
  int64_t nw, nm;
  const double* eps;   /* (nw, nw, nm, nk) c128, out-of-window bands zero */
  const double* ek;    /* (nw, nk) */
  const double* ekq;   /* (nw, nk) */
  const double* uk;    /* (nw, nw, nk) c128, zero outside the k window */
  const double* ukq;   /* (nw, nw, nk) c128, zero outside the k+q window */
  const double* wtk;   /* (nk) */
  const double* xk;    /* (3, nk) */
  const int32_t* ik;   /* (nk) index of each k in the caller's k list */
  const double* omega; /* (nm) phonon frequencies at q */
  void* stream;        /* cudaStream_t */
} epb_kbatch_payload;

/* One calculator: calculator_begin!/end!(OuterIteration) and run_calculator!(::EPDataKBatched)
   (src/calculator/AbstractCalculator.jl). A non-zero return aborts the loop with EPB_ERR_ARG. */
typedef struct epb_outer_q_calc {
  int (*begin_q)(void* user, int64_t iq, void* stream);
  int (*run_batch)(void* user, const epb_kbatch_payload* p);
  int (*end_q)(void* user, int64_t iq, void* stream);
  void* user;
} epb_outer_q_calc;

/* xk_host (3 x nk), wtk_host (nk, NULL: 1), xq_host (3 x nq) on the host; stats_host (4): kept k, k batch,
   q chunk, batches. */
EPB_API int epb_eph_outer_q(epb_ctx* ctx, epb_model* model, const double* xk_host, const double* wtk_host, int64_t nk,
                            const double* xq_host, int64_t nq, const epb_outer_q_params* params,
                            const epb_outer_q_calc* calcs, int ncalc, double* A_out, int64_t* stats_host);

/* ---- calculator hooks of the batched loop -------------------------------------------------- */
/* Window scatter of one batch into a device-resident calculator buffer: for every (m, n, nu, j) of
   g2vals (nbandkq, nbandk, nm, nq_batch), i = imap_i_col[n], f = imap_f[m, ikqs[j]] (Int64, 1-based,
   0 = out of window; imap_f column-major with leading dimension ld_imap_f); when both are > 0,
   g2_out / omega_out at the 1-based slot nu + nm (i - i0 - 1) + nm ni_stride (f - 1) receive
   g2vals[m, n, nu, j] / omega[nu, j]. Slots are unique across a run (no atomics).
   Replaces: eph_window_scatter! (src/calculator/calculator_utils.jl:36-50, ext:280-313). */
EPB_API int epb_eph_window_scatter(epb_ctx* ctx, double* g2_out, double* omega_out, const double* g2vals,
                                   const int64_t* imap_i_col, const int64_t* imap_f, int64_t ld_imap_f,
                                   const int64_t* ikqs, const double* omega, int64_t nbandkq, int64_t nbandk,
                                   int64_t nm, int64_t nq_batch, int64_t ni_stride, int64_t i0);
/* Boltzmann accumulation of one batch: for every (m, n, j) with i = imap_i_at_k[n] > 0 and
   f = imap_f[m, ikqs[j]] > 0, and every temperature iT, the increments of
   bte_scattering_increments(method, e_i[i], e_f[f], omega[nu, j], g2vals[m, n, nu, j], wf[f],
   mus[iT], ts[iT], etas[iT]) summed over modes with omega >= omega_cutoff:
   sout[i, iT] += s_out (sout (n_i, nT)); sin[i - i0, f, iT] = s_in (sin (ni_tile, n_f, nT), may be
   NULL). Replaces: bte_window_accumulate! (src/boltzmann/boltzmann_calculator.jl:336-362,
   ext:323-372). */
EPB_API int epb_bte_window_accumulate(epb_ctx* ctx, double* sout, int64_t n_i, double* sin, int64_t ni_tile,
                                      int64_t n_f, const double* g2vals, const double* omega,
                                      const int64_t* imap_i_at_k, const int64_t* imap_f, int64_t ld_imap_f,
                                      const int64_t* ikqs, const double* e_i, const double* e_f, const double* wf,
                                      const double* mus, const double* ts, const double* etas, int64_t nT,
                                      int method, double omega_cutoff, int64_t nbandkq, int64_t nbandk,
                                      int64_t nmodes, int64_t nq_batch, int64_t i0);

/* ---- EPW reader ------------------------------------------------------------------------------ */
/* Reads `<prefix>.epmatwp` (raw complex128, EPW order (iw, jw, iRe, imode, iRp)) into `out` (device,
   nw^2 nmodes nr_ep x nr_el for layout 0 = "el", nw^2 nmodes nr_el x nr_ep for layout 1 = "ph"), applying
   the R sort (ind_el, ind_ep: Julia sortperm, 1-based, new <- old) and the Wigner-Seitz divisions with the
   sorted degeneracy arrays: ndegen_ep (ndegen_ep_dim1 x ndegen_ep_dim2 x nr_ep, (1, 1) or (nw, nat))
   unless skip_ndegen_ep or ndegen_pre_divided, then ndegen_el (d x d x nr_el, d = 1 or nw) unless
   ndegen_pre_divided; zero where a degeneracy is 0. Replaces: read_epmat (src/model_new.jl:487-568). */
EPB_API int epb_read_epmat(epb_ctx* ctx, const char* filename, int64_t nw, int64_t nmodes, int64_t nr_el,
                           int64_t nr_ep, const int64_t* ind_el, const int64_t* ind_ep, const int32_t* ndegen_el,
                           int64_t ndegen_el_dim, const int32_t* ndegen_ep, int64_t ndegen_ep_dim1,
                           int64_t ndegen_ep_dim2, int skip_ndegen_ep, int ndegen_pre_divided, int layout,
                           double* out);

/* ---- tiled device output of the batched calculators ---------------------------------------- */
/* TiledDeviceOutput (src/calculator/tiled_device_output.jl): narr arrays (elements of elem_bytes = 4, 8 or
   16) of the column-major shape dims, axis i_axis (0-based) running over the outer states; iks (n_states,
   host) the 1-based k index of each state, nk k points, batches of at most n_batch_max k. force_block: -1
   decide from free device memory (block when headroom x the full bytes exceed it), 0 whole output resident,
   1 one outer-k tile at a time. The scatter into epb_tiled_device_array uses tile_offset / tile_stride. */
typedef struct epb_tiled epb_tiled;
typedef struct epb_tiled_info {
  int allocated, block;
  int64_t ni_cap;       /* tile capacity along the tiled axis (block mode) */
  int64_t tile_offset;  /* global state offset of the current tile (0 in full mode) (tile_offset) */
  int64_t tile_length;  /* states in the current tile (tile_length) */
  int64_t tile_stride;  /* the buffers' extent along the tiled axis (tile_stride) */
} epb_tiled_info;
/* (first, last) 1-based states of the k range kstart:kend, (1, 0) when empty; EPB_ERR_ARG when they are not
   contiguous. Replaces: ind_range_for_k_range (src/band_states.jl:416-428). Host only. */
EPB_API int epb_ind_range_for_k_range(const int64_t* iks, int64_t n, int64_t nk, int64_t kstart, int64_t kend,
                                      int64_t* first, int64_t* last);
/* The block-mode tile capacity: the largest state count of the k batches 1:n_batch_max, ... Host only. */
EPB_API int epb_tiled_plan(const int64_t* iks, int64_t n, int64_t nk, int64_t n_batch_max, int64_t* ni_cap);
/* residency_use_block (tiled_device_output.jl:59-60). */
EPB_API int epb_residency_use_block(epb_ctx* ctx, int64_t full_bytes, double headroom, int* use_block);
EPB_API int epb_tiled_create(epb_ctx* ctx, const int64_t* dims, int ndims, int i_axis, int narr, int64_t elem_bytes,
                             int force_block, double headroom, const int64_t* iks, int64_t n_states, int64_t nk,
                             int64_t n_batch_max, epb_tiled** out);
/* tile_begin! for the 1-based k batch kstart:kend: the first call decides residency and allocates; in block
   mode each call sets the tile range and zeroes its region. */
EPB_API int epb_tiled_begin(epb_ctx* ctx, epb_tiled* t, int64_t kstart, int64_t kend);
EPB_API int epb_tiled_get_info(const epb_tiled* t, epb_tiled_info* info);
EPB_API int epb_tiled_device_array(const epb_tiled* t, int k, void** ptr);
/* tile_download!: array k to host (block: the current tile, extent tile_length along the tiled axis,
   contiguous; full: the whole array); synchronises the context stream. */
EPB_API int epb_tiled_download(epb_ctx* ctx, const epb_tiled* t, int k, void* host);
/* tile_free!: release the buffers and the residency decision (the object can be reused). */
EPB_API int epb_tiled_free(epb_tiled* t);
EPB_API int epb_tiled_destroy(epb_tiled* t);

/* ---- SERTA Boltzmann consumer -------------------------------------------------------------- */
typedef struct {
  int64_t ngrid;            /* k = q grid ngrid^3 (commensurate), k fastest (kpoints.jl:135-153)   */
  double wmin, wmax;        /* energy window (Ry) of the initial and final electron states         */
  double mu, temperature;   /* chemical potential, temperature (Ry)                                */
  double smearing;          /* Gaussian width (Ry)                                                */
  double omega_cutoff;      /* phonon modes below it are skipped (Ry; constants.jl:5)               */
  double spin_degeneracy;
  double volume;            /* unit-cell volume                                                  */
  double lattice[9];        /* column-major, column d = lattice vector a_d (Cartesian)            */
  int32_t method;           /* occupation method 1..6 (bte_scattering_core.jl:9-84)               */
  int32_t prec;             /* EPB_PREC_FP64, or EPB_PREC_MIXED: g(k, Rp) on the tensor cores (model
                               created with the mixed flag), everything else FP64                  */
  int64_t k_batch;          /* kept k per batch (<= 256); <= 0: 128                              */
  int64_t pair_chunk;       /* (k, q) pairs per rotation launch, a multiple of 128; <= 0: 65536   */
  int64_t shard_rank;       /* this rank's share of the kept k (contiguous ranges, sizes within one)  */
  int64_t shard_count;      /* number of shards (ranks); <= 1: all kept k. Each shard's sigma is a
                               partial sum: the shards' sigmas add up to the whole (one 9-value
                               all-reduce); inv_tau and the state / pair counts are the shard's */
} epb_bte_params;

/* SERTA conductivity over commensurate k = q grids: electron states, windows and phonons on the grid,
   band velocities (Hellmann-Feynman with dH/dk from the Fourier sum), |g|^2 of every in-window
   (n at k, m at k+q, nu) triple in the q convention, out-scattering rates S_out[n, k] from the
   occupation increments with Gaussian smearing and weight 1/N per final state, and
   sigma_ab = (spin / V) sum_{k, n in window} (1/N) (-f'(e - mu) / S_out) v_a v_b (host, 9 values,
   column-major). inv_tau (device, capacity inv_tau_cap, may be NULL with capacity 0): S_out of the
   window states, kept k ascending then band ascending. stats_host (4 int64, may be NULL): kept k,
   window states, (k, q) pairs with a non-empty k+q window, widest window. Synchronises.
   Replaces: the batched k / k+q loop with the Boltzmann calculator
   (src/calculator/run_eph_over_k_and_kq.jl:792-892, src/boltzmann/boltzmann_calculator.jl:336-362)
   and the SERTA conductivity of solve_electron_bte (src/boltzmann/electron_lbte.jl:43-49,153-185). */
EPB_API int epb_bte_serta(epb_ctx* ctx, epb_model* model, const epb_bte_params* params, double* sigma_host,
                          double* inv_tau, int64_t inv_tau_cap, int64_t* stats_host);

#ifdef __cplusplus
}
#endif
#endif /* EPB200_H */
