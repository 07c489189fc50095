// Split-BF16 tensor-core (tcgen05) Fourier path: placeholder until the sm_100a kernel lands.
#include "epb_common.cuh"

struct epb_model;

namespace epb {

int fourier_mixed(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                  const double* xk, int64_t N, double2* out, int64_t ldo) {
  (void)ctx; (void)op; (void)ld; (void)M; (void)rs; (void)xk; (void)N; (void)out; (void)ldo;
  set_error("epb_fourier: EPB_PREC_MIXED is not available in this build");
  return EPB_ERR_UNSUPPORTED;
}

int mixed_model_prepare(epb_ctx* ctx, epb_model* m) {
  (void)ctx; (void)m;
  set_error("mixed-precision planes are not available in this build");
  return EPB_ERR_UNSUPPORTED;
}

void mixed_model_free(epb_model* m) { (void)m; }

int mixed_pass_batch(epb_ctx* ctx, epb_model* m, const double* xk_b, int64_t nkb, const double* xq,
                     int64_t nq, const double2* uk_b, const double2* uph, const double* omega,
                     const double2* phase, double* g2sum_b, double* g2_sample_b, int64_t sample_stride,
                     int64_t* stats) {
  set_error("mixed-precision pass is not available in this build");
  return EPB_ERR_UNSUPPORTED;
}

}  // namespace epb
