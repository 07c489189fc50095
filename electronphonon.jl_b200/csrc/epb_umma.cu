// Split-BF16 tensor-core (tcgen05) Fourier path: placeholder until the sm_100a kernel lands.
#include "epb_common.cuh"

namespace epb {

int fourier_mixed(epb_ctx* ctx, const double2* op, int64_t ld, int64_t M, const epb_rset* rs,
                  const double* xk, int64_t N, double2* out, int64_t ldo) {
  (void)ctx; (void)op; (void)ld; (void)M; (void)rs; (void)xk; (void)N; (void)out; (void)ldo;
  set_error("epb_fourier: EPB_PREC_MIXED is not available in this build");
  return EPB_ERR_UNSUPPORTED;
}

}  // namespace epb
