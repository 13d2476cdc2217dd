// fx_gemm_tc.cu -- tensor-core (tcgen05) NT GEMMs for the DCT stage.
#include "fx_internal.h"
#include "fx_gemm.cuh"

namespace fx {

int gemm_nt_tc(fx_ctx *ctx, int precision, int G, const GemmOperands &A,
               const GemmOperands &B, const float *S, const GemmOperands &D,
               cudaStream_t s) {
  (void)ctx; (void)G; (void)A; (void)B; (void)S; (void)D; (void)s;
  set_error("gemm_nt: precision %d is not available in this build", precision);
  return FX_EINVAL;
}

}  // namespace fx
