// gram_tc.cu — tensor-core (tcgen05) Gram of the centred per-sample Jacobian.
#include "minsr.cuh"

namespace nqs {

size_t gram_tc_workspace(int W, int64_t P, int prec) {
  (void)W; (void)P; (void)prec;
  return 0;
}

int gram_tc(const void* O, int o_dtype, const double* mu, int W, int64_t P, int prec, double* T,
            Arena& ws, int nsm, cudaStream_t st) {
  (void)O; (void)o_dtype; (void)mu; (void)W; (void)P; (void)prec; (void)T; (void)ws; (void)nsm;
  (void)st;
  set_error("tensor-core Gram not built yet");
  return NQS_ERR_UNSUPPORTED;
}

}  // namespace nqs
