// Tensor-core (tcgen05) Legendre stage: placeholder until the split-precision
// kernels land; plans asking for SHT_PREC_BF16X3 / SHT_PREC_FP16X3 fail with
// SHT_EUNSUPPORTED.
#include "sht_internal.h"

namespace sht {
int tc_supported() { return 0; }
cudaError_t tc_prepare(Plan&) { return cudaErrorNotSupported; }
void tc_release(Plan&) {}
cudaError_t launch_legendre_synthesis_tc(const Plan&, const float2*, int64_t, int, cudaStream_t) {
    return cudaErrorNotSupported;
}
cudaError_t launch_legendre_analysis_tc(const Plan&, float2*, int64_t, int, bool, cudaStream_t) {
    return cudaErrorNotSupported;
}
}  // namespace sht
