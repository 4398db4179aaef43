// lik_tc.cu -- tensor-core likelihood (filled in after the exact path).
#include "fbp_internal.cuh"

namespace fbp {

bool tc_supported(const Dims&) { return false; }

int launch_likelihood_tc(const Dims&, const Work&, const float*, const float*, const float*,
                         const uint32_t*, uint32_t, float*, bool, cudaStream_t, uint64_t*)
{
    return fail(FBP_E_ARG, "tensor-core likelihood not available");
}

int launch_tc_prepare_templates(const Dims&, const Work&, const float*, cudaStream_t) { return FBP_OK; }

int launch_tc_update_voltage(const Dims&, const Work&, const float*, const uint32_t*, const uint32_t*,
                             uint32_t, bool, cudaStream_t)
{
    return FBP_OK;
}

}  // namespace fbp
