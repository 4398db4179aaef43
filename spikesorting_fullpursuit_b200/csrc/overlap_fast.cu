// overlap_fast.cu -- screened overlap recheck (filled in after the exact path).
#include "fbp_internal.cuh"

namespace fbp {

int launch_overlap_fast(const Dims& d, const Work& w, const float* V, const float* T, const float* theta,
                        uint32_t nflag_max, cudaStream_t st)
{
    return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
}

}  // namespace fbp
