// separability.cu -- per-template noise model of the pursuit's thresholds, on the device.
//
// compute_separability_metrics + set_bp_threshold
// (spikesorting_fullpursuit/overlap/neuron_separability.py:113-195, 319-331) give
// binary_pursuit its bias (-0.5 * template_SS) and accept thresholds.  Per
// template n (one CTA):
//   template_SS[n]   = np.sum(T[n] ** 2) in the templates' type, numpy's pairwise order
//   variance[n]      = sum_c T[n,c,:] Cov_c T[n,c,:]^T        (FP64)
//   expectation      = 0.5 * template_SS[n]                   (same type)
//   lower_CI[n]      = expectation - sigma_bp_CI * sqrt(variance)
//   threshold[n]     = -expectation + sigma_bp_noise * sqrt(variance)
//   peak_channel[n]  = argmax |T[n]| // W  (first maximum)
//   contamination[n] = P(N(-expectation, sqrt(variance)) > threshold)
//                    = 0.5 erfc((threshold + expectation) / (sqrt(variance) sqrt 2))
// and, with set_bp_threshold, threshold = max(threshold, 0, lower_CI).
// The quadratic forms are summed in a fixed tree order in FP64 (numpy's
// matrix products use BLAS, whose order is not specified), so variances agree
// with the reference to FP64 rounding, not bit for bit.
#include <cub/cub.cuh>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sq(const float* a, uint32_t i) { return __fmul_rn(a[i], a[i]); }
__device__ __forceinline__ double sq(const double* a, uint32_t i) { return __dmul_rn(a[i], a[i]); }

// numpy's pairwise sum of a[i]^2 over [0, n) in the array's own type
template <class F>
__device__ F pairwise_sq_sum(const F* a, uint32_t n)
{
    if (n < 8) {
        F res = 0;
        for (uint32_t i = 0; i < n; ++i) res = add_rn(res, sq(a, i));
        return res;
    }
    if (n <= 128) {
        F r[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = sq(a, j);
        uint32_t i = 8;
        for (; i < n - (n % 8); i += 8) {
#pragma unroll
            for (int j = 0; j < 8; ++j) r[j] = add_rn(r[j], sq(a, i + j));
        }
        F res = add_rn(add_rn(add_rn(r[0], r[1]), add_rn(r[2], r[3])), add_rn(add_rn(r[4], r[5]), add_rn(r[6], r[7])));
        for (; i < n; ++i) res = add_rn(res, sq(a, i));
        return res;
    }
    uint32_t n2 = n / 2;
    n2 -= n2 % 8;
    return add_rn(pairwise_sq_sum(a, n2), pairwise_sq_sum(a + n2, n - n2));
}

__device__ __forceinline__ uint32_t abs_bits(float x) { return __float_as_uint(fabsf(x)); }
__device__ __forceinline__ unsigned long long abs_bits(double x)
{
    return (unsigned long long)__double_as_longlong(fabs(x));
}

constexpr int kSepThreads = 256;

struct SepOut {
    void* ss;   // template_SS in the templates' own type
    double* variance;
    double* lower_ci;
    double* threshold;
    double* contamination;
    int64_t* peak;
};

template <class F>
__global__ void __launch_bounds__(kSepThreads) separability_kernel(const F* __restrict__ T,
                                                                   const double* __restrict__ cov, uint32_t C,
                                                                   uint32_t W, double sigma_noise, double sigma_ci,
                                                                   int apply_bp_threshold, SepOut out)
{
    typedef cub::BlockReduce<double, kSepThreads> RD;
    __shared__ typename RD::TempStorage rd;
    __shared__ unsigned long long s_bits;
    __shared__ uint32_t s_idx;
    const uint32_t n = blockIdx.x;
    const F* t = T + (uint64_t)n * C * W;
    // FP64 quadratic forms: thread-strided partial sums over (c, i), each a row
    // of Cov_c against the template, then one block reduction
    double part = 0.0;
    for (uint64_t e = threadIdx.x; e < (uint64_t)C * W; e += blockDim.x) {
        const uint32_t c = (uint32_t)(e / W), i = (uint32_t)(e % W);
        const double* row = cov + ((uint64_t)c * W + i) * W;
        const F* tc = t + (uint64_t)c * W;
        double r = 0.0;
        for (uint32_t j = 0; j < W; ++j) r = fma(row[j], (double)tc[j], r);
        part = fma((double)tc[i], r, part);
    }
    const double var = RD(rd).Sum(part);
    // first maximum of |T[n]|: largest magnitude bits, then the lowest index
    if (threadIdx.x == 0) { s_bits = 0ull; s_idx = 0xFFFFFFFFu; }
    __syncthreads();
    unsigned long long bb = 0ull;
    uint32_t bi = 0xFFFFFFFFu;
    for (uint32_t e = threadIdx.x; e < C * W; e += blockDim.x) {
        const unsigned long long b = abs_bits(t[e]);
        if (bi == 0xFFFFFFFFu || b > bb) { bb = b; bi = e; }
    }
    if (bi != 0xFFFFFFFFu) atomicMax(&s_bits, bb);
    __syncthreads();
    if (bi != 0xFFFFFFFFu && bb == s_bits) atomicMin(&s_idx, bi);
    __syncthreads();
    if (threadIdx.x == 0) {
        const F ss = pairwise_sq_sum(t, C * W);
        const F expectation = (F)0.5 * ss;   // exact (a power of two)
        const double sd = sqrt(var);
        const double lower_ci = (double)expectation - sigma_ci * sd;
        double thr = (double)(-expectation) + sigma_noise * sd;
        // norm.sf(thr, -expectation, sd) = ndtr(-(thr + expectation) / sd); scipy gives NaN for sd == 0
        const double z = (thr + (double)expectation) / sd;
        out.contamination[n] = sd > 0.0 ? 0.5 * erfc(z * 0.70710678118654752440) : __longlong_as_double(0x7ff8000000000000ll);
        if (apply_bp_threshold) {
            thr = thr > 0.0 ? thr : 0.0;
            thr = thr > lower_ci ? thr : lower_ci;
        }
        static_cast<F*>(out.ss)[n] = ss;
        out.variance[n] = var;
        out.lower_ci[n] = lower_ci;
        out.threshold[n] = thr;
        out.peak[n] = (int64_t)(s_idx / W);
    }
}

}  // namespace
}  // namespace fbp

using namespace fbp;

extern "C" int fbp_separability(const void* templates, int templates_f64, const double* channel_cov,
                                uint32_t n_templates, uint32_t n_chans, uint32_t template_len, double sigma_bp_noise,
                                double sigma_bp_ci, int apply_bp_threshold, void* template_ss, double* variance,
                                double* lower_ci, double* threshold, double* contamination, int64_t* peak_channel,
                                void* stream)
{
    set_error("");
    if (n_templates == 0) return FBP_OK;
    if (n_chans == 0 || template_len == 0) return fail(FBP_E_ARG, "invalid sizes");
    if ((uint64_t)n_chans * template_len >= (1ull << 31)) return fail(FBP_E_ARG, "template too long");
    if (!templates || !channel_cov || !template_ss || !variance || !lower_ci || !threshold || !contamination ||
        !peak_channel)
        return fail(FBP_E_ARG, "null pointer argument");
    SepOut out{template_ss, variance, lower_ci, threshold, contamination, peak_channel};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (templates_f64)
        separability_kernel<double><<<n_templates, kSepThreads, 0, st>>>(
            static_cast<const double*>(templates), channel_cov, n_chans, template_len, sigma_bp_noise, sigma_bp_ci,
            apply_bp_threshold, out);
    else
        separability_kernel<float><<<n_templates, kSepThreads, 0, st>>>(
            static_cast<const float*>(templates), channel_cov, n_chans, template_len, sigma_bp_noise, sigma_bp_ci,
            apply_bp_threshold, out);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}
