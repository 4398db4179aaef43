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

// ---- pairwise_separability (neuron_separability.py:348-444) ----
//
// Per pair (n1, n2), one CTA:
//   shift      first arg-max over lags k in [-max_shift, max_shift] of
//              |sum_n T1[n+k] T2[n]| over the flattened templates (np.correlate,
//              mode "full", then its centre slice; consolidate.py:27-41), the sums
//              in FP64 (float products are exact there)
//   P1, P2     T1 and T2 aligned per channel by the shift, zero padded
//              (consolidate.py:43-91): sample i of a channel is kept where
//              max(shift, 0) <= i < W + min(shift, 0), P1 = T1[i], P2 = T2[i - shift]
//   var_diff   sum_c (P1 - P2)_c Cov_c (P1 - P2)_c^T     (FP64)
//   SS12       P1 . P2
//   E_diff     0.5 SS[n1] - (SS12 - 0.5 SS[n2])
//   pair       var_diff > 0 ? P(N(E_diff, sqrt(var_diff)) < 0) : 0
// The reference keeps its types: with shift 0 it works on the templates
// themselves (their own type: the difference, the dot product and E_diff are
// float32 for float32 templates), otherwise on float64 zero-padded copies.
// Float32 dot products here are the FP64 sum rounded once (the reference's
// BLAS order is not specified); FP64 sums agree to rounding.
constexpr int kPairThreads = 256;

__device__ __forceinline__ double ndtr_upper(double x)   // P(Z > x) = 0.5 erfc(x / sqrt 2)
{
    return 0.5 * erfc(x * 0.70710678118654752440);
}

template <class F>
__global__ void __launch_bounds__(kPairThreads) pair_separability_kernel(
    const F* __restrict__ T, const F* __restrict__ ss, const double* __restrict__ cov,
    const double* __restrict__ variance, const double* __restrict__ threshold, uint32_t M, uint32_t C, uint32_t W,
    int max_shift, double* pair, double* noise_contamination, double* noise_misses, int32_t* shift_out)
{
    typedef cub::BlockReduce<double, kPairThreads> RD;
    __shared__ typename RD::TempStorage rd;
    __shared__ int s_shift;
    extern __shared__ __align__(16) unsigned char sraw[];
    const uint32_t n1 = blockIdx.y, n2 = blockIdx.x;
    const uint32_t L = C * W, nlag = 2u * (uint32_t)max_shift + 1u;
    F* t1 = reinterpret_cast<F*>(sraw);
    F* t2 = t1 + L;
    double* cc = reinterpret_cast<double*>(sraw + (((size_t)2 * L * sizeof(F) + 15) & ~(size_t)15));   // [nlag]
    for (uint32_t e = threadIdx.x; e < L; e += blockDim.x) {
        t1[e] = T[(uint64_t)n1 * L + e];
        t2[e] = T[(uint64_t)n2 * L + e];
    }
    __syncthreads();
    // |cross-correlation| at each lag of the centre slice, one warp per lag
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t li = warp; li < nlag; li += nwarps) {
        const int k = (int)li - max_shift;
        const uint32_t lo = k < 0 ? (uint32_t)(-k) : 0u, hi = k > 0 ? L - (uint32_t)k : L;
        double acc = 0.0;
        for (uint32_t n = lo + lane; n < hi; n += 32) acc = fma((double)t1[n + k], (double)t2[n], acc);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) cc[li] = fabs(acc);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t best = 0;
        for (uint32_t li = 1; li < nlag; ++li)
            if (cc[li] > cc[best]) best = li;   // first maximum
        s_shift = (int)best - max_shift;
    }
    __syncthreads();
    const int sh = s_shift;
    const bool same_type = sh == 0;   // the reference works on the templates themselves
    const int ilo = sh > 0 ? sh : 0, ihi = (int)W + (sh < 0 ? sh : 0);
    // aligned difference of channel c at sample i, in the type the reference forms it in
    auto diff = [&](uint32_t c, int i) -> double {
        if (i < ilo || i >= ihi) return 0.0;
        const F a = t1[c * W + i], b = t2[(int)(c * W) + i - sh];
        return same_type ? (double)(F)(a - b) : (double)a - (double)b;
    };
    double qpart = 0.0, dpart = 0.0;
    for (uint32_t e = threadIdx.x; e < L; e += blockDim.x) {
        const uint32_t c = e / W;
        const int i = (int)(e - c * W);
        const double di = diff(c, i);
        if (i >= ilo && i < ihi) dpart = fma((double)t1[e], (double)t2[(int)e - sh], dpart);
        if (di == 0.0) continue;
        const double* row = cov + ((uint64_t)c * W + (uint32_t)i) * W;
        double r = 0.0;
        for (int j = ilo; j < ihi; ++j) r = fma(row[j], diff(c, j), r);
        qpart = fma(di, r, qpart);
    }
    const double var_diff = RD(rd).Sum(qpart);
    __syncthreads();
    const double ss12 = RD(rd).Sum(dpart);
    if (threadIdx.x == 0) {
        const F e1 = (F)0.5 * ss[n1];   // expected n1 likelihood given an n1 spike
        double e_diff;
        if (same_type) {
            const F e2 = (F)ss12 - (F)0.5 * ss[n2];
            e_diff = (double)(F)(e1 - e2);
        } else {
            const double e2 = ss12 - (double)((F)0.5 * ss[n2]);
            e_diff = (double)e1 - e2;
        }
        // norm.cdf(0, E_diff, sd) = P(Z > E_diff / sd)
        pair[(uint64_t)n1 * M + n2] = var_diff > 0.0 ? ndtr_upper(e_diff / sqrt(var_diff)) : 0.0;
        if (shift_out) shift_out[(uint64_t)n1 * M + n2] = sh;
        if (n2 == 0) {
            const double sd = sqrt(variance[n1]), thr = threshold[n1], e = (double)e1;
            const double nan = __longlong_as_double(0x7ff8000000000000ll);
            // norm.cdf(thr, E, sd) and norm.sf(thr, -E, sd); scipy gives NaN for sd == 0
            noise_misses[n1] = sd > 0.0 ? ndtr_upper((e - thr) / sd) : nan;
            noise_contamination[n1] = sd > 0.0 ? ndtr_upper((thr + e) / sd) : nan;
        }
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

extern "C" int fbp_pair_separability(const void* templates, int templates_f64, const void* template_ss,
                                     const double* channel_cov, const double* variance, const double* threshold,
                                     uint32_t n_templates, uint32_t n_chans, uint32_t template_len, int32_t max_shift,
                                     double* pair_matrix, double* noise_contamination, double* noise_misses,
                                     int32_t* optimal_shift, void* stream)
{
    set_error("");
    if (n_templates == 0) return FBP_OK;
    if (n_chans == 0 || template_len == 0) return fail(FBP_E_ARG, "invalid sizes");
    if (max_shift < 0 || (uint32_t)max_shift >= template_len)
        return fail(FBP_E_ARG, "max_shift must lie in [0, template_len)");
    if (n_templates > 65535) return fail(FBP_E_ARG, "at most 65535 templates");
    if (!templates || !template_ss || !channel_cov || !variance || !threshold || !pair_matrix ||
        !noise_contamination || !noise_misses)
        return fail(FBP_E_ARG, "null pointer argument");
    const uint64_t L = (uint64_t)n_chans * template_len;
    const size_t fsz = templates_f64 ? 8 : 4;
    const size_t smem = ((2 * L * fsz + 15) & ~(size_t)15) + (size_t)(2 * max_shift + 1) * 8;
    int dev = 0, optin = 0;
    FBP_CUDA(cudaGetDevice(&dev));
    FBP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (L >= (1ull << 31) || smem + 2048 > (size_t)optin) return fail(FBP_E_ARG, "templates too long for one CTA");
    const dim3 grid(n_templates, n_templates);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (templates_f64) {
        FBP_CUDA(allow_max_dyn_smem(pair_separability_kernel<double>));
        pair_separability_kernel<double><<<grid, kPairThreads, smem, st>>>(
            static_cast<const double*>(templates), static_cast<const double*>(template_ss), channel_cov, variance,
            threshold, n_templates, n_chans, template_len, max_shift, pair_matrix, noise_contamination, noise_misses,
            optimal_shift);
    } else {
        FBP_CUDA(allow_max_dyn_smem(pair_separability_kernel<float>));
        pair_separability_kernel<float><<<grid, kPairThreads, smem, st>>>(
            static_cast<const float*>(templates), static_cast<const float*>(template_ss), channel_cov, variance,
            threshold, n_templates, n_chans, template_len, max_shift, pair_matrix, noise_contamination, noise_misses,
            optimal_shift);
    }
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}
