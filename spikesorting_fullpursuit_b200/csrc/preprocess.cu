// preprocess.cu -- the pursuit's inputs built on the device (full_binary_pursuit's pre-processing).
//
// full_binary_pursuit (spikesorting_fullpursuit/overlap/full_binary_pursuit.py:325-349)
// builds the pursuit's templates and noise model from the sorted spikes: per unit,
// its clips on all channels (get_clips, processing/clip_utils.py:501-632), a robust
// template (calculate_robust_template, clip_utils.py:202-248), and from all units'
// clip-minus-template residuals one noise covariance per channel
// (get_channel_covariance_matrix, full_binary_pursuit.py:863-923).  Here:
//   * gather_clips_kernel: clips[k][n*Wc + j] = V[chans[n]][ev[k] + w0 + j].
//   * robust_template_kernel: per clip sample (column) of n clips, in float32 as
//     numpy computes it: med = median(x); mad = median(|x - med|) / 0.6745;
//     the template is median(x[med - mad < x < med + mad]), or med if that set is
//     empty.  Medians are exact order statistics (the mean of the two middle
//     values for an even count, as np.median), found by radix selection over
//     order-preserving integer keys: 4 passes of 8 bits, each a shared-memory
//     histogram of the candidates.  A CTA handles 32 adjacent columns, lanes
//     over columns, so every pass reads rows of 128 contiguous bytes.
//   * covariance_kernel: per channel, the FP64 covariance (ddof 0) of the
//     selected residual rows' samples on that channel: column means summed over
//     the rows in order (numpy's axis-0 order), then centred products.  numpy
//     multiplies with BLAS, so covariances agree to FP64 rounding.
#include <cub/cub.cuh>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

__global__ void gather_clips_kernel(const float* __restrict__ V, uint64_t N, const uint32_t* __restrict__ chans,
                                    uint32_t nch, const int64_t* __restrict__ ev, uint32_t n, int32_t w0, uint32_t wc,
                                    float* clips)
{
    const uint64_t len = (uint64_t)nch * wc;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < (uint64_t)n * len;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = e / len, r = e - k * len;
        const uint32_t ci = (uint32_t)(r / wc), j = (uint32_t)(r - (uint64_t)ci * wc);
        const int64_t s = ev[k] + w0 + (int64_t)j;
        clips[e] = V[(uint64_t)chans[ci] * N + (uint64_t)s];
    }
}

// order-preserving key of a float (finite or infinite)
__device__ __forceinline__ uint32_t fkey(float x)
{
    const uint32_t u = __float_as_uint(x);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unkey(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

constexpr int kRtCols = 32;      // columns per CTA (one per lane)
constexpr int kRtThreads = 256;  // 8 warps over the rows

// What a selection ranks, per column: 0 = x, 1 = |x - med|, 2 = x restricted to
// (lo, hi) (strict bounds).
struct RtColumn {
    float med, lo, hi;
};

// k-th smallest key (0-based) of each lane's column among its candidates.
// All threads of the CTA call it; returns the key for the calling lane's column.
__device__ uint32_t select_kth(const float* __restrict__ clips, uint32_t n, uint32_t len, uint32_t col0, int mode,
                               const RtColumn* cols, const uint32_t* kth, uint32_t* hist, uint32_t* s_prefix,
                               uint32_t* s_k)
{
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    if (threadIdx.x < kRtCols) {
        s_prefix[threadIdx.x] = 0;
        s_k[threadIdx.x] = kth[threadIdx.x];
    }
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 24 - 8 * pass;
        for (uint32_t e = threadIdx.x; e < kRtCols * 256; e += blockDim.x) hist[e] = 0;
        __syncthreads();
        const uint32_t col = col0 + lane;
        const uint32_t prefix = s_prefix[lane];
        const uint32_t pmask = pass == 0 ? 0u : (0xFFFFFFFFu << (shift + 8));
        if (col < len) {
            const RtColumn c = cols[lane];
            for (uint32_t i = warp; i < n; i += nwarps) {
                const float x = clips[(uint64_t)i * len + col];
                float v = x;
                if (mode == 1) v = fabsf(__fsub_rn(x, c.med));
                if (mode == 2 && !(x > c.lo && x < c.hi)) continue;
                const uint32_t key = fkey(v);
                if ((key & pmask) != (prefix & pmask)) continue;
                atomicAdd(&hist[lane * 256 + ((key >> shift) & 0xFFu)], 1u);
            }
        }
        __syncthreads();
        if (threadIdx.x < kRtCols) {
            const uint32_t* h = hist + threadIdx.x * 256;
            uint32_t k = s_k[threadIdx.x], b = 0;
            for (; b < 255; ++b) {
                if (k < h[b]) break;
                k -= h[b];
            }
            s_k[threadIdx.x] = k;
            s_prefix[threadIdx.x] |= b << shift;
        }
        __syncthreads();
    }
    return s_prefix[lane];
}

// median of a column's candidates: the middle key, or the float32 mean of the two
// middle values (np.median -> np.mean of two float32 values)
__device__ float column_median(const float* __restrict__ clips, uint32_t n, uint32_t len, uint32_t col0, int mode,
                               RtColumn* cols, uint32_t* cnt, uint32_t* kth, uint32_t* hist, uint32_t* s_prefix,
                               uint32_t* s_k)
{
    const uint32_t lane = threadIdx.x & 31;
    if (threadIdx.x < kRtCols) kth[threadIdx.x] = cnt[threadIdx.x] > 0 ? (cnt[threadIdx.x] - 1) / 2 : 0;
    __syncthreads();
    const float a = unkey(select_kth(clips, n, len, col0, mode, cols, kth, hist, s_prefix, s_k));
    __syncthreads();
    if (threadIdx.x < kRtCols) kth[threadIdx.x] = cnt[threadIdx.x] / 2;
    __syncthreads();
    const float b = unkey(select_kth(clips, n, len, col0, mode, cols, kth, hist, s_prefix, s_k));
    __syncthreads();
    const uint32_t c = cnt[lane];
    return (c & 1u) ? a : __fdiv_rn(__fadd_rn(a, b), 2.0f);
}

__global__ void __launch_bounds__(kRtThreads) robust_template_kernel(const float* __restrict__ clips, uint32_t n,
                                                                     uint32_t len, float* tmpl)
{
    __shared__ uint32_t hist[kRtCols * 256];
    __shared__ uint32_t s_prefix[kRtCols], s_k[kRtCols], kth[kRtCols], cnt[kRtCols];
    __shared__ RtColumn cols[kRtCols];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t col0 = blockIdx.x * kRtCols, col = col0 + lane;
    if (threadIdx.x < kRtCols) {
        cnt[threadIdx.x] = n;
        cols[threadIdx.x] = RtColumn{0.f, 0.f, 0.f};
    }
    __syncthreads();
    const float med = column_median(clips, n, len, col0, 0, cols, cnt, kth, hist, s_prefix, s_k);
    if (threadIdx.x < kRtCols) cols[threadIdx.x].med = med;
    __syncthreads();
    const float mad = __fdiv_rn(column_median(clips, n, len, col0, 1, cols, cnt, kth, hist, s_prefix, s_k), 0.6745f);
    if (threadIdx.x < kRtCols) {
        cols[threadIdx.x].lo = __fsub_rn(med, mad);
        cols[threadIdx.x].hi = __fadd_rn(med, mad);
        cnt[threadIdx.x] = 0;
    }
    __syncthreads();
    // size of the within-1-MAD set per column
    if (col < len) {
        const RtColumn c = cols[lane];
        uint32_t m = 0;
        for (uint32_t i = warp; i < n; i += blockDim.x >> 5) {
            const float x = clips[(uint64_t)i * len + col];
            m += (x > c.lo && x < c.hi) ? 1u : 0u;
        }
        atomicAdd(&cnt[lane], m);
    }
    __syncthreads();
    const float sel = column_median(clips, n, len, col0, 2, cols, cnt, kth, hist, s_prefix, s_k);
    if (threadIdx.x < kRtCols && col < len) tmpl[col] = cnt[threadIdx.x] > 0 ? sel : med;
}

// Per channel c (blockIdx.y) and output row i (blockIdx.x): means of the
// channel's selected residual rows (rows[c][0..n_rows)) over its samples
// [c*Wc, (c+1)*Wc), and row i of its covariance.
// Residual row r = clips[rows[r]] - template[unit[rows[r]]] in float32, then FP64.
__global__ void covariance_kernel(const float* __restrict__ clips, const float* __restrict__ tmpls,
                                  const uint32_t* __restrict__ unit_of, const int64_t* __restrict__ rows,
                                  uint32_t n_rows, uint32_t len, uint32_t wc, double* cov)
{
    extern __shared__ double mean[];   // [wc]
    const uint32_t c = blockIdx.y, i = blockIdx.x;
    const uint32_t base = c * wc;
    for (uint32_t j = threadIdx.x; j < wc; j += blockDim.x) {
        double acc = 0.0;
        bool first = true;
        for (uint32_t r = 0; r < n_rows; ++r) {
            const uint64_t row = (uint64_t)rows[(uint64_t)c * n_rows + r];
            const double x = (double)__fsub_rn(clips[row * len + base + j], tmpls[(uint64_t)unit_of[row] * len + base + j]);
            acc = first ? x : __dadd_rn(acc, x);
            first = false;
        }
        mean[j] = acc / (double)n_rows;
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < wc; j += blockDim.x) {
        double acc = 0.0;
        for (uint32_t r = 0; r < n_rows; ++r) {
            const uint64_t row = (uint64_t)rows[(uint64_t)c * n_rows + r];
            const uint64_t u = (uint64_t)unit_of[row] * len + base;
            const double xi = (double)__fsub_rn(clips[row * len + base + i], tmpls[u + i]) - mean[i];
            const double xj = (double)__fsub_rn(clips[row * len + base + j], tmpls[u + j]) - mean[j];
            acc = fma(xi, xj, acc);
        }
        cov[((uint64_t)c * wc + i) * wc + j] = acc * (1.0 / (double)n_rows);   // np.cov scales by 1 / fact
    }
}

}  // namespace
}  // namespace fbp

using namespace fbp;

extern "C" int fbp_gather_clips(const float* voltage, uint32_t n_chans, uint64_t n_samples, const uint32_t* chans,
                                uint32_t n_nbr, const int64_t* event_indices, uint32_t n, int32_t win0,
                                uint32_t win_len, float* clips, void* stream)
{
    set_error("");
    if (n == 0) return FBP_OK;
    if (!voltage || !chans || !event_indices || !clips || n_nbr == 0 || win_len == 0 || n_chans == 0)
        return fail(FBP_E_ARG, "invalid arguments");
    const uint64_t total = (uint64_t)n * n_nbr * win_len;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
    gather_clips_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(voltage, n_samples, chans, n_nbr,
                                                                              event_indices, n, win0, win_len, clips);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

extern "C" int fbp_robust_template(const float* clips, uint32_t n, uint32_t clip_len, float* tmpl, void* stream)
{
    set_error("");
    if (n == 0 || clip_len == 0) return fail(FBP_E_ARG, "no clips");
    if (!clips || !tmpl) return fail(FBP_E_ARG, "null pointer argument");
    robust_template_kernel<<<(clip_len + kRtCols - 1) / kRtCols, kRtThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        clips, n, clip_len, tmpl);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

extern "C" int fbp_residual_covariance(const float* clips, const float* templates, const uint32_t* unit_of,
                                       const int64_t* rows, uint32_t n_rows, uint32_t clip_len, uint32_t n_chans,
                                       uint32_t n_samples_per_chan, double* cov, void* stream)
{
    set_error("");
    if (n_rows == 0 || n_chans == 0 || n_samples_per_chan == 0) return fail(FBP_E_ARG, "invalid sizes");
    if ((uint64_t)n_chans * n_samples_per_chan > clip_len) return fail(FBP_E_ARG, "clip shorter than channels x samples");
    if (!clips || !templates || !unit_of || !rows || !cov) return fail(FBP_E_ARG, "null pointer argument");
    const size_t smem = (size_t)n_samples_per_chan * 8;
    if (smem > 48 * 1024) return fail(FBP_E_ARG, "samples per channel too large");
    covariance_kernel<<<dim3(n_samples_per_chan, n_chans), 128, smem, static_cast<cudaStream_t>(stream)>>>(
        clips, templates, unit_of, rows, n_rows, clip_len, n_samples_per_chan, cov);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}
