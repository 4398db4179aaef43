// postprocess.cu -- duplicate removal on the pursuit's device-resident output.
//
// remove_binary_pursuit_duplicates (spikesorting_fullpursuit/analyze_spike_timing.py:148-193)
// walks one unit's spikes in order: when two spikes lie within tol_inds samples
// and binary pursuit found both, the one whose clip is farther (sum of squared
// differences) from the unit's template is dropped.  Its per-unit call site
// (WorkItemSummary.remove_segment_binary_pursuit_duplicates,
// spikesorting_fullpursuit/postprocessing.py:646-675) uses the unit's mean clip
// as the template.
//
// Here:
//   * mean_clip_kernel: np.mean(clips, axis=0) in float32 -- each column summed
//     over the rows in order, then divided by n (numpy's order for an axis-0
//     reduction of a C-contiguous array).
//   * sse_kernel: np.sum((clip - template) ** 2) in float32 with numpy's
//     pairwise summation (blocks of at most 128 values summed with 8 partial
//     sums, larger ranges split in two at a multiple of 8).
//   * The walk is sequential in the reference.  At a spike j with
//     ev[j] - max(ev[0..j-1]) > tol no earlier spike is within tol of it, so
//     the walk always arrives there with curr = j: such spikes start independent
//     segments, one thread each (segment_start_kernel, walk_kernel).
#include <cub/cub.cuh>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

__global__ void mean_clip_kernel(const float* __restrict__ clips, uint32_t n, uint32_t len, float* mean)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < len; k += gridDim.x * blockDim.x) {
        float acc = clips[k];
        for (uint32_t i = 1; i < n; ++i) acc = __fadd_rn(acc, clips[(uint64_t)i * len + k]);
        mean[k] = __fdiv_rn(acc, (float)n);
    }
}

__device__ __forceinline__ float sq_diff(const float* __restrict__ a, const float* __restrict__ b, uint32_t i)
{
    const float d = __fsub_rn(a[i], b[i]);
    return __fmul_rn(d, d);
}

// numpy's pairwise sum of (a - b)^2 over [0, n)
__device__ float pairwise_sq(const float* __restrict__ a, const float* __restrict__ b, uint32_t n)
{
    if (n < 8) {
        float res = 0.f;
        for (uint32_t i = 0; i < n; ++i) res = __fadd_rn(res, sq_diff(a, b, i));
        return res;
    }
    if (n <= 128) {
        float r[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = sq_diff(a, b, j);
        uint32_t i = 8;
        for (; i < n - (n % 8); i += 8) {
#pragma unroll
            for (int j = 0; j < 8; ++j) r[j] = __fadd_rn(r[j], sq_diff(a, b, i + j));
        }
        float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                              __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
        for (; i < n; ++i) res = __fadd_rn(res, sq_diff(a, b, i));
        return res;
    }
    uint32_t n2 = n / 2;
    n2 -= n2 % 8;
    return __fadd_rn(pairwise_sq(a, b, n2), pairwise_sq(a + n2, b + n2, n - n2));
}

__global__ void sse_kernel(const float* __restrict__ clips, const float* __restrict__ tmpl, uint32_t n, uint32_t len,
                           float* sse)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        sse[i] = pairwise_sq(clips + (uint64_t)i * len, tmpl, len);
}

// start[j] = 1 where no earlier spike lies within tol of spike j (exclusive
// running maximum of the event indices, one CTA over tiles).
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) segment_start_kernel(const int64_t* __restrict__ ev, uint32_t n,
                                                                     int64_t tol, uint8_t* start)
{
    typedef cub::BlockScan<long long, kScanThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = LLONG_MIN;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += kScanThreads) {
        const uint32_t j = base + threadIdx.x;
        const long long v = j < n ? (long long)ev[j] : LLONG_MIN;
        long long excl, total;
        Scan(tmp).ExclusiveScan(v, excl, cub::Max(), total);
        const long long c = carry;
        const long long before = threadIdx.x == 0 ? c : (excl > c ? excl : c);
        if (j < n) start[j] = (j == 0 || (before != LLONG_MIN && (long long)ev[j] - before > tol)) ? 1 : 0;
        __syncthreads();
        if (threadIdx.x == 0) carry = total > c ? total : c;
        __syncthreads();
    }
}

// The reference's walk over one segment [j, next start).
__global__ void walk_kernel(const int64_t* __restrict__ ev, const uint8_t* __restrict__ bp,
                            const float* __restrict__ sse, const uint8_t* __restrict__ start, uint32_t n, int64_t tol,
                            uint8_t* keep)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (!start[j]) continue;
        uint32_t end = j + 1;
        while (end < n && !start[end]) ++end;
        for (uint32_t i = j; i < end; ++i) keep[i] = 1;
        uint32_t cur = j, nxt = j + 1;
        while (nxt < end) {
            if ((long long)ev[nxt] - (long long)ev[cur] <= tol) {
                if (bp[cur] && bp[nxt]) {
                    if (sse[cur] <= sse[nxt]) {
                        keep[nxt] = 0;
                        ++nxt;
                    } else {
                        keep[cur] = 0;
                        cur = nxt;
                        ++nxt;
                    }
                } else if (bp[cur] && !bp[nxt]) {
                    ++nxt;
                } else {
                    cur = nxt;
                    ++nxt;
                }
            } else {
                cur = nxt;
                ++nxt;
            }
        }
    }
}

size_t dup_workspace(uint32_t n)
{
    return ((size_t)n * 4 + 255) / 256 * 256 + ((size_t)n + 255) / 256 * 256;
}

}  // namespace
}  // namespace fbp

using namespace fbp;

extern "C" int fbp_mean_clip(const float* clips, uint32_t n, uint32_t clip_len, float* mean, void* stream)
{
    set_error("");
    if (n == 0 || clip_len == 0) return fail(FBP_E_ARG, "no clips");
    if (!clips || !mean) return fail(FBP_E_ARG, "null pointer argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mean_clip_kernel<<<(clip_len + 255) / 256, 256, 0, st>>>(clips, n, clip_len, mean);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

extern "C" size_t fbp_bp_duplicates_workspace(uint32_t n) { return dup_workspace(n); }

extern "C" int fbp_bp_duplicates(const int64_t* event_indices, const float* clips, const float* unit_template,
                                 const uint8_t* bp, uint32_t n, uint32_t clip_len, int64_t tol_inds,
                                 uint8_t* keep, void* workspace, size_t workspace_bytes, void* stream)
{
    set_error("");
    if (n == 0) return FBP_OK;
    if (clip_len == 0) return fail(FBP_E_ARG, "clip_len is 0");
    if (!event_indices || !clips || !unit_template || !bp || !keep || !workspace)
        return fail(FBP_E_ARG, "null pointer argument");
    if (workspace_bytes < dup_workspace(n)) return fail(FBP_E_WORKSPACE, "workspace too small");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    float* sse = reinterpret_cast<float*>(ws);
    uint8_t* start = ws + ((size_t)n * 4 + 255) / 256 * 256;
    const uint32_t g = (n + 255) / 256 < 148u * 16 ? (n + 255) / 256 : 148u * 16;
    sse_kernel<<<g, 256, 0, st>>>(clips, unit_template, n, clip_len, sse);
    segment_start_kernel<<<1, kScanThreads, 0, st>>>(event_indices, n, tol_inds, start);
    walk_kernel<<<g, 256, 0, st>>>(event_indices, bp, sse, start, n, tol_inds, keep);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}
