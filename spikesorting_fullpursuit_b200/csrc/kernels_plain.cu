// kernels_plain.cu -- exact FP32 kernels of the binary-pursuit pass.
//
// Every float operation of the reference kernels
// (spikesorting_fullpursuit/kernels/binary_pursuit.cl) is reproduced in its
// order with round-to-nearest intrinsics (__fadd_rn/__fmul_rn/__fsub_rn are
// never contracted into FMAs), so results are bit-identical to the reference
// run with its work-groups in order.  Steps whose reference outcome depends on
// execution order are computed in that canonical order by construction:
//   * per-window argmax: lexicographic first (t, s) among the maxima;
//   * overlap recheck winner: max value, then lowest work-group, then the
//     tree-reduction slot order inside the group (bit-reversed local id);
//   * reassignment and pruning chains: resolved by walking the chain back;
//   * spike output: window-list order; residual: list order for overlaps.
#include <cub/cub.cuh>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

constexpr int kChainCap = 4096;

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }

__global__ void iota_kernel(uint32_t* out, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = i;
}

// ---------------------------------------------------------------------------
// Likelihood (compute_full_likelihood + compute_maximum_likelihood,
// binary_pursuit.cl:216-300).  One CTA per listed window, one thread per
// sample, Q templates per smem stage: thread x computes L[t][id*W+x] for the Q
// templates with Q independent accumulators, each summed from bias[t] over
// channels then taps in the reference order.
// ---------------------------------------------------------------------------
template <int Q>
__global__ void __launch_bounds__(1024) lik_exact_kernel(Dims d, const float* __restrict__ V,
                                                         const float* __restrict__ T,
                                                         const float* __restrict__ bias,
                                                         const uint32_t* __restrict__ list,
                                                         uint32_t nlist, float* __restrict__ L)
{
    extern __shared__ __align__(16) float sm[];
    const uint32_t SW = (2 * d.W + 3) & ~3u;   // strip length, 2W-1 used
    const uint32_t Wp = (d.W + 3) & ~3u;       // template row pitch
    float* Vs = sm;                             // [C][SW]
    float* Ts = sm + d.C * SW;                  // [Q][C][Wp]
    const uint32_t tq_stride = d.C * Wp;
    for (uint32_t wi = blockIdx.x; wi < nlist; wi += gridDim.x) {
        const uint32_t id = list ? list[wi] : wi;
        const uint64_t s0 = (uint64_t)id * d.W;
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < d.C * SW; e += blockDim.x) {
            const uint32_t c = e / SW, x = e - c * SW;
            const uint64_t g = s0 + x;
            Vs[e] = (x < 2 * d.W - 1 && g < d.N) ? V[(uint64_t)c * d.N + g] : 0.f;
        }
        const uint32_t x = threadIdx.x;
        const uint64_t s = s0 + x;
        const bool active = x < d.W && s < d.N;
        const bool valid = active && s + d.W < d.N;
        for (uint32_t t0 = 0; t0 < d.M; t0 += Q) {
            __syncthreads();
            for (uint32_t e = threadIdx.x; e < Q * tq_stride; e += blockDim.x) {
                const uint32_t q = e / tq_stride, r = e - q * tq_stride;
                const uint32_t c = r / Wp, j = r - c * Wp;
                Ts[e] = (t0 + q < d.M && j < d.W) ? T[((uint64_t)(t0 + q) * d.C + c) * d.W + j] : 0.f;
            }
            __syncthreads();
            if (!active) continue;
            float acc[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) acc[q] = (t0 + q < d.M) ? bias[t0 + q] : 0.f;
            if (valid) {
                for (uint32_t c = 0; c < d.C; ++c) {
                    const float* vr = Vs + c * SW + x;
                    const float* tr = Ts + c * Wp;
                    uint32_t j = 0;
                    for (; j + 4 <= d.W; j += 4) {
                        const float v0 = vr[j], v1 = vr[j + 1], v2 = vr[j + 2], v3 = vr[j + 3];
#pragma unroll
                        for (int q = 0; q < Q; ++q) {
                            const float4 t4 = *reinterpret_cast<const float4*>(tr + q * tq_stride + j);
                            acc[q] = fadd(acc[q], fmul(t4.x, v0));
                            acc[q] = fadd(acc[q], fmul(t4.y, v1));
                            acc[q] = fadd(acc[q], fmul(t4.z, v2));
                            acc[q] = fadd(acc[q], fmul(t4.w, v3));
                        }
                    }
                    for (; j < d.W; ++j) {
                        const float v = vr[j];
#pragma unroll
                        for (int q = 0; q < Q; ++q) acc[q] = fadd(acc[q], fmul(tr[q * tq_stride + j], v));
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (t0 + q < d.M) L[(uint64_t)(t0 + q) * d.N + s] = valid ? acc[q] : 0.f;
        }
    }
}

// ---------------------------------------------------------------------------
// Per-window argmax (compute_template_maximum_likelihood, binary_pursuit.cl:350-441,
// the M sequential host launches folded into one).  One warp per listed window.
// ---------------------------------------------------------------------------
struct Best {
    float v;
    uint32_t t, s;
    bool have;
};

__device__ __forceinline__ bool better(const Best& a, const Best& b)
{
    if (!a.have) return false;
    if (!b.have) return true;
    if (a.v != b.v) return a.v > b.v;
    if (a.t != b.t) return a.t < b.t;
    return a.s < b.s;
}

__global__ void argmax_kernel(Dims d, const float* __restrict__ L, const uint32_t* __restrict__ list,
                              uint32_t nlist, float* best_lik, uint32_t* best_lab, uint32_t* best_idx,
                              uint8_t* check, uint8_t* orech, uint32_t* ov_idx, uint32_t* ov_lab)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k = warp; k < nlist; k += nwarps) {
        const uint32_t id = list[k];
        const uint64_t start = (uint64_t)id * d.W, end = start + d.W;
        if (end >= (uint64_t)d.N - d.W) continue;
        const uint64_t lo = (d.W > start) ? 0 : start - d.W;
        const uint64_t hi = (end + d.W > d.N) ? d.N : end + d.W;
        Best b{0.f, 0u, 0u, false};
        bool flag = false;
        for (uint32_t t = 0; t < d.M; ++t) {
            const float* Lt = L + (uint64_t)t * d.N;
            for (uint64_t s = lo + lane; s < hi; s += 32) {
                const float v = Lt[s];
                if (v > b.v) { b.v = v; b.t = t; b.s = (uint32_t)s; b.have = true; }
                if (v > 0.f && s >= start && s < end) flag = true;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            Best o;
            o.v = __shfl_down_sync(0xffffffffu, b.v, off);
            o.t = __shfl_down_sync(0xffffffffu, b.t, off);
            o.s = __shfl_down_sync(0xffffffffu, b.s, off);
            o.have = __shfl_down_sync(0xffffffffu, (int)b.have, off) != 0;
            if (better(o, b)) b = o;
        }
        const bool any_flag = __any_sync(0xffffffffu, flag);
        if (lane == 0) {
            if (any_flag) check[id] = 1;
            uint32_t lab = best_lab[id], idx = best_idx[id];
            float bl = 0.f;
            if (b.have) { bl = b.v; lab = b.t; idx = b.s; }
            orech[id] = (bl > 0.f && idx >= start && idx < end) ? 1 : 0;
            best_lik[id] = bl;
            best_lab[id] = lab;
            best_idx[id] = idx;
            ov_idx[id] = idx;
            ov_lab[id] = lab;
        }
    }
}

// ---------------------------------------------------------------------------
// Ordered stream compaction: count per block, scan of block counts, scatter.
// A functor supplies pred(i), emit(i, pos) and after(i) (run in the scatter).
// ---------------------------------------------------------------------------
constexpr int kCompactThreads = 256;
constexpr int kCompactItems = 4;
constexpr int kCompactTile = kCompactThreads * kCompactItems;

template <class F>
__global__ void __launch_bounds__(kCompactThreads) compact_count(F f, const uint32_t* n_dev, uint32_t n_host,
                                                                  uint32_t* blk)
{
    typedef cub::BlockReduce<uint32_t, kCompactThreads> R;
    __shared__ typename R::TempStorage tmp;
    const uint32_t n = n_dev ? *n_dev : n_host;
    const uint64_t base = (uint64_t)blockIdx.x * kCompactTile + threadIdx.x * kCompactItems;
    uint32_t cnt = 0;
#pragma unroll
    for (int r = 0; r < kCompactItems; ++r) {
        const uint64_t i = base + r;
        if (i < n && f.pred((uint32_t)i)) ++cnt;
    }
    const uint32_t tot = R(tmp).Sum(cnt);
    if (threadIdx.x == 0) blk[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) compact_scan(uint32_t* blk, uint32_t nblk, uint32_t* total)
{
    typedef cub::BlockScan<uint32_t, 1024> S;
    __shared__ typename S::TempStorage tmp;
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < nblk; b0 += 1024) {
        const uint32_t i = b0 + threadIdx.x;
        const uint32_t v = i < nblk ? blk[i] : 0u;
        uint32_t ex, agg;
        S(tmp).ExclusiveSum(v, ex, agg);
        if (i < nblk) blk[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class F>
__global__ void __launch_bounds__(kCompactThreads) compact_scatter(F f, const uint32_t* n_dev, uint32_t n_host,
                                                                    const uint32_t* blk)
{
    typedef cub::BlockScan<uint32_t, kCompactThreads> S;
    __shared__ typename S::TempStorage tmp;
    const uint32_t n = n_dev ? *n_dev : n_host;
    const uint64_t base = (uint64_t)blockIdx.x * kCompactTile + threadIdx.x * kCompactItems;
    bool p[kCompactItems];
    uint32_t cnt = 0;
#pragma unroll
    for (int r = 0; r < kCompactItems; ++r) {
        const uint64_t i = base + r;
        p[r] = i < n && f.pred((uint32_t)i);
        cnt += p[r];
    }
    uint32_t ex;
    S(tmp).ExclusiveSum(cnt, ex);
    uint32_t pos = blk[blockIdx.x] + ex;
#pragma unroll
    for (int r = 0; r < kCompactItems; ++r) {
        const uint64_t i = base + r;
        if (p[r]) f.emit((uint32_t)i, pos++);
        if (i < n) f.after((uint32_t)i);
    }
}

template <class F>
int compact(F f, const uint32_t* n_dev, uint32_t n_upper, uint32_t* blk, uint32_t* total,
            cudaStream_t st)
{
    const uint32_t nb = (n_upper + kCompactTile - 1) / kCompactTile;
    if (nb == 0) {
        FBP_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), st));
        return FBP_OK;
    }
    count_launch(3);
    compact_count<F><<<nb, kCompactThreads, 0, st>>>(f, n_dev, n_upper, blk);
    compact_scan<<<1, 1024, 0, st>>>(blk, nb, total);
    compact_scatter<F><<<nb, kCompactThreads, 0, st>>>(f, n_dev, n_upper, blk);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

struct FlagF {
    const uint32_t* list;
    const uint8_t* orech;
    uint32_t* out;
    __device__ bool pred(uint32_t k) const { return orech[list[k]] == 1; }
    __device__ void emit(uint32_t k, uint32_t pos) const { out[pos] = list[k]; }
    __device__ void after(uint32_t) const {}
};

struct SpikeF {
    const uint32_t* list;
    const uint8_t* has;
    const uint32_t* best_idx;
    const uint32_t* best_lab;
    uint32_t *pidx, *plab, *pwin;
    __device__ bool pred(uint32_t k) const { return has[k] != 0; }
    __device__ void emit(uint32_t k, uint32_t pos) const
    {
        const uint32_t id = list[k];
        pidx[pos] = best_idx[id];
        plab[pos] = best_lab[id];
        pwin[pos] = id;
    }
    __device__ void after(uint32_t) const {}
};

struct NextF {
    uint8_t* check;
    uint32_t* out;
    __device__ bool pred(uint32_t x) const { return check[x] != 0; }
    __device__ void emit(uint32_t x, uint32_t pos) const { out[pos] = x; }
    __device__ void after(uint32_t x) const { check[x] = 0; }
};

// ---------------------------------------------------------------------------
// Overlap recheck, brute force (overlap_recheck_indices + max_local_reduction +
// the group scan of parse_overlap_recheck_indices, binary_pursuit.cl:167-186,
// 444-654, 690-706).  One CTA per (flagged window, template t).  A thread
// evaluates four consecutive template shifts b for one fixed shift a, sliding
// the shifted template t through registers.  Each item's value is summed in
// the reference order.  Winners are folded into one 64-bit key per window:
// (value bits << 32) | ~priority, priority = group * WG + bitrev(local id).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t item_priority(uint64_t r, uint32_t WG, uint32_t lbits)
{
    const uint32_t g = (uint32_t)(r / WG), l = (uint32_t)(r % WG);
    const uint32_t br = lbits ? (__brev(l) >> (32 - lbits)) : 0u;
    return g * WG + br;
}

// Best (lowest) priority among the work-item slots that hold item r.
__device__ __forceinline__ uint32_t best_copy_priority(uint64_t r, uint64_t items, uint64_t slots,
                                                       uint32_t WG, uint32_t lbits)
{
    uint32_t best = item_priority(r, WG, lbits);
    for (uint64_t rr = r + items; rr < slots; rr += items) {
        const uint32_t p = item_priority(rr, WG, lbits);
        best = p < best ? p : best;
    }
    return best;
}

__device__ __forceinline__ unsigned long long make_key(float v, uint32_t prio)
{
    return ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xFFFFFFFFu - prio);
}

constexpr int kOvThreads = 256;
constexpr int kOvPerThread = 8;
constexpr int kOvRound = kOvThreads * kOvPerThread;

__global__ void __launch_bounds__(kOvThreads) overlap_plain_kernel(
    Dims d, const float* __restrict__ V, const float* __restrict__ T, const float* __restrict__ L,
    const float* __restrict__ theta, const uint32_t* __restrict__ flag, const DevStatus* status,
    const uint32_t* __restrict__ best_lab, const uint32_t* __restrict__ best_idx,
    unsigned long long* keys, unsigned long long* item_counter)
{
    typedef cub::BlockScan<uint32_t, kOvThreads> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ unsigned long long s_best;
    extern __shared__ __align__(16) float sm[];
    const uint32_t S = d.S, W = d.W, C = d.C;
    const uint32_t S2 = 2 * S + 1;
    const uint32_t RW = W + 2 * S + 4;          // padded template row
    const uint32_t OFF = S + 4;                 // padded index of template sample 0
    float* Fp = sm;                             // [C][RW] best template f
    float* Tp = Fp + C * RW;                    // [C][RW] template t
    float* Vw = Tp + C * RW;                    // [C][W] residual window
    uint8_t* fa = reinterpret_cast<uint8_t*>(Vw + C * W);  // per shift: bit0 in bounds, bit1 L_f > 0
    uint8_t* ft = fa + S2;                                  // per shift: bit1 L_t > 0
    const size_t cand_off = ((size_t)(ft + S2 - reinterpret_cast<uint8_t*>(sm)) + 15) & ~(size_t)15;
    uint32_t* cand = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(sm) + cand_off);
    const uint32_t nblk4 = (S2 + 3) / 4;
    const uint64_t items = (uint64_t)S2 * S2 * d.M;
    const uint64_t nloc = (items - 1) / d.WG + 1;
    const uint64_t slots = nloc * d.WG;
    uint32_t lbits = 0;
    while ((1u << lbits) < d.WG) ++lbits;
    const uint32_t nflag = status->n_flag;
    const uint64_t ntask = (uint64_t)nflag * d.M;
    unsigned long long my_items = 0;
    for (uint64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
        const uint32_t k = (uint32_t)(task / d.M), t = (uint32_t)(task % d.M);
        const uint32_t id = flag[k];
        const uint32_t f = best_lab[id], p = best_idx[id];
        if (L[(uint64_t)f * d.N + p] < theta[f]) continue;
        if ((uint64_t)p >= (uint64_t)d.N - W) continue;
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < C * RW; e += blockDim.x) {
            const uint32_t c = e / RW, x = e - c * RW;
            const int64_t j = (int64_t)x - OFF;
            const bool in = j >= 0 && j < (int64_t)W;
            Fp[e] = in ? T[((uint64_t)f * C + c) * W + j] : 0.f;
            Tp[e] = in ? T[((uint64_t)t * C + c) * W + j] : 0.f;
        }
        for (uint32_t e = threadIdx.x; e < C * W; e += blockDim.x) {
            const uint32_t c = e / W, j = e - c * W;
            Vw[e] = V[(uint64_t)c * d.N + p + j];
        }
        for (uint32_t a = threadIdx.x; a < S2; a += blockDim.x) {
            const uint64_t ap = (uint64_t)a + p;
            const bool inb = ap >= S && ap < (uint64_t)d.N - W + S;
            uint8_t fl = inb ? 1 : 0, tl = 0;
            if (inb) {
                if (L[(uint64_t)f * d.N + ap - S] > 0.f) fl |= 2;
                if (L[(uint64_t)t * d.N + ap - S] > 0.f) tl = 2;
            }
            fa[a] = fl;
            ft[a] = tl;
        }
        if (threadIdx.x == 0) s_best = 0ull;
        __syncthreads();
        unsigned long long kbest = 0ull;
        const uint32_t ncand_total = S2 * nblk4;
        for (uint32_t base = 0; base < ncand_total; base += kOvRound) {
            uint32_t mine[kOvPerThread];
            uint32_t cnt = 0;
#pragma unroll
            for (int r = 0; r < kOvPerThread; ++r) {
                const uint32_t ci = base + threadIdx.x * kOvPerThread + r;
                bool ok = false;
                if (ci < ncand_total) {
                    const uint32_t a = ci / nblk4, b0 = (ci - a * nblk4) * 4;
                    const uint8_t fla = fa[a];
                    if (fla & 1) {
                        for (uint32_t q = 0; q < 4; ++q) {
                            const uint32_t b = b0 + q;
                            if (b >= S2) break;
                            const uint32_t dab = a > b ? a - b : b - a;
                            if ((fa[b] & 1) && dab <= W && ((fla & 2) || (ft[b] & 2))) { ok = true; break; }
                        }
                    }
                }
                if (ok) mine[cnt++] = ci;
            }
            uint32_t off, tot;
            Scan(scan_tmp).ExclusiveSum(cnt, off, tot);
            for (uint32_t r = 0; r < cnt; ++r) cand[off + r] = mine[r];
            __syncthreads();
            for (uint32_t e = threadIdx.x; e < tot; e += blockDim.x) {
                const uint32_t ci = cand[e];
                const uint32_t a = ci / nblk4, b0 = (ci - a * nblk4) * 4;
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                const uint32_t fbase = 2 * S + 4 - a;   // padded index of F at j = 0
                const uint32_t tbase = 2 * S + 4 - b0;  // padded index of T(b0) at j = 0
                for (uint32_t c = 0; c < C; ++c) {
                    const float* fr = Fp + c * RW + fbase;
                    const float* tr = Tp + c * RW + tbase;
                    const float* vr = Vw + c * W;
                    float t0 = tr[0], t1 = tr[-1], t2 = tr[-2], t3 = tr[-3];
                    float ss[4] = {0.f, 0.f, 0.f, 0.f};
                    for (uint32_t j = 0; j < W; ++j) {
                        const float fv = fr[j], v = vr[j];
                        const float s0 = fadd(fv, t0), s1 = fadd(fv, t1), s2 = fadd(fv, t2), s3 = fadd(fv, t3);
                        ss[0] = fadd(ss[0], fmul(s0, s0)); acc[0] = fadd(acc[0], fmul(s0, v));
                        ss[1] = fadd(ss[1], fmul(s1, s1)); acc[1] = fadd(acc[1], fmul(s1, v));
                        ss[2] = fadd(ss[2], fmul(s2, s2)); acc[2] = fadd(acc[2], fmul(s2, v));
                        ss[3] = fadd(ss[3], fmul(s3, s3)); acc[3] = fadd(acc[3], fmul(s3, v));
                        t3 = t2; t2 = t1; t1 = t0; t0 = tr[j + 1];
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (ss[q] > 0.f) acc[q] = fsub(acc[q], fmul(0.5f, ss[q]));
                }
                const uint8_t fla = fa[a];
#pragma unroll
                for (uint32_t q = 0; q < 4; ++q) {
                    const uint32_t b = b0 + q;
                    if (b >= S2) break;
                    const uint32_t dab = a > b ? a - b : b - a;
                    if (!((fa[b] & 1) && dab <= W && ((fla & 2) || (ft[b] & 2)))) continue;
                    ++my_items;
                    if (acc[q] > 0.f) {
                        const uint64_t r = (uint64_t)t + (uint64_t)d.M * a + (uint64_t)d.M * S2 * b;
                        const uint32_t pr = best_copy_priority(r, items, slots, d.WG, lbits);
                        const unsigned long long key = make_key(acc[q], pr);
                        kbest = key > kbest ? key : kbest;
                    }
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int off2 = 16; off2 > 0; off2 >>= 1) {
            const unsigned long long o = __shfl_down_sync(0xffffffffu, kbest, off2);
            kbest = o > kbest ? o : kbest;
        }
        if ((threadIdx.x & 31) == 0 && kbest) atomicMax(&s_best, kbest);
        __syncthreads();
        if (threadIdx.x == 0 && s_best) atomicMax(&keys[k], s_best);
    }
    if (my_items) atomicAdd(item_counter, my_items);
}

// ---------------------------------------------------------------------------
// parse_overlap_recheck_indices (binary_pursuit.cl:657-815), one thread per
// flagged window, from the winner key.
// ---------------------------------------------------------------------------
// Exact likelihood of (t, s) in the reference order (compute_maximum_likelihood,
// binary_pursuit.cl:216-252) from the current voltage, by a whole warp: each
// lane forms the products of 32 taps at a time (each product rounds the same
// wherever it is formed), and every lane adds them in tap order, so all lanes
// end with the reference's sum.  Channels where the template is entirely zero
// add 0 * v terms in the reference, which leave a nonzero sum unchanged.
__device__ float warp_exact_lik(const Dims& d, const float* __restrict__ V, const float* __restrict__ T, float b,
                                uint32_t t, uint32_t s, const float* __restrict__ tnorm)
{
    const uint32_t lane = threadIdx.x & 31;
    float acc = b;
    for (uint32_t c = 0; c < d.C; ++c) {
        if (tnorm[(uint64_t)t * d.C + c] == 0.f) continue;
        const float* tr = T + ((uint64_t)t * d.C + c) * d.W;
        const float* vr = V + (uint64_t)c * d.N + s;
        for (uint32_t j0 = 0; j0 < d.W; j0 += 32) {
            const uint32_t j = j0 + lane;
            const float p = j < d.W ? fmul(__ldg(tr + j), vr[j]) : 0.f;
            const uint32_t n = d.W - j0 < 32u ? d.W - j0 : 32u;
#pragma unroll 8
            for (uint32_t k = 0; k < n; ++k) acc = fadd(acc, __shfl_sync(0xffffffffu, p, k));
        }
    }
    return acc;
}

// L[t][s], made exact where the tensor-core likelihood may have left an estimate
// (a positive value in a flagged window row; the window's voltage is unchanged
// since it was computed, so the current voltage gives the exact value).  Called
// by a whole warp with the same (t, s) on every lane.
__device__ __forceinline__ float warp_lik_value(const Dims& d, const float* __restrict__ L, const LazyRef& z,
                                                uint32_t t, uint32_t s)
{
    const float v = L[(uint64_t)t * d.N + s];
    if (z.wflag != nullptr && v > 0.f && z.wflag[(uint64_t)(s / d.W) * d.M + t])
        return warp_exact_lik(d, z.V, z.T, z.bias[t], t, s, z.tnorm);
    return v;
}

// One warp per flagged window (every lane evaluates the same decisions; lane 0
// writes them).
__global__ void parse_kernel(Dims d, const float* __restrict__ L, const float* __restrict__ theta,
                             const uint32_t* __restrict__ flag, const DevStatus* status,
                             const unsigned long long* __restrict__ keys, float* best_lik,
                             const uint32_t* __restrict__ best_lab, const uint32_t* __restrict__ best_idx,
                             uint8_t* orech, uint32_t* ov_idx, uint32_t* ov_lab, LazyRef z)
{
    const uint32_t nflag = status->n_flag;
    const uint64_t S2 = 2ull * d.S + 1;
    const uint64_t items = S2 * S2 * d.M;
    const bool lead = (threadIdx.x & 31) == 0;
    uint32_t lbits = 0;
    while ((1u << lbits) < d.WG) ++lbits;
    const uint32_t wpb = blockDim.x >> 5;
    for (uint32_t k = blockIdx.x * wpb + (threadIdx.x >> 5); k < nflag; k += gridDim.x * wpb) {
        const uint32_t id = flag[k];
        const float seed = best_lik[id];
        const unsigned long long key = keys[k];
        const bool have = key != 0ull;
        const float gv = have ? __uint_as_float((uint32_t)(key >> 32)) : 0.f;
        if (!have || gv <= seed || gv <= 0.f) {
            if (lead) orech[id] = 0;
            continue;
        }
        const uint32_t prio = 0xFFFFFFFFu - (uint32_t)(key & 0xFFFFFFFFull);
        const uint32_t g = prio / d.WG, lb = prio % d.WG;
        const uint32_t l = lbits ? (__brev(lb) >> (32 - lbits)) : 0u;
        const uint64_t r = (uint64_t)g * d.WG + l;
        if (r >= items) {
            if (lead) orech[id] = 0;
            continue;
        }
        const uint32_t f = best_lab[id], p = best_idx[id];
        const uint32_t t = (uint32_t)(r % d.M);
        const uint64_t a = (r / d.M) % S2, b = (r / (S2 * d.M)) % S2;
        const uint32_t afi = (uint32_t)(p + a - d.S), asi = (uint32_t)(p + b - d.S);
        const float l1 = warp_lik_value(d, L, z, f, afi);
        const float l2 = warp_lik_value(d, L, z, t, asi);
        if (!lead) continue;
        if (gv < l1 || gv < l2) { orech[id] = 0; continue; }
        if (l1 <= 0.f || l2 <= 0.f) { orech[id] = 0; continue; }
        if (l1 >= l2 && l1 > theta[f]) { best_lik[id] = l1; ov_lab[id] = f; ov_idx[id] = afi; }
        else if (l2 > l1 && l2 > theta[t]) { best_lik[id] = l2; ov_lab[id] = t; ov_idx[id] = asi; }
        else if (l1 > theta[f]) { best_lik[id] = l1; ov_lab[id] = f; ov_idx[id] = afi; }
        else { ov_idx[id] = best_idx[id]; ov_lab[id] = best_lab[id]; orech[id] = 0; }
    }
}

// ---------------------------------------------------------------------------
// check_overlap_reassignments (binary_pursuit.cl:822-875) in ascending order.
// fin(x) = parse(x) && !(moved_left(x) && fin(x-2)); a window's final recheck
// flag is resolved by walking its stride-2 chain back.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool moved_left(const Dims& d, const uint32_t* ov_idx, uint32_t x)
{
    return x > 1 && (uint64_t)ov_idx[x] < (uint64_t)x * d.W;
}

__global__ void reassign_resolve_kernel(Dims d, const uint32_t* __restrict__ flag, DevStatus* status,
                                        const uint8_t* __restrict__ orech, const uint32_t* __restrict__ ov_idx,
                                        uint8_t* orech_fin)
{
    const uint32_t nflag = status->n_flag;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nflag; k += gridDim.x * blockDim.x) {
        const uint32_t id = flag[k];
        if (!orech[id]) { orech_fin[id] = 0; continue; }
        uint32_t j = id;
        int steps = 0;
        while (orech[j] && moved_left(d, ov_idx, j) && steps < kChainCap) { j -= 2; ++steps; }
        if (steps >= kChainCap) { atomicOr(&status->chain_overflow, 1u); orech_fin[id] = 0; continue; }
        uint8_t fv = orech[j] ? 1 : 0;
        for (uint32_t x = j + 2; x <= id; x += 2) fv = (orech[x] && !(moved_left(d, ov_idx, x) && fv)) ? 1 : 0;
        orech_fin[id] = fv;
    }
}

__device__ __forceinline__ void reassign_apply_one(const Dims& d, uint32_t id, bool fin_prev,
                                                   uint32_t* best_idx, uint32_t* best_lab, uint8_t* check,
                                                   const uint32_t* ov_idx, const uint32_t* ov_lab)
{
    const uint64_t start = (uint64_t)id * d.W, end = start + d.W;
    best_idx[id] = ov_idx[id];
    best_lab[id] = ov_lab[id];
    if ((uint64_t)ov_idx[id] < start && id > 1) {
        if (fin_prev) {
            best_idx[id] = 0;
            check[id - 1] = 2;
            check[id] = 2;
            check[id + 1] = 2;
        } else {
            check[id - 2] = 2;
        }
    }
    if ((uint64_t)ov_idx[id] >= end && (uint64_t)id + 2 < d.nwf) check[id + 2] = 2;
}

__global__ void reassign_apply_kernel(Dims d, const uint32_t* __restrict__ flag, const DevStatus* status,
                                      const uint8_t* __restrict__ orech, const uint8_t* __restrict__ orech_fin,
                                      uint32_t* best_idx, uint32_t* best_lab, uint8_t* check,
                                      const uint32_t* __restrict__ ov_idx, const uint32_t* __restrict__ ov_lab)
{
    if (status->chain_overflow) return;
    const uint32_t nflag = status->n_flag;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nflag; k += gridDim.x * blockDim.x) {
        const uint32_t id = flag[k];
        if (!orech[id]) continue;
        const bool prev = id > 1 && orech[id - 2] && orech_fin[id - 2];
        reassign_apply_one(d, id, prev, best_idx, best_lab, check, ov_idx, ov_lab);
    }
}

__global__ void reassign_commit_kernel(const uint32_t* __restrict__ flag, const DevStatus* status,
                                       uint8_t* orech, const uint8_t* __restrict__ orech_fin)
{
    if (status->chain_overflow) return;
    const uint32_t nflag = status->n_flag;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nflag; k += gridDim.x * blockDim.x) {
        const uint32_t id = flag[k];
        if (orech[id]) orech[id] = orech_fin[id];
    }
}

// Sequential form, used only when a chain exceeded the walk limit.
__global__ void reassign_sequential_kernel(Dims d, const uint32_t* __restrict__ flag, const DevStatus* status,
                                           uint8_t* orech, uint32_t* best_idx, uint32_t* best_lab,
                                           uint8_t* check, const uint32_t* __restrict__ ov_idx,
                                           const uint32_t* __restrict__ ov_lab)
{
    if (!status->chain_overflow || threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t nflag = status->n_flag;
    for (uint32_t k = 0; k < nflag; ++k) {
        const uint32_t id = flag[k];
        if (!orech[id]) continue;
        const bool moved = (uint64_t)ov_idx[id] < (uint64_t)id * d.W && id > 1;
        const bool prev = moved && orech[id - 2] == 1;
        reassign_apply_one(d, id, prev, best_idx, best_lab, check, ov_idx, ov_lab);
        if (prev) orech[id] = 0;
    }
}

// ---------------------------------------------------------------------------
// Accept + prune (binary_pursuit kernel, binary_pursuit.cl:918-1063) with
// work-groups of WG list entries in order: inside a group all accepts happen
// first, then the prune rules entry by entry.
// ---------------------------------------------------------------------------
struct AcceptCtx {
    Dims d;
    const uint32_t* list;
    uint32_t n;
    const uint8_t* has;
    const uint8_t* check;   // values at kernel start (c0)
    const float* best_lik;
    const uint32_t* best_lab;
    const uint32_t* best_idx;
    const float* theta;

    __device__ bool at(int64_t k, uint32_t x) const { return k >= 0 && k < (int64_t)n && list[k] == x; }
    __device__ bool same_group(uint32_t a, uint32_t b) const { return a / d.WG == b / d.WG; }
    // does the accept of the window at position kk write 3 into check[x]?
    __device__ bool writes3(uint32_t kk, uint32_t x) const
    {
        if (!has[kk]) return false;
        const uint32_t y = list[kk];
        return x == y || (y > 0 && x == y - 1) || ((uint64_t)y + 1 < d.nwf && x == y + 1);
    }
    __device__ bool guard(uint32_t x) const { return (uint64_t)(x + 1) * d.W < (uint64_t)d.N - d.W; }
    // check[id(k)] when entry k runs its prune rules
    __device__ uint8_t cur(uint32_t k) const
    {
        const uint32_t x = list[k];
        if (has[k]) return 3;
        if (x > 0 && at((int64_t)k - 1, x - 1) && writes3(k - 1, x)) return 3;
        if (at((int64_t)k + 1, x + 1) && same_group(k, k + 1) && writes3(k + 1, x)) return 3;
        return check[x];
    }
    __device__ bool needs_pred(uint32_t k) const
    {
        const uint32_t x = list[k];
        if (has[k] || !guard(x) || x == 0) return false;
        if (!at((int64_t)k - 1, x - 1)) return false;
        return (uint64_t)best_idx[x] < (uint64_t)x * d.W && cur(k) == 1;
    }
    // value of check[id(k)] right after entry k's prune rules
    __device__ uint8_t post(uint32_t k, uint8_t pred_post) const
    {
        const uint32_t x = list[k];
        if (has[k]) return 3;
        uint8_t v = cur(k);
        if (!guard(x)) return v;
        const float ml = best_lik[x];
        const uint32_t lab = best_lab[x], idx = best_idx[x];
        const uint64_t start = (uint64_t)x * d.W, end = start + d.W;
        if (idx < start && v == 1 && x > 0) {
            bool z;
            if (at((int64_t)k - 1, x - 1)) {
                z = pred_post == 0;
            } else {
                uint8_t val = check[x - 1];
                if (x >= 2 && at((int64_t)k - 1, x - 2) && writes3(k - 1, x - 1)) val = 3;
                z = val == 0;
            }
            if (z) v = 0;
        }
        if (idx >= end && v == 1 && (uint64_t)x + 1 < d.nwf) {
            uint8_t val = check[x + 1];
            for (uint32_t dk = 1; dk <= 2; ++dk) {
                const uint64_t kk = (uint64_t)k + dk;
                if (kk < n && same_group(k, (uint32_t)kk) && list[kk] <= x + 2 && writes3((uint32_t)kk, x + 1))
                    val = 3;
            }
            if (val == 0) v = 0;
        }
        if (ml <= theta[lab] && v < 3) v = 0;
        return v;
    }
    __device__ uint8_t final_value(uint32_t k, uint8_t post_v) const
    {
        const uint32_t x = list[k];
        if (writes3(k, x)) return 3;
        if (k > 0 && writes3(k - 1, x)) return 3;
        if (k + 1 < n && writes3(k + 1, x)) return 3;
        return post_v;
    }
};

__global__ void accept_decide_kernel(Dims d, const uint32_t* __restrict__ list, uint32_t n,
                                     const float* __restrict__ theta, const float* __restrict__ best_lik,
                                     const uint32_t* __restrict__ best_lab, const uint32_t* __restrict__ best_idx,
                                     const uint8_t* __restrict__ orech, uint8_t* has)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t id = list[k];
        const uint64_t start = (uint64_t)id * d.W, end = start + d.W;
        float ml = 0.f;
        uint32_t lab = 0, idx = 0;
        if (end < (uint64_t)d.N - d.W) { ml = best_lik[id]; lab = best_lab[id]; idx = best_idx[id]; }
        const bool o = orech[id] == 1;
        has[k] = ((ml > theta[lab] || o) && ((idx >= start && idx < end) || o)) ? 1 : 0;
    }
}

__global__ void accept_prune_kernel(AcceptCtx cx, uint8_t* newval, DevStatus* status)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cx.n; k += gridDim.x * blockDim.x) {
        uint32_t j = k;
        int steps = 0;
        while (cx.needs_pred(j) && steps < kChainCap) { --j; ++steps; }
        if (steps >= kChainCap) { atomicOr(&status->chain_overflow, 2u); continue; }
        uint8_t p = cx.post(j, 0);
        for (uint32_t i = j + 1; i <= k; ++i) p = cx.post(i, p);
        newval[k] = cx.final_value(k, p);
    }
}

__global__ void accept_prune_sequential_kernel(AcceptCtx cx, uint8_t* newval, const DevStatus* status)
{
    if (!(status->chain_overflow & 2u) || threadIdx.x != 0 || blockIdx.x != 0) return;
    uint8_t p = 0;
    for (uint32_t k = 0; k < cx.n; ++k) {
        p = cx.post(k, p);
        newval[k] = cx.final_value(k, p);
    }
}

__global__ void accept_write_kernel(AcceptCtx cx, const uint8_t* __restrict__ newval, uint8_t* check)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cx.n; k += gridDim.x * blockDim.x) {
        const uint32_t x = cx.list[k];
        check[x] = newval[k];
        if (cx.has[k]) {
            if (x > 0 && !cx.at((int64_t)k - 1, x - 1)) check[x - 1] = 3;
            if ((uint64_t)x + 1 < cx.d.nwf && !cx.at((int64_t)k + 1, x + 1)) check[x + 1] = 3;
        }
    }
}

// ---------------------------------------------------------------------------
// Residual (compute_residual, binary_pursuit.cl:57-102).  Spikes whose ranges
// overlap an earlier spike of the list are deferred and applied in list order
// by one CTA; all others are applied in parallel.
// ---------------------------------------------------------------------------
__global__ void residual_parallel_kernel(Dims d, float* V, const float* __restrict__ T,
                                         const uint32_t* __restrict__ idx, const uint32_t* __restrict__ lab,
                                         const uint32_t* __restrict__ win, uint32_t n, uint32_t back,
                                         uint8_t* conf, uint32_t* n_conf)
{
    const uint32_t k = blockIdx.x;
    if (k >= n) return;
    const uint64_t s = idx[k];
    const uint32_t l = lab[k];
    if (l >= d.M) { if (threadIdx.x == 0) conf[k] = 0; return; }
    __shared__ int s_conf;
    if (threadIdx.x == 0) {
        int c = 0;
        for (int64_t kk = (int64_t)k - 1; kk >= 0; --kk) {
            if (win[k] - win[kk] > back) break;
            if (lab[kk] >= d.M) continue;
            const uint64_t s2 = idx[kk];
            if (s < s2 + d.W && s2 < s + d.W) { c = 1; break; }
        }
        s_conf = c;
        conf[k] = (uint8_t)c;
        if (c) atomicAdd(n_conf, 1u);
    }
    __syncthreads();
    if (s_conf) return;
    // one warp per channel row: the row's span [s, min(s+W, N)) is updated with
    // 16-byte loads and stores over its 16-byte-aligned body, scalar at the ends
    // (each element is still one float32 subtraction)
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const uint64_t end = s + d.W < d.N ? s + d.W : d.N;
    for (uint32_t c = warp; c < d.C; c += nwarps) {
        float* row = V + (uint64_t)c * d.N;
        const float* tr = T + ((uint64_t)l * d.C + c) * d.W - s;   // tr[x] = T[l][c][x - s]
        // first index at a 16-byte-aligned address (the row is float-aligned)
        const uint64_t mis = (reinterpret_cast<uintptr_t>(row + s) >> 2) & 3u;
        uint64_t a = s + ((4u - mis) & 3u);
        a = a < end ? a : end;
        const uint64_t b = a + ((end - a) & ~3ull);                    // end of the aligned body
        for (uint64_t x = s + lane; x < a; x += 32) row[x] = fsub(row[x], tr[x]);
        for (uint64_t x = a + 4ull * lane; x < b; x += 128) {
            float4 v = *reinterpret_cast<float4*>(row + x);
            v.x = fsub(v.x, tr[x]);
            v.y = fsub(v.y, tr[x + 1]);
            v.z = fsub(v.z, tr[x + 2]);
            v.w = fsub(v.w, tr[x + 3]);
            *reinterpret_cast<float4*>(row + x) = v;
        }
        for (uint64_t x = b + lane; x < end; x += 32) row[x] = fsub(row[x], tr[x]);
    }
}

__global__ void __launch_bounds__(1024) residual_ordered_kernel(Dims d, float* V, const float* __restrict__ T,
                                                                const uint32_t* __restrict__ idx,
                                                                const uint32_t* __restrict__ lab, uint32_t n,
                                                                const uint8_t* __restrict__ conf,
                                                                const uint32_t* n_conf)
{
    if (*n_conf == 0) return;
    typedef cub::BlockScan<uint32_t, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t todo[1024];
    __shared__ uint32_t s_tot;
    const uint32_t CW = d.C * d.W;
    for (uint32_t b0 = 0; b0 < n; b0 += 1024) {
        const uint32_t k = b0 + threadIdx.x;
        const uint32_t f = (k < n && conf[k]) ? 1u : 0u;
        uint32_t off, tot;
        Scan(tmp).ExclusiveSum(f, off, tot);
        if (f) todo[off] = k;
        if (threadIdx.x == 0) s_tot = tot;
        __syncthreads();
        for (uint32_t i = 0; i < s_tot; ++i) {
            const uint32_t kk = todo[i];
            const uint64_t s = idx[kk];
            const uint32_t l = lab[kk];
            for (uint32_t e = threadIdx.x; e < CW; e += blockDim.x) {
                const uint32_t c = e / d.W, j = e - c * d.W;
                if (s + j >= d.N) continue;
                float* vp = V + (uint64_t)c * d.N + s + j;
                *vp = fsub(*vp, T[((uint64_t)l * d.C + c) * d.W + j]);
            }
            __syncthreads();
        }
        __syncthreads();
    }
}

// get_adjusted_clips (binary_pursuit.cl:1088-1130)
__global__ void clips_kernel(Dims d, const float* __restrict__ V, const float* __restrict__ T,
                             const uint32_t* __restrict__ idx, const uint32_t* __restrict__ lab, uint32_t n,
                             float* clips)
{
    const uint32_t CW = d.C * d.W;
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const uint64_t s = idx[k];
        const uint32_t l = lab[k];
        if (l >= d.M) continue;
        for (uint32_t e = threadIdx.x; e < CW; e += blockDim.x) {
            const uint32_t c = e / d.W, j = e - c * d.W;
            if (s + j >= d.N) continue;
            clips[(uint64_t)k * CW + e] = fadd(V[(uint64_t)c * d.N + s + j], T[((uint64_t)l * d.C + c) * d.W + j]);
        }
    }
}

inline uint32_t grid_for(uint64_t n, uint32_t threads, uint32_t cap = 148 * 32)
{
    uint64_t g = (n + threads - 1) / threads;
    if (g == 0) g = 1;
    return (uint32_t)(g < cap ? g : cap);
}

}  // namespace

int launch_iota(uint32_t* list, uint32_t n, cudaStream_t st)
{
    count_launch();
    iota_kernel<<<grid_for(n, 256), 256, 0, st>>>(list, n);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_likelihood_exact(const Dims& d, const float* V, const float* T, const float* bias,
                            const uint32_t* list, uint32_t nlist, float* L, cudaStream_t st)
{
    if (nlist == 0) return FBP_OK;
    if (d.W > 1024) return fail(FBP_E_ARG, "template_len above 1024 is not supported");
    const uint32_t SW = (2 * d.W + 3) & ~3u, Wp = (d.W + 3) & ~3u;
    const size_t strip = (size_t)d.C * SW * 4, per_t = (size_t)d.C * Wp * 4;
    const size_t budget = 200 * 1024;
    const uint32_t threads = (d.W + 31) & ~31u;
    const uint32_t grid = nlist < (1u << 30) ? nlist : (1u << 30);
    int Q = 8;
    while (Q > 1 && strip + Q * per_t > budget) Q >>= 1;
    const size_t smem = strip + Q * per_t;
    if (smem > budget) return fail(FBP_E_ARG, "channels x template_len too large for the likelihood kernel");
#define FBP_LIK(QQ)                                                                               \
    case QQ:                                                                                      \
        FBP_CUDA(allow_max_dyn_smem(lik_exact_kernel<QQ>)); \
        lik_exact_kernel<QQ><<<grid, threads, smem, st>>>(d, V, T, bias, list, nlist, L);       \
        break;
    count_launch();
    KScope ks(&fbp_chunk_stats::ms_lik_exact, st);
    switch (Q) {
        FBP_LIK(8)
        FBP_LIK(4)
        FBP_LIK(2)
        FBP_LIK(1)
    }
#undef FBP_LIK
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_argmax(const Dims& d, const Work& w, const uint32_t* list, uint32_t nlist, cudaStream_t st)
{
    if (nlist == 0) return FBP_OK;
    const uint32_t threads = 256;
    const uint64_t warps = nlist;
    count_launch();
    argmax_kernel<<<grid_for(warps * 32, threads, 148 * 64), threads, 0, st>>>(
        d, w.L(), list, nlist, w.best_lik(), w.best_lab(), w.best_idx(), w.check(), w.orech(),
        w.ov_idx(), w.ov_lab());
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_compact_flagged(const Dims& d, const Work& w, uint32_t nlist, cudaStream_t st)
{
    (void)d;
    FlagF f{w.list(), w.orech(), w.flag()};
    return compact(f, nullptr, nlist, w.blk(), &w.status()->n_flag, st);
}

int launch_overlap_plain(const Dims& d, const Work& w, const float* V, const float* T, const float* theta,
                         uint32_t nflag_max, cudaStream_t st)
{
    if (nflag_max == 0) return FBP_OK;
    const uint32_t S2 = 2 * d.S + 1;
    const uint32_t RW = d.W + 2 * d.S + 4;
    size_t smem = ((size_t)2 * d.C * RW + (size_t)d.C * d.W) * 4 + 2 * (size_t)S2;
    smem = (smem + 15) & ~(size_t)15;
    smem += (size_t)kOvRound * 4 + 16;
    if (smem > 220 * 1024) return fail(FBP_E_ARG, "overlap recheck working set exceeds shared memory");
    FBP_CUDA(allow_max_dyn_smem(overlap_plain_kernel));
    FBP_CUDA(cudaMemsetAsync(w.keys(), 0, sizeof(unsigned long long) * nflag_max, st));
    const uint64_t tasks = (uint64_t)nflag_max * d.M;
    const uint32_t grid = (uint32_t)(tasks < 148ull * 8 ? tasks : 148ull * 8);
    count_launch();
    KScope ks(&fbp_chunk_stats::ms_overlap_plain, st);
    overlap_plain_kernel<<<grid, kOvThreads, smem, st>>>(d, V, T, w.L(), theta, w.flag(), w.status(),
                                                         w.best_lab(), w.best_idx(), w.keys(),
                                                         &w.status()->pair_items);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_parse_reassign(const Dims& d, const Work& w, const float* theta, uint32_t nflag_max, cudaStream_t st,
                          const float* V, const float* T, const float* bias, bool lazy)
{
    if (nflag_max == 0) return FBP_OK;
    const uint32_t g = grid_for(nflag_max, 256);
    const uint32_t gw = grid_for(nflag_max, 8);   // parse: one warp per window
    LazyRef z{nullptr, nullptr, V, T, bias};
    if (lazy) {
        z.wflag = w.at<uint8_t>(w.lay->off_wflag);
        z.tnorm = w.at<float>(w.lay->off_tnorm);
    }
    count_launch(5);
    parse_kernel<<<gw, 256, 0, st>>>(d, w.L(), theta, w.flag(), w.status(), w.keys(), w.best_lik(),
                                    w.best_lab(), w.best_idx(), w.orech(), w.ov_idx(), w.ov_lab(), z);
    reassign_resolve_kernel<<<g, 256, 0, st>>>(d, w.flag(), w.status(), w.orech(), w.ov_idx(), w.orech_fin());
    reassign_apply_kernel<<<g, 256, 0, st>>>(d, w.flag(), w.status(), w.orech(), w.orech_fin(), w.best_idx(),
                                             w.best_lab(), w.check(), w.ov_idx(), w.ov_lab());
    reassign_sequential_kernel<<<1, 32, 0, st>>>(d, w.flag(), w.status(), w.orech(), w.best_idx(), w.best_lab(),
                                                  w.check(), w.ov_idx(), w.ov_lab());
    reassign_commit_kernel<<<g, 256, 0, st>>>(w.flag(), w.status(), w.orech(), w.orech_fin());
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_accept(const Dims& d, const Work& w, const float* theta, uint32_t nlist, cudaStream_t st)
{
    if (nlist == 0) {
        FBP_CUDA(cudaMemsetAsync(&w.status()->n_spikes, 0, 4, st));
        return FBP_OK;
    }
    const uint32_t g = grid_for(nlist, 256);
    count_launch(4);
    accept_decide_kernel<<<g, 256, 0, st>>>(d, w.list(), nlist, theta, w.best_lik(), w.best_lab(),
                                            w.best_idx(), w.orech(), w.has());
    AcceptCtx cx{d, w.list(), nlist, w.has(), w.check(), w.best_lik(), w.best_lab(), w.best_idx(), theta};
    accept_prune_kernel<<<g, 256, 0, st>>>(cx, w.newval(), w.status());
    accept_prune_sequential_kernel<<<1, 32, 0, st>>>(cx, w.newval(), w.status());
    accept_write_kernel<<<g, 256, 0, st>>>(cx, w.newval(), w.check());
    FBP_CUDA(cudaGetLastError());
    SpikeF f{w.list(), w.has(), w.best_idx(), w.best_lab(), w.pidx(), w.plab(), w.pwin()};
    return compact(f, nullptr, nlist, w.blk(), &w.status()->n_spikes, st);
}

int launch_next_list(const Dims& d, const Work& w, cudaStream_t st)
{
    NextF f{w.check(), w.list2()};
    return compact(f, nullptr, d.nw, w.blk(), &w.status()->n_next, st);
}

int launch_residual(const Dims& d, const Work& w, float* V, const float* T, const uint32_t* idx,
                    const uint32_t* lab, const uint32_t* win, uint32_t n, cudaStream_t st)
{
    if (n == 0) return FBP_OK;
    const uint32_t back = 4 + 2 * ((d.S + d.W - 1) / d.W);
    FBP_CUDA(cudaMemsetAsync(&w.status()->n_conf, 0, 4, st));
    count_launch(2);
    residual_parallel_kernel<<<n, 128, 0, st>>>(d, V, T, idx, lab, win, n, back, w.pconf(), &w.status()->n_conf);
    residual_ordered_kernel<<<1, 1024, 0, st>>>(d, V, T, idx, lab, n, w.pconf(), &w.status()->n_conf);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_adjusted_clips(const Dims& d, const float* V, const float* T, const uint32_t* idx,
                          const uint32_t* lab, uint32_t n, float* clips, cudaStream_t st)
{
    if (n == 0) return FBP_OK;
    count_launch();
    clips_kernel<<<n < 65535u * 4 ? n : 65535u * 4, 128, 0, st>>>(d, V, T, idx, lab, n, clips);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

}  // namespace fbp
