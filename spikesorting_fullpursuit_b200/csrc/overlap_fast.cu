// overlap_fast.cu -- overlap recheck by screening, with exact results.
//
// The reference scores every item (a, t, b) of a flagged window
// (overlap_recheck_indices, binary_pursuit.cl:444-654) with C*W sequential
// float operations.  Its value expands as
//     v(a,t,b) = G_f(a) + G_t(b) - X_ft(a,b)
//     G_x(s)   = sum_cj X_s[c,j] v[c,j] - 0.5 sum_cj X_s[c,j]^2   (X_s: template x
//                shifted by s-S and cut to the window)
//     X_ft     = sum_cj F_a[c,j] T_b[c,j]
// G is a partial correlation of every template with the window (computed per
// window), X_ft depends only on the template pair and the two shifts (a table
// built once per call).  |v_ref - estimate| is bounded rigorously by a
// function of truncated template energies and the window's norm (see
// est_bound in screen_kernel).  Only items whose interval can reach the best lower bound (and
// the window's seed likelihood) are scored exactly in the reference's float
// order; the winner key -- value, then work-group, then tree slot -- is
// therefore the reference's.
#include <cub/cub.cuh>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }

// Truncated energy of template t at shift x: sum over the template samples u
// that land inside the window, u in [S-x, S-x+W) and [0, W).
__global__ void energy_table_kernel(Dims d, const float* __restrict__ T, double* Et)
{
    const uint32_t S2 = 2 * d.S + 1;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < d.M * S2; i += gridDim.x * blockDim.x) {
        const uint32_t t = i / S2, x = i % S2;
        const int lo = max(0, (int)d.S - (int)x), hi = min((int)d.W, (int)d.S - (int)x + (int)d.W);
        double e = 0.0;
        for (uint32_t c = 0; c < d.C; ++c) {
            const float* r = T + ((uint64_t)t * d.C + c) * d.W;
            for (int u = lo; u < hi; ++u) e += (double)r[u] * (double)r[u];
        }
        Et[i] = e;
    }
}

// Pair cross terms X_ft(a, b) for |a-b| <= W, one CTA per (f, t): products
// P_delta[u] = sum_c F[c,u] T[c,u+delta] in double, prefix sums over u, then
// X_ft(a, b) = Q_delta[hi] - Q_delta[lo] with delta = a-b.
constexpr int kLagChunk = 16;

__global__ void __launch_bounds__(256) cross_table_kernel(Dims d, const float* __restrict__ T, float* XT)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const uint32_t f = blockIdx.x / d.M, t = blockIdx.x % d.M;
    const uint32_t S2 = 2 * d.S + 1, W = d.W, C = d.C;
    float* Fs = reinterpret_cast<float*>(smraw);
    float* Ts = Fs + C * W;
    double* Q = reinterpret_cast<double*>(Ts + C * W);  // [kLagChunk][W+1]; 8*C*W bytes in, aligned
    for (uint32_t e = threadIdx.x; e < C * W; e += blockDim.x) {
        Fs[e] = T[(uint64_t)f * C * W + e];
        Ts[e] = T[(uint64_t)t * C * W + e];
    }
    __syncthreads();
    const int dmax = (int)min(W, 2 * d.S);
    for (int d0 = -dmax; d0 <= dmax; d0 += kLagChunk) {
        for (uint32_t e = threadIdx.x; e < kLagChunk * W; e += blockDim.x) {
            const int li = e / W, u = e % W, delta = d0 + li;
            double acc = 0.0;
            if (delta <= dmax && u + delta >= 0 && u + delta < (int)W)
                for (uint32_t c = 0; c < C; ++c) acc += (double)Fs[c * W + u] * (double)Ts[c * W + u + delta];
            Q[li * (W + 1) + u + 1] = acc;
        }
        __syncthreads();
        if (threadIdx.x < kLagChunk) {
            double* q = Q + threadIdx.x * (W + 1);
            q[0] = 0.0;
            for (uint32_t u = 1; u <= W; ++u) q[u] += q[u - 1];
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < kLagChunk * S2; e += blockDim.x) {
            const int li = e / S2, a = e % S2, delta = d0 + li;
            const int b = a - delta;
            if (delta > dmax || b < 0 || b >= (int)S2) continue;
            const int lo = max(max(0, -delta), (int)d.S - a);
            const int hi = min(min((int)W, (int)W - delta), (int)d.S - a + (int)W);
            const double v = hi > lo ? Q[li * (W + 1) + hi] - Q[li * (W + 1) + lo] : 0.0;
            XT[(((uint64_t)f * d.M + t) * S2 + a) * S2 + b] = (float)v;
        }
        __syncthreads();
    }
}

// Template processing order for the partial correlations: sorted by the
// first non-zero channel so groups of neighbouring templates share channels.
__global__ void template_order_kernel(Dims d, const float* __restrict__ T, uint32_t* perm)
{
    extern __shared__ uint32_t key[];
    for (uint32_t t = threadIdx.x; t < d.M; t += blockDim.x) {
        uint32_t first = d.C;
        for (uint32_t c = 0; c < d.C && first == d.C; ++c)
            for (uint32_t j = 0; j < d.W; ++j)
                if (T[((uint64_t)t * d.C + c) * d.W + j] != 0.f) { first = c; break; }
        key[t] = first;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t t = 0; t < d.M; ++t) perm[t] = t;
        for (uint32_t i = 1; i < d.M; ++i) {  // stable insertion sort by key
            const uint32_t v = perm[i];
            int j = (int)i - 1;
            while (j >= 0 && key[perm[j]] > key[v]) { perm[j + 1] = perm[j]; --j; }
            perm[j + 1] = v;
        }
    }
}

__device__ __forceinline__ bool window_skipped(const Dims& d, const float* L, const float* theta, uint32_t f,
                                               uint32_t p)
{
    return L[(uint64_t)f * d.N + p] < theta[f] || (uint64_t)p >= (uint64_t)d.N - d.W;
}

// Partial correlations G[k][t][b] = X_t(b) - 0.5 Et[t][b] of every template
// with the flagged window (masked to [p, p+W)).  One CTA per (window, group
// of Q templates in perm order), one thread per shift b.
template <int Q>
__global__ void __launch_bounds__(1024) partial_corr_kernel(Dims d, const float* __restrict__ V,
                                                            const float* __restrict__ T,
                                                            const float* __restrict__ L,
                                                            const float* __restrict__ theta,
                                                            const double* __restrict__ Et,
                                                            const uint32_t* __restrict__ perm,
                                                            const uint32_t* __restrict__ flag,
                                                            const DevStatus* status,
                                                            const uint32_t* __restrict__ best_lab,
                                                            const uint32_t* __restrict__ best_idx,
                                                            uint32_t k0, float* G)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ uint32_t chans[256];
    __shared__ uint32_t nch;
    const uint32_t k = k0 + blockIdx.x;
    if (k >= status->n_flag) return;
    const uint32_t id = flag[k];
    const uint32_t f = best_lab[id], p = best_idx[id];
    if (window_skipped(d, L, theta, f, p)) return;
    const uint32_t S2 = 2 * d.S + 1, W = d.W, C = d.C;
    const uint32_t SL = (2 * d.S + W + 3) & ~3u;
    const uint32_t Wp = (W + 3) & ~3u;
    float* Vs = sm;                  // [C][SL] window masked into a zero strip
    float* Ts = sm + C * SL;         // [Q][C][Wp]
    const uint32_t tq = C * Wp;
    const uint32_t g0 = blockIdx.y * Q;
    for (uint32_t e = threadIdx.x; e < C * SL; e += blockDim.x) {
        const uint32_t c = e / SL, y = e - c * SL;
        Vs[e] = (y >= d.S && y < d.S + W) ? V[(uint64_t)c * d.N + p - d.S + y] : 0.f;
    }
    for (uint32_t e = threadIdx.x; e < Q * tq; e += blockDim.x) {
        const uint32_t q = e / tq, r = e - q * tq, c = r / Wp, j = r - c * Wp;
        const uint32_t gi = g0 + q;
        Ts[e] = (gi < d.M && j < W) ? T[((uint64_t)perm[gi] * C + c) * W + j] : 0.f;
    }
    if (threadIdx.x == 0) nch = 0;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
        bool nz = false;
        for (uint32_t q = 0; q < Q && !nz; ++q)
            for (uint32_t j = 0; j < W; ++j)
                if (Ts[q * tq + c * Wp + j] != 0.f) { nz = true; break; }
        if (nz) chans[atomicAdd(&nch, 1u)] = c;  // order is irrelevant for an estimate
    }
    __syncthreads();
    const uint32_t b = threadIdx.x;
    if (b >= S2) return;
    float acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) acc[q] = 0.f;
    for (uint32_t ci = 0; ci < nch; ++ci) {
        const uint32_t c = chans[ci];
        const float* vr = Vs + c * SL + b;
        const float* tr = Ts + c * Wp;
        uint32_t j = 0;
        for (; j + 4 <= W; j += 4) {
            const float v0 = vr[j], v1 = vr[j + 1], v2 = vr[j + 2], v3 = vr[j + 3];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float4 t4 = *reinterpret_cast<const float4*>(tr + q * tq + j);
                acc[q] = fmaf(t4.x, v0, acc[q]);
                acc[q] = fmaf(t4.y, v1, acc[q]);
                acc[q] = fmaf(t4.z, v2, acc[q]);
                acc[q] = fmaf(t4.w, v3, acc[q]);
            }
        }
        for (; j < W; ++j) {
            const float v = vr[j];
#pragma unroll
            for (int q = 0; q < Q; ++q) acc[q] = fmaf(tr[q * tq + j], v, acc[q]);
        }
    }
    float* Gk = G + (uint64_t)(k - k0) * d.M * S2;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const uint32_t gi = g0 + q;
        if (gi < d.M) {
            const uint32_t t = perm[gi];
            Gk[(uint64_t)t * S2 + b] = (float)((double)acc[q] - 0.5 * Et[(uint64_t)t * S2 + b]);
        }
    }
}

// Exact pair likelihood in the reference's float order (binary_pursuit.cl:578-632).
__device__ float pair_exact(const Dims& d, const float* __restrict__ T, const float* __restrict__ V,
                            uint32_t f, uint32_t t, uint32_t p, uint32_t a, uint32_t b)
{
    const int W = (int)d.W, fa = (int)d.S - (int)a, ta = (int)d.S - (int)b;
    float acc = 0.f;
    for (uint32_t c = 0; c < d.C; ++c) {
        const float* fr = T + ((uint64_t)f * d.C + c) * d.W;
        const float* tr = T + ((uint64_t)t * d.C + c) * d.W;
        const float* vr = V + (uint64_t)c * d.N + p;
        float ss = 0.f;
        for (int j = 0; j < W; ++j) {
            const int xf = fa + j, xt = ta + j;
            const float fv = (xf >= 0 && xf < W) ? fr[xf] : 0.f;
            const float tv = (xt >= 0 && xt < W) ? tr[xt] : 0.f;
            const float s = fadd(fv, tv);
            ss = fadd(ss, fmul(s, s));
            acc = fadd(acc, fmul(s, vr[j]));
        }
        if (ss > 0.f) acc = fsub(acc, fmul(0.5f, ss));
    }
    return acc;
}

__device__ __forceinline__ uint32_t item_priority(uint64_t r, uint32_t WG, uint32_t lbits)
{
    const uint32_t g = (uint32_t)(r / WG), l = (uint32_t)(r % WG);
    const uint32_t br = lbits ? (__brev(l) >> (32 - lbits)) : 0u;
    return g * WG + br;
}

constexpr int kScrThreads = 256;

struct ScreenShared {
    double lb;
    double nv;
    unsigned long long best;
    uint32_t nA;
    uint32_t nTB;
};

// Screening of one flagged window per CTA.
__global__ void __launch_bounds__(kScrThreads) screen_kernel(
    Dims d, const float* __restrict__ V, const float* __restrict__ T, const float* __restrict__ L,
    const float* __restrict__ theta, const double* __restrict__ Et, const float* __restrict__ XT,
    const float* __restrict__ G, uint32_t k0, uint32_t kcount, const uint32_t* __restrict__ flag,
    DevStatus* status, const uint32_t* __restrict__ best_lab, const uint32_t* __restrict__ best_idx,
    const float* __restrict__ best_lik, unsigned long long* keys)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ ScreenShared sh;
    typedef cub::BlockReduce<double, kScrThreads> RD;
    typedef cub::BlockScan<uint32_t, kScrThreads> SC;
    __shared__ union {
        typename RD::TempStorage rd;
        typename SC::TempStorage sc;
    } tmp;
    const uint32_t S = d.S, W = d.W, M = d.M, S2 = 2 * S + 1;
    uint8_t* fa = smraw;                                            // [S2] bit0 in bounds, bit1 L_f > 0
    uint8_t* pt = fa + ((S2 + 15) & ~15u);                          // [M][S2] L_t > 0
    uint32_t* alist = reinterpret_cast<uint32_t*>(pt + ((M * S2 + 15) & ~15u));  // [S2]
    uint32_t* tb = alist + S2;                                      // [M*S2] (t,b) with L_t > 0
    const uint64_t items = (uint64_t)S2 * S2 * M;
    const uint64_t nloc = (items - 1) / d.WG + 1;
    const uint64_t slots = nloc * d.WG;
    uint32_t lbits = 0;
    while ((1u << lbits) < d.WG) ++lbits;
    const double u = 1.0 / 16777216.0;
    const double K = 1.05 * u * 2.0 * ((double)d.C * W + d.C + W + 8);
    const uint32_t nflag = status->n_flag;
    unsigned long long exact_n = 0, item_n = 0;
    for (uint32_t kk = blockIdx.x; kk < kcount; kk += gridDim.x) {
        const uint32_t k = k0 + kk;
        if (k >= nflag) break;
        const uint32_t id = flag[k];
        const uint32_t f = best_lab[id], p = best_idx[id];
        if (window_skipped(d, L, theta, f, p)) continue;
        const float seed = best_lik[id];
        const float* Gk = G + (uint64_t)kk * M * S2;
        __syncthreads();
        // window norm, shift flags, positive-likelihood flags
        double nv2 = 0.0;
        for (uint32_t e = threadIdx.x; e < d.C * W; e += blockDim.x) {
            const uint32_t c = e / W, j = e - c * W;
            const double v = V[(uint64_t)c * d.N + p + j];
            nv2 += v * v;
        }
        const double nvs = RD(tmp.rd).Sum(nv2);
        if (threadIdx.x == 0) { sh.nv = sqrt(nvs) * 1.001; sh.best = 0ull; sh.nA = 0; }
        for (uint32_t x = threadIdx.x; x < S2; x += blockDim.x) {
            const uint64_t xp = (uint64_t)x + p;
            const bool inb = xp >= S && xp < (uint64_t)d.N - W + S;
            fa[x] = inb ? ((L[(uint64_t)f * d.N + xp - S] > 0.f) ? 3 : 1) : 0;
        }
        for (uint32_t e = threadIdx.x; e < M * S2; e += blockDim.x) {
            const uint32_t t = e / S2, x = e - t * S2;
            const uint64_t xp = (uint64_t)x + p;
            const bool inb = xp >= S && xp < (uint64_t)d.N - W + S;
            pt[e] = (inb && L[(uint64_t)t * d.N + xp - S] > 0.f) ? 1 : 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t n = 0;
            for (uint32_t x = 0; x < S2; ++x) if (fa[x] == 3) alist[n++] = x;
            sh.nA = n;
        }
        // compact the (t, b) pairs with L_t > 0
        {
            uint32_t base = 0;
            for (uint32_t r0 = 0; r0 < M * S2; r0 += blockDim.x) {
                const uint32_t e = r0 + threadIdx.x;
                const uint32_t fl = (e < M * S2 && pt[e]) ? 1u : 0u;
                uint32_t off, tot;
                SC(tmp.sc).ExclusiveSum(fl, off, tot);
                if (fl) tb[base + off] = e;
                base += tot;
                __syncthreads();
            }
            if (threadIdx.x == 0) sh.nTB = base;
        }
        __syncthreads();
        const uint32_t nA = sh.nA, nTB = sh.nTB;
        const double nv = sh.nv;
        // item enumeration: (a in A+, all t, b) then ((t,b) with L_t > 0, a not in A+)
        auto est_bound = [&](uint32_t a, uint32_t t, uint32_t b, double& est, double& bound) {
            const double ef = Et[(uint64_t)f * S2 + a], et = Et[(uint64_t)t * S2 + b];
            est = (double)Gk[(uint64_t)f * S2 + a] + (double)Gk[(uint64_t)t * S2 + b] -
                  (double)XT[(((uint64_t)f * M + t) * S2 + a) * S2 + b];
            bound = K * ((sqrt(ef) + sqrt(et)) * nv + ef + et);
        };
        const uint64_t n1 = (uint64_t)nA * M * S2;
        const uint64_t n2 = (uint64_t)nTB * S2;
        // pass 1: lower bound on the best pair value
        double lb = -1e300;
        for (uint64_t i = threadIdx.x; i < n1 + n2; i += blockDim.x) {
            uint32_t a, t, b;
            if (i < n1) {
                b = (uint32_t)(i % S2);
                const uint64_t r = i / S2;
                t = (uint32_t)(r % M);
                a = alist[r / M];
                if (!(fa[b] & 1) || (a > b ? a - b : b - a) > W) continue;
            } else {
                const uint64_t i2 = i - n1;
                a = (uint32_t)(i2 % S2);
                const uint32_t e = tb[i2 / S2];
                t = e / S2;
                b = e - t * S2;
                if (fa[a] != 1 || (a > b ? a - b : b - a) > W) continue;
            }
            double est, bound;
            est_bound(a, t, b, est, bound);
            lb = fmax(lb, est - bound);
            ++item_n;
        }
        const double lbs = RD(tmp.rd).Reduce(lb, cub::Max());
        if (threadIdx.x == 0) sh.lb = lbs;
        __syncthreads();
        const double thr = fmax(fmax(sh.lb, (double)seed), 0.0);
        // pass 2: exact scores of the items that can reach the threshold
        unsigned long long kbest = 0ull;
        for (uint64_t i = threadIdx.x; i < n1 + n2; i += blockDim.x) {
            uint32_t a, t, b;
            if (i < n1) {
                b = (uint32_t)(i % S2);
                const uint64_t r = i / S2;
                t = (uint32_t)(r % M);
                a = alist[r / M];
                if (!(fa[b] & 1) || (a > b ? a - b : b - a) > W) continue;
            } else {
                const uint64_t i2 = i - n1;
                a = (uint32_t)(i2 % S2);
                const uint32_t e = tb[i2 / S2];
                t = e / S2;
                b = e - t * S2;
                if (fa[a] != 1 || (a > b ? a - b : b - a) > W) continue;
            }
            double est, bound;
            est_bound(a, t, b, est, bound);
            if (est + bound < thr) continue;
            const float v = pair_exact(d, T, V, f, t, p, a, b);
            ++exact_n;
            if (!(v > 0.f)) continue;
            const uint64_t r = (uint64_t)t + (uint64_t)M * a + (uint64_t)M * S2 * b;
            uint32_t pr = item_priority(r, d.WG, lbits);
            for (uint64_t rr = r + items; rr < slots; rr += items) {
                const uint32_t p2 = item_priority(rr, d.WG, lbits);
                pr = p2 < pr ? p2 : pr;
            }
            const unsigned long long key =
                ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xFFFFFFFFu - pr);
            kbest = key > kbest ? key : kbest;
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_down_sync(0xffffffffu, kbest, off);
            kbest = o > kbest ? o : kbest;
        }
        if ((threadIdx.x & 31) == 0 && kbest) atomicMax(&sh.best, kbest);
        __syncthreads();
        if (threadIdx.x == 0 && sh.best) keys[k] = sh.best;
    }
    if (exact_n) atomicAdd(&status->n_pair_exact, (uint32_t)exact_n);
    if (item_n) atomicAdd(&status->pair_items, item_n);
}

}  // namespace

int launch_overlap_tables(const Dims& d, const Work& w, const float* T, cudaStream_t st)
{
    const Layout& L = *w.lay;
    if (!L.screened) return FBP_OK;
    const uint32_t S2 = 2 * d.S + 1;
    energy_table_kernel<<<(d.M * S2 + 255) / 256, 256, 0, st>>>(d, T, w.at<double>(L.off_et));
    const size_t smem = (size_t)2 * d.C * d.W * 4 + 8 + (size_t)kLagChunk * (d.W + 1) * 8;
    if (smem > 200 * 1024) return fail(FBP_E_ARG, "template too large for the pair table kernel");
    FBP_CUDA(cudaFuncSetAttribute(cross_table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cross_table_kernel<<<d.M * d.M, 256, smem, st>>>(d, T, w.at<float>(L.off_xt));
    template_order_kernel<<<1, 256, d.M * 4, st>>>(d, T, w.at<uint32_t>(L.off_perm));
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_overlap_fast(const Dims& d, const Work& w, const float* V, const float* T, const float* theta,
                        uint32_t nflag_max, cudaStream_t st)
{
    const Layout& L = *w.lay;
    if (!L.screened) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    if (nflag_max == 0) return FBP_OK;
    const uint32_t S2 = 2 * d.S + 1;
    if (S2 > 1024 || d.C > 256) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    FBP_CUDA(cudaMemsetAsync(w.keys(), 0, sizeof(unsigned long long) * nflag_max, st));
    const uint32_t SL = (2 * d.S + d.W + 3) & ~3u, Wp = (d.W + 3) & ~3u;
    const size_t strip = (size_t)d.C * SL * 4, per_t = (size_t)d.C * Wp * 4;
    int Q = 8;
    while (Q > 1 && strip + Q * per_t > 200 * 1024) Q >>= 1;
    const size_t smem_a = strip + Q * per_t;
    if (smem_a > 200 * 1024) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    const size_t smem_b = ((S2 + 15) & ~15u) + (((size_t)d.M * S2 + 15) & ~(size_t)15) + (size_t)S2 * 4 +
                          (size_t)d.M * S2 * 4;
    if (smem_b > 200 * 1024) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    FBP_CUDA(cudaFuncSetAttribute(screen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
    const uint32_t threads_a = (S2 + 31) & ~31u;
    const uint32_t groups = (d.M + Q - 1) / Q;
    float* G = w.at<float>(L.off_g);
    const double* Et = w.at<double>(L.off_et);
    const float* XT = w.at<float>(L.off_xt);
    const uint32_t* perm = w.at<uint32_t>(L.off_perm);
    for (uint32_t k0 = 0; k0 < nflag_max; k0 += (uint32_t)L.gbatch) {
        const uint32_t kc = (uint32_t)((nflag_max - k0) < L.gbatch ? (nflag_max - k0) : L.gbatch);
        dim3 ga(kc, groups);
#define FBP_PC(QQ)                                                                                       \
    case QQ:                                                                                             \
        FBP_CUDA(cudaFuncSetAttribute(partial_corr_kernel<QQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a)); \
        partial_corr_kernel<QQ><<<ga, threads_a, smem_a, st>>>(d, V, T, w.L(), theta, Et, perm, w.flag(), w.status(), \
                                                              w.best_lab(), w.best_idx(), k0, G);        \
        break;
        switch (Q) {
            FBP_PC(8)
            FBP_PC(4)
            FBP_PC(2)
            FBP_PC(1)
        }
#undef FBP_PC
        const uint32_t gb = kc < 148u * 8 ? kc : 148u * 8;
        screen_kernel<<<gb, kScrThreads, smem_b, st>>>(d, V, T, w.L(), theta, Et, XT, G, k0, kc, w.flag(), w.status(),
                                                       w.best_lab(), w.best_idx(), w.best_lik(), w.keys());
        FBP_CUDA(cudaGetLastError());
    }
    return FBP_OK;
}

}  // namespace fbp
