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
// that land inside the window, u in [S-x, S-x+W) and [0, W).  Stored as
// (E, sqrt(E)), each rounded up, for the screening bound and the partial
// correlations.
__global__ void energy_table_kernel(Dims d, const float* __restrict__ T, float2* Et)
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
        Et[i] = make_float2(__double2float_ru(e * (1.0 + 1e-12)), __double2float_ru(sqrt(e) * (1.0 + 1e-12)));
    }
}

// Pair cross terms X_ft(a, b) for |a-b| <= W, one CTA per (f, t): products
// P_delta[u] = sum_c F[c,u] T[c,u+delta] in double, prefix sums over u, then
// X_ft(a, b) = Q_delta[hi] - Q_delta[lo] with delta = a-b.
constexpr int kLagChunk = 16;

__global__ void __launch_bounds__(256) cross_table_kernel(Dims d, const float* __restrict__ T, float* XT,
                                                          float* max_negx)
{
    typedef cub::BlockReduce<float, 256> RF;
    __shared__ typename RF::TempStorage rtmp;
    float mneg = 0.f;
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
            const float xv = (float)v;
            XT[(((uint64_t)f * d.M + t) * S2 + a) * S2 + b] = xv;
            mneg = fmaxf(mneg, -xv);
        }
        __syncthreads();
    }
    const float m = RF(rtmp).Reduce(mneg, cub::Max());
    if (threadIdx.x == 0) max_negx[blockIdx.x] = m;
}

// Per template: max over shifts of sqrt(E) and of E (bounds for whole rows).
__global__ void energy_max_kernel(Dims d, const float2* __restrict__ Et, float* maxs)
{
    const uint32_t S2 = 2 * d.S + 1;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < d.M; t += gridDim.x * blockDim.x) {
        float ms = 0.f, me = 0.f;
        for (uint32_t x = 0; x < S2; ++x) {
            ms = fmaxf(ms, Et[(uint64_t)t * S2 + x].y);
            me = fmaxf(me, Et[(uint64_t)t * S2 + x].x);
        }
        maxs[t] = ms;
        maxs[d.M + t] = me;
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
                                                            const float2* __restrict__ Et,
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
            Gk[(uint64_t)t * S2 + b] = acc[q] - 0.5f * Et[(uint64_t)t * S2 + b].x;
        }
    }
}

// Exact pair likelihood in the reference's float order (binary_pursuit.cl:578-632),
// with the window's voltage vw[C][W] in shared memory.
__device__ float pair_exact_sv(const Dims& d, const float* __restrict__ T, const float* vw, uint32_t f, uint32_t t,
                               uint32_t a, uint32_t b)
{
    const int W = (int)d.W, fa = (int)d.S - (int)a, ta = (int)d.S - (int)b;
    const int jlo_f = max(0, -fa), jhi_f = min(W, W - fa);
    const int jlo_t = max(0, -ta), jhi_t = min(W, W - ta);
    float acc = 0.f;
    for (uint32_t c = 0; c < d.C; ++c) {
        const float* fr = T + ((uint64_t)f * d.C + c) * d.W + fa;
        const float* tr = T + ((uint64_t)t * d.C + c) * d.W + ta;
        const float* vr = vw + c * d.W;
        float ss = 0.f;
#pragma unroll 4
        for (int j = 0; j < W; ++j) {
            const float fv = (j >= jlo_f && j < jhi_f) ? __ldg(fr + j) : 0.f;
            const float tv = (j >= jlo_t && j < jhi_t) ? __ldg(tr + j) : 0.f;
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
constexpr int kRowCap = 8192;   // per-row upper bounds kept in shared memory
constexpr int kCandCap = 2048;  // exact-scoring candidates per window pass

struct ScreenShared {
    float lb;
    float nv;
    unsigned long long best;
    uint32_t nA;
    uint32_t nTB;
};

// Screening of one flagged window per CTA.  Items are enumerated as rows:
// part 1 = (a in A+, t) rows over all b; part 2 = ((t, b) with L_t > 0) rows
// over the a not in A+.  A warp handles a row, lanes the varying shift.
// Pass 1 gives the lower bound LB = max(est - bound) and per-row maxima of
// est + bound; pass 2 revisits only rows that can reach max(LB, seed) and
// scores their candidates exactly.
__global__ void __launch_bounds__(kScrThreads) screen_kernel(
    Dims d, const float* __restrict__ V, const float* __restrict__ T, const float* __restrict__ L,
    const float* __restrict__ theta, const float2* __restrict__ Etab, const float* __restrict__ XT,
    const float* __restrict__ G, uint32_t k0, uint32_t kcount, const uint32_t* __restrict__ flag,
    DevStatus* status, const uint32_t* __restrict__ best_lab, const uint32_t* __restrict__ best_idx,
    const float* __restrict__ best_lik, unsigned long long* keys, const float* __restrict__ mx)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ ScreenShared sh;
    typedef cub::BlockReduce<float, kScrThreads> RF;
    typedef cub::BlockScan<uint32_t, kScrThreads> SC;
    __shared__ union {
        typename RF::TempStorage rf;
        typename SC::TempStorage sc;
    } tmp;
    const uint32_t S = d.S, W = d.W, M = d.M, S2 = 2 * S + 1;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = kScrThreads / 32;
    uint8_t* fa = smraw;                                            // [S2] bit0 in bounds, bit1 L_f > 0
    uint8_t* pt = fa + ((S2 + 15) & ~15u);                          // [M][S2] L_t > 0
    uint32_t* alist = reinterpret_cast<uint32_t*>(pt + ((M * S2 + 15) & ~15u));  // [S2]
    uint32_t* tb = alist + S2;                                      // [M*S2] (t,b) with L_t > 0
    float* rowmax = reinterpret_cast<float*>(tb + M * S2);          // [kRowCap]
    float* vw = rowmax + kRowCap;                                   // [C][W] window voltage
    float* gmax = vw + d.C * W;                                     // [M] max_b G_t(b) of this window
    uint32_t* cand = reinterpret_cast<uint32_t*>(gmax + M);         // [kCandCap][3] (a, t, b)
    __shared__ uint32_t s_ncand;
    const uint64_t items = (uint64_t)S2 * S2 * M;
    const uint64_t nloc = (items - 1) / d.WG + 1;
    const uint64_t slots = nloc * d.WG;
    uint32_t lbits = 0;
    while ((1u << lbits) < d.WG) ++lbits;
    const float u = 1.0f / 16777216.0f;
    const float K = 1.01f * 1.05f * u * 2.0f * ((float)d.C * W + d.C + W + 8);
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
        float nv2 = 0.f;
        for (uint32_t e = threadIdx.x; e < d.C * W; e += blockDim.x) {
            const uint32_t c = e / W, j = e - c * W;
            const float v = V[(uint64_t)c * d.N + p + j];
            vw[e] = v;
            nv2 = fmaf(v, v, nv2);
        }
        const float nvs = RF(tmp.rf).Sum(nv2);
        if (threadIdx.x == 0) { sh.nv = sqrtf(nvs) * 1.001f; sh.best = 0ull; }
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
        // per-template maxima of the partial correlations over the shifts in bounds
        for (uint32_t t = warp; t < M; t += nwarps) {
            float m = -INFINITY;
            for (uint32_t x = lane; x < S2; x += 32) {
                const uint64_t xp = (uint64_t)x + p;
                if (xp >= S && xp < (uint64_t)d.N - W + S) m = fmaxf(m, Gk[(uint64_t)t * S2 + x]);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
            if (lane == 0) gmax[t] = m;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t n = 0;
            for (uint32_t x = 0; x < S2; ++x) if (fa[x] == 3) alist[n++] = x;
            sh.nA = n;
        }
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
        const float nv = sh.nv;
        const uint32_t rows1 = nA * M, rows = rows1 + nTB;
        const bool keep_rows = rows <= (uint32_t)kRowCap;
        auto score = [&](uint32_t a, uint32_t t, uint32_t b, unsigned long long& kb) {
            const float v = pair_exact_sv(d, T, vw, f, t, a, b);
            ++exact_n;
            if (!(v > 0.f)) return;
            const uint64_t r = (uint64_t)t + (uint64_t)M * a + (uint64_t)M * S2 * b;
            uint32_t pr = item_priority(r, d.WG, lbits);
            for (uint64_t rr = r + items; rr < slots; rr += items) {
                const uint32_t p2 = item_priority(rr, d.WG, lbits);
                pr = p2 < pr ? p2 : pr;
            }
            const unsigned long long key =
                ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xFFFFFFFFu - pr);
            kb = key > kb ? key : kb;
        };
        // one row: (a fixed, t, lanes over b) or (t, b fixed, lanes over a)
        auto row_scan = [&](uint32_t row, float thr, bool exact_pass, float& lbm, float& ubm,
                            unsigned long long& kb) {
            uint32_t a = 0, t, b = 0;
            bool fixed_a;
            if (row < rows1) {
                a = alist[row / M];
                t = row % M;
                fixed_a = true;
            } else {
                const uint32_t e = tb[row - rows1];
                t = e / S2;
                b = e - t * S2;
                fixed_a = false;
            }
            const float* xt_ft = XT + ((uint64_t)f * M + t) * S2 * S2;
            if (!exact_pass) {
                // row bound: every component at least the item's, same float order
                const float nx = mx[(uint64_t)f * M + t];
                float ub;
                if (fixed_a) {
                    const float2 ea = Etab[(uint64_t)f * S2 + a];
                    ub = Gk[(uint64_t)f * S2 + a] + gmax[t] + nx +
                         K * ((ea.y + mx[M * M + t]) * nv + ea.x + mx[M * M + M + t]);
                } else {
                    const float2 eb = Etab[(uint64_t)t * S2 + b];
                    ub = gmax[f] + Gk[(uint64_t)t * S2 + b] + nx +
                         K * ((mx[M * M + f] + eb.y) * nv + mx[M * M + M + f] + eb.x);
                }
                if (ub < thr) { ubm = -INFINITY; return; }
            }
            for (uint32_t x = lane; x < S2; x += 32) {
                if (fixed_a) {
                    b = x;
                    if (!(fa[b] & 1)) continue;
                } else {
                    a = x;
                    if (fa[a] != 1) continue;
                }
                if ((a > b ? a - b : b - a) > W) continue;
                const float2 ea = Etab[(uint64_t)f * S2 + a], eb = Etab[(uint64_t)t * S2 + b];
                const float est = Gk[(uint64_t)f * S2 + a] + Gk[(uint64_t)t * S2 + b] - xt_ft[(uint64_t)a * S2 + b];
                const float bound = K * ((ea.y + eb.y) * nv + ea.x + eb.x);
                if (!exact_pass) {
                    lbm = fmaxf(lbm, est - bound);
                    ubm = fmaxf(ubm, est + bound);
                    ++item_n;
                    continue;
                }
                if (est + bound < thr) continue;
                const uint32_t slot = atomicAdd(&s_ncand, 1u);
                if (slot < (uint32_t)kCandCap) {
                    cand[3 * slot] = a;
                    cand[3 * slot + 1] = t;
                    cand[3 * slot + 2] = b;
                } else {
                    score(a, t, b, kb);   // list full: score in place
                }
            }
        };
        float lb = -INFINITY;
        unsigned long long kbest = 0ull;
        const float thr0 = fmaxf(seed, 0.f);
        for (uint32_t row = warp; row < rows; row += nwarps) {
            float lbm = -INFINITY, ubm = -INFINITY;
            row_scan(row, thr0, false, lbm, ubm, kbest);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) ubm = fmaxf(ubm, __shfl_xor_sync(0xffffffffu, ubm, off));
            if (keep_rows && lane == 0) rowmax[row] = ubm;
            lb = fmaxf(lb, lbm);
        }
        const float lbs = RF(tmp.rf).Reduce(lb, cub::Max());
        if (threadIdx.x == 0) { sh.lb = lbs; s_ncand = 0; }
        __syncthreads();
        const float thr = fmaxf(fmaxf(sh.lb, seed), 0.f);
        for (uint32_t row = warp; row < rows; row += nwarps) {
            if (keep_rows && rowmax[row] < thr) continue;
            float lbm, ubm;
            row_scan(row, thr, true, lbm, ubm, kbest);
        }
        __syncthreads();
        const uint32_t nc = min(s_ncand, (uint32_t)kCandCap);
        for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) score(cand[3 * i], cand[3 * i + 1], cand[3 * i + 2], kbest);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_down_sync(0xffffffffu, kbest, off);
            kbest = o > kbest ? o : kbest;
        }
        if (lane == 0 && kbest) atomicMax(&sh.best, kbest);
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
    energy_table_kernel<<<(d.M * S2 + 255) / 256, 256, 0, st>>>(d, T, w.at<float2>(L.off_et));
    const size_t smem = (size_t)2 * d.C * d.W * 4 + 8 + (size_t)kLagChunk * (d.W + 1) * 8;
    if (smem > 200 * 1024) return fail(FBP_E_ARG, "template too large for the pair table kernel");
    FBP_CUDA(cudaFuncSetAttribute(cross_table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cross_table_kernel<<<d.M * d.M, 256, smem, st>>>(d, T, w.at<float>(L.off_xt), w.at<float>(L.off_mx));
    energy_max_kernel<<<(d.M + 127) / 128, 128, 0, st>>>(d, w.at<float2>(L.off_et), w.at<float>(L.off_mx) + (size_t)d.M * d.M);
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
                          (size_t)d.M * S2 * 4 + (size_t)kRowCap * 4 + (size_t)d.C * d.W * 4 + (size_t)d.M * 4 +
                          (size_t)kCandCap * 12;
    if (smem_b > 200 * 1024) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    FBP_CUDA(cudaFuncSetAttribute(screen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
    const uint32_t threads_a = (S2 + 31) & ~31u;
    const uint32_t groups = (d.M + Q - 1) / Q;
    float* G = w.at<float>(L.off_g);
    const float2* Et = w.at<float2>(L.off_et);
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
                                                       w.best_lab(), w.best_idx(), w.best_lik(), w.keys(),
                                                       w.at<float>(L.off_mx));
        FBP_CUDA(cudaGetLastError());
    }
    return FBP_OK;
}

}  // namespace fbp
