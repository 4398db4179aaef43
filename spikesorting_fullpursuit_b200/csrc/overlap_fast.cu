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

#include <vector>

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

// Pair cross terms X_ft(a, b) for |a-b| <= W, one CTA per (f, t), stored as
// XT[f][t][a][b] and transposed as XTT[f][t][b][a]: products
// P_delta[u] = sum_c F[c,u] T[c,u+delta] in double, prefix sums over u, then
// X_ft(a, b) = Q_delta[hi] - Q_delta[lo] with delta = a-b.
constexpr int kLagChunk = 16;

__global__ void __launch_bounds__(256) cross_table_kernel(Dims d, const float* __restrict__ T, float* XT, float* XTT,
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
            XTT[(((uint64_t)f * d.M + t) * S2 + b) * S2 + a] = xv;
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
__global__ void template_order_kernel(Dims d, const float* __restrict__ T, uint32_t* perm,
                                      unsigned long long* chmask)
{
    extern __shared__ uint32_t key[];
    for (uint32_t t = threadIdx.x; t < d.M; t += blockDim.x) {
        uint32_t first = d.C;
        unsigned long long m = 0ull;
        for (uint32_t c = 0; c < d.C; ++c) {
            bool nz = false;
            for (uint32_t j = 0; j < d.W && !nz; ++j) nz = T[((uint64_t)t * d.C + c) * d.W + j] != 0.f;
            if (nz) {
                if (first == d.C) first = c;
                m |= c < 64 ? (1ull << c) : 0ull;
            }
        }
        key[t] = first;
        chmask[t] = d.C <= 64 ? m : ~0ull;   // more than 64 channels: no skipping
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
// with each flagged window (masked to [p, p+W)).  A CTA owns one group of Q
// templates (in perm order; only the group's union of non-zero channels is
// staged) and walks over the windows kPcWin at a time.  Lane = (window, shift
// sub-block): a warp covers 16 consecutive shifts of 8 windows, so the taps
// that can meet the window's W live samples form one range per warp (the
// zero triangle of the masked correlation is skipped), and each lane computes
// 4 consecutive shifts for the Q templates from aligned 16-byte strip loads.
// The strips keep their zero margins from one clearing; each window writes
// only its W live samples per channel (cp.async).  The sums are estimates:
// any order, FMA allowed.
constexpr int kPcR = 4;       // shifts per lane
constexpr int kPcWin = 8;     // windows per CTA iteration (lane bits 2..4)
constexpr int kPcPad = 20;    // zero margin around the live samples in a staged strip
constexpr int kPcMaxWarps = 12;   // two CTAs of 12 warps fit an SM at <= 80 registers

struct PcGeom {
    uint32_t Wp, Z, SLc, WS;  // padded taps; strip index of window sample 0; strip length; window stride
    int o;                    // shift b reads strip index b - o + j  (o = S - Z, a multiple of 4)
};

__host__ __device__ inline PcGeom pc_geom(const Dims& d, uint32_t Cu)
{
    PcGeom g;
    g.Wp = (d.W + 3) & ~3u;
    g.Z = kPcPad + (d.S & 3u);
    g.o = (int)d.S - (int)g.Z;
    g.SLc = (g.Z + d.W + kPcPad + 3) & ~3u;
    uint32_t ws = Cu * g.SLc;
    ws += (16u - ws % 32u + 32u) % 32u;   // windows 16 banks apart: a quarter-warp's two windows do not collide
    g.WS = ws;
    return g;
}

__host__ __device__ inline size_t pc_smem_bytes(const Dims& d, uint32_t Cu, int Q)
{
    const PcGeom g = pc_geom(d, Cu);
    return ((size_t)Q * Cu * g.Wp + (size_t)kPcWin * g.WS) * 4;
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src)
{
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src) : "memory");
}

template <int Q>
__global__ void __launch_bounds__(kPcMaxWarps * 32, 2) partial_corr_kernel(
    Dims d, const float* __restrict__ V, const float* __restrict__ T, const float* __restrict__ L,
    const float* __restrict__ theta, const float2* __restrict__ Et, const uint32_t* __restrict__ perm,
    const unsigned long long* __restrict__ chmask, const uint32_t* __restrict__ flag, const DevStatus* status,
    const uint32_t* __restrict__ best_lab, const uint32_t* __restrict__ best_idx, uint32_t k0, uint32_t kc,
    float* G)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ uint32_t chans[256];
    __shared__ uint32_t s_nch;
    __shared__ uint32_t s_p[kPcWin];
    __shared__ int s_ok[kPcWin];
    const uint32_t S2 = 2 * d.S + 1, W = d.W, M = d.M;
    const uint32_t g0 = blockIdx.y * Q;
    if (threadIdx.x == 0) {
        unsigned long long m = 0ull;
        for (uint32_t q = 0; q < Q; ++q)
            if (g0 + q < M) m |= chmask[perm[g0 + q]];
        uint32_t n = 0;
        for (uint32_t c = 0; c < d.C; ++c)
            if (c >= 64 || ((m >> c) & 1ull)) chans[n++] = c;
        s_nch = n;
    }
    __syncthreads();
    const uint32_t Cu = s_nch;
    const PcGeom gm = pc_geom(d, Cu);
    const uint32_t Wp = gm.Wp;
    float* Ts = sm;                                   // [Q][Cu][Wp]
    float* Vs = sm + (size_t)Q * Cu * Wp;              // [kPcWin][WS], row ci at ci * SLc
    for (uint32_t e = threadIdx.x; e < Q * Cu * Wp; e += blockDim.x) {
        const uint32_t q = e / (Cu * Wp), r = e - q * Cu * Wp, ci = r / Wp, j = r - ci * Wp;
        Ts[e] = (g0 + q < M && j < W) ? T[((uint64_t)perm[g0 + q] * d.C + chans[ci]) * W + j] : 0.f;
    }
    for (uint32_t e = threadIdx.x; e < kPcWin * gm.WS; e += blockDim.x) Vs[e] = 0.f;
    const uint32_t nflag = status->n_flag;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t wi = lane >> 2, bs = lane & 3;
    unsigned long long macs = 0;   // multiply-adds this thread does
    for (uint32_t base = blockIdx.x * kPcWin; base < kc; base += gridDim.x * kPcWin) {
        __syncthreads();
        if (threadIdx.x < kPcWin) {
            const uint32_t kk = base + threadIdx.x;
            int ok = 0;
            uint32_t p = 0;
            if (kk < kc && k0 + kk < nflag) {
                const uint32_t id = flag[k0 + kk];
                const uint32_t f = best_lab[id];
                p = best_idx[id];
                ok = !window_skipped(d, L, theta, f, p);
            }
            s_ok[threadIdx.x] = ok;
            s_p[threadIdx.x] = p;
        }
        __syncthreads();
        for (uint32_t r = warp; r < kPcWin * Cu; r += nwarps) {
            const uint32_t w = r / Cu, ci = r - w * Cu;
            if (!s_ok[w]) continue;
            const float* src = V + (uint64_t)chans[ci] * d.N + s_p[w];
            float* dst = Vs + (size_t)w * gm.WS + (size_t)ci * gm.SLc + gm.Z;
            for (uint32_t j = lane; j < W; j += 32) cp_async4(dst + j, src + j);
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        if (!s_ok[wi]) continue;
        float* Gk = G + (uint64_t)(base + wi) * M * S2;
        const float* vw = Vs + (size_t)wi * gm.WS;
        for (uint32_t bw = warp * 16; bw < S2; bw += nwarps * 16) {
            const uint32_t b0 = bw + kPcR * bs;
            int jlo = (int)d.S - (int)bw - 15;
            jlo = jlo < 0 ? 0 : (jlo & ~3);
            int jhi = ((int)(d.S + W) - (int)bw + 3) & ~3;
            jhi = jhi > (int)Wp ? (int)Wp : jhi;
            float acc[Q][kPcR];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < kPcR; ++r) acc[q][r] = 0.f;
            const int vb = (int)b0 - gm.o;
            if (jhi > jlo) macs += (unsigned long long)Q * kPcR * (uint32_t)(jhi - jlo) * Cu;
            for (uint32_t ci = 0; ci < Cu; ++ci) {
                const float* vr = vw + (size_t)ci * gm.SLc;
                const float* tr = Ts + (size_t)ci * Wp;
                for (int j0 = jlo; j0 < jhi; j0 += 4) {
                    const float4 va = *reinterpret_cast<const float4*>(vr + vb + j0);
                    const float4 vc = *reinterpret_cast<const float4*>(vr + vb + j0 + 4);
                    const float v[8] = {va.x, va.y, va.z, va.w, vc.x, vc.y, vc.z, vc.w};
#pragma unroll
                    for (int q = 0; q < Q; ++q) {
                        const float4 t4 = *reinterpret_cast<const float4*>(tr + (size_t)q * Cu * Wp + j0);
#pragma unroll
                        for (int r = 0; r < kPcR; ++r) {
                            float a = acc[q][r];
                            a = fmaf(t4.x, v[r], a);
                            a = fmaf(t4.y, v[r + 1], a);
                            a = fmaf(t4.z, v[r + 2], a);
                            a = fmaf(t4.w, v[r + 3], a);
                            acc[q][r] = a;
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                if (g0 + q >= M) continue;
                const uint32_t t = perm[g0 + q];
#pragma unroll
                for (int r = 0; r < kPcR; ++r) {
                    const uint32_t bb = b0 + r;
                    if (bb < S2) Gk[(uint64_t)t * S2 + bb] = acc[q][r] - 0.5f * Et[(uint64_t)t * S2 + bb].x;
                }
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) macs += __shfl_xor_sync(0xffffffffu, macs, off);
    if (lane == 0 && macs) atomicAdd(&const_cast<DevStatus*>(status)->pc_macs, macs);
}

// Exact pair likelihood in the reference's float order (binary_pursuit.cl:578-632),
// operands read from memory.
// Channels on which both templates are entirely zero are skipped: there the
// reference adds 0 * v and 0 * 0 terms, which leave its sums unchanged (acc
// starts at +0, so no step of the reference makes it -0 either).
__device__ float pair_exact_g(const Dims& d, const float* __restrict__ T, const float* __restrict__ V, uint32_t f,
                              uint32_t t, uint32_t p, uint32_t a, uint32_t b, unsigned long long chans)
{
    const int W = (int)d.W, fa = (int)d.S - (int)a, ta = (int)d.S - (int)b;
    const int jlo_f = max(0, -fa), jhi_f = min(W, W - fa), jlo_t = max(0, -ta), jhi_t = min(W, W - ta);
    float acc = 0.f;
    for (uint32_t c = 0; c < d.C; ++c) {
        if (c < 64 && !((chans >> c) & 1ull)) continue;
        const float* fr = T + ((uint64_t)f * d.C + c) * d.W + fa;
        const float* tr = T + ((uint64_t)t * d.C + c) * d.W + ta;
        const float* vr = V + (uint64_t)c * d.N + p;
        float ss = 0.f;
#pragma unroll 8
        for (int j = 0; j < W; ++j) {
            const float fv = (j >= jlo_f && j < jhi_f) ? __ldg(fr + j) : 0.f;
            const float tv = (j >= jlo_t && j < jhi_t) ? __ldg(tr + j) : 0.f;
            const float sv = fadd(fv, tv);
            ss = fadd(ss, fmul(sv, sv));
            acc = fadd(acc, fmul(sv, __ldg(vr + j)));
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

constexpr int kScrThreads = 384;
constexpr int kRowCap = 2048;   // surviving rows kept in shared memory
constexpr int kCandCap = 256;   // candidates buffered in shared memory per window (more go straight to the global list)
constexpr int kScanQ = 8;       // items per lane of a row chunk (32 * kScanQ shifts)
constexpr uint32_t kBStage = 96 * 1024;   // per-window item tables staged in shared memory up to this size
constexpr uint32_t kScreenGrid = 148 * 2;  // persistent CTAs (two per SM); also sizes the unstaged table scratch

struct ScreenShared {
    float lb;
    float maxau2;
    unsigned long long best;
    uint32_t nA;
    uint32_t nrows;
    uint32_t ncand;
    uint32_t gfull;   // the global candidate list ran out of room for this window
};

// Shared-memory bytes of screen_kernel for these sizes (tables staged or not).
__host__ __device__ inline size_t screen_smem_bytes(uint32_t M, uint32_t S2, bool staged)
{
    const size_t s2p = (S2 + 3) & ~3u, mp = (M + 3) & ~3u;
    size_t b = 5 * s2p * 4 + 3 * mp * 4 + 256 * 4 + (size_t)kRowCap * 8 + (size_t)kCandCap * 12;
    b += (((size_t)S2 + 15) & ~(size_t)15) + (((size_t)M * S2 + 15) & ~(size_t)15);
    if (staged) b += (size_t)M * S2 * 8;
    return b + 64;
}

// One row of items seen from the lanes of a warp: the row's fixed part (uf,
// lf), the per-item parts (ua[x], la[x]) and the cross terms xr[x] for x in
// [lo, hi).  Item bounds: UB = (uf + ua[x]) - X, LB = (lf + la[x]) - X.
struct ScreenRow {
    float uf, lf;
    const float* ua;
    const float* la;
    const float* xr;   // null: the templates share no channel, X == 0
    int lo, hi;
    uint32_t t, y;
    bool fixed_a;
};

// Screening of one flagged window per CTA.
//   rows, kind 1: (a in A+, t) -- a fixed, the lanes run over b (cross table XT[f][t][a][:]);
//   rows, kind 2: (t, b) with L_t(b) > 0 -- b fixed, the lanes run over a not in A+
//                 (transposed cross table XTT[f][t][b][:]).
// Per window the CTA stages Bu/Bl[t][b] = G_t(b) +- beta_t(b) and Au/Al[a] =
// G_f(a) +- alpha(a), with alpha + beta = K (sqrt E_f(a) |v|_f + sqrt E_t(b) |v|_t +
// E_f(a) + E_t(b)) the rigorous bound of |estimate - reference float value|
// (|v|_x: the window's norm over template x's non-zero channels)
// (K carries slack for the few float operations of this regrouping).  Phase B
// bounds every row from shared-memory maxima (each component at least the
// item's, same monotone float order) and keeps the rows that can reach the
// window's seed; a quick lower bound from the best row of each warp prunes
// them further.  Phase C scans the kept rows two at a time per warp (all
// loads of both rows in flight together): LB = max(LB items) and per-row
// maxima of UB.  Phase D lists the items of rows reaching max(LB, seed, 0)
// whose UB does; score_kernel scores them exactly.
__global__ void __launch_bounds__(kScrThreads, 2) screen_kernel(
    Dims d, const float* __restrict__ V, const float* __restrict__ T, const float* __restrict__ L,
    const float* __restrict__ theta, const float2* __restrict__ Etab, const float* __restrict__ XT,
    const float* __restrict__ XTT, const float* __restrict__ G, uint32_t k0, uint32_t kcount,
    const uint32_t* __restrict__ flag, DevStatus* status, const uint32_t* __restrict__ best_lab,
    const uint32_t* __restrict__ best_idx, const float* __restrict__ best_lik, unsigned long long* keys,
    const float* __restrict__ mx, unsigned long long* gcand, uint32_t gcand_cap,
    const unsigned long long* __restrict__ chmask, float* bscratch, const uint32_t* __restrict__ order)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ ScreenShared sh;
    __shared__ uint32_t s_gbase;
    typedef cub::BlockReduce<float, kScrThreads> RF;
    typedef cub::BlockScan<uint32_t, kScrThreads> SC;
    __shared__ union {
        typename RF::TempStorage rf;
        typename SC::TempStorage sc;
    } tmp;
    const uint32_t S = d.S, W = d.W, M = d.M, S2 = 2 * S + 1;
    const uint32_t s2p = (S2 + 3) & ~3u, mp = (M + 3) & ~3u;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = kScrThreads / 32;
    const bool staged = (uint64_t)M * S2 * 8 <= kBStage;
    // shared layout
    float* Au = reinterpret_cast<float*>(smraw);   // [S2] G_f(a) + alpha(a), a in bounds
    float* Al = Au + s2p;                          // [S2] G_f(a) - alpha(a)
    float* Au2 = Al + s2p;                         // [S2] as Au for a in bounds and not in A+, else -inf
    float* Al2 = Au2 + s2p;
    uint32_t* alist = reinterpret_cast<uint32_t*>(Al2 + s2p);   // [S2] A+ in ascending order
    float* gmaxu = reinterpret_cast<float*>(alist + s2p);       // [M] max_b Bu[t][b]
    float* nx = gmaxu + mp;                                     // [M] max -X_ft over items
    float* nvt = nx + mp;                                       // [M] window norm over template t's channels
    float* vc2 = nvt + mp;                                      // [C <= 256] window energy per channel
    float* rowmax = vc2 + 256;                                  // [kRowCap]
    uint32_t* rows = reinterpret_cast<uint32_t*>(rowmax + kRowCap);   // [kRowCap]
    uint32_t* cand = rows + kRowCap;                            // [kCandCap][3]
    uint8_t* fa = reinterpret_cast<uint8_t*>(cand + 3 * kCandCap);   // [S2] bit0 in bounds, bit1 L_f > 0
    uint8_t* pt = fa + ((S2 + 15) & ~15u);                      // [M][S2] L_t(b) > 0, b in bounds
    float* Bu = staged ? reinterpret_cast<float*>(pt + ((M * S2 + 15) & ~15u))
                       : bscratch + (uint64_t)blockIdx.x * M * S2 * 2;   // [M][S2]
    float* Bl = Bu + (size_t)M * S2;                                        // [M][S2]
    const uint64_t items = (uint64_t)S2 * S2 * M;
    const uint64_t nloc = (items - 1) / d.WG + 1;
    const uint64_t slots = nloc * d.WG;
    uint32_t lbits = 0;
    while ((1u << lbits) < d.WG) ++lbits;
    const float u = 1.0f / 16777216.0f;
    const float K = 1.01f * 1.05f * u * 2.0f * ((float)d.C * W + d.C + W + 24);
    const uint32_t nflag = status->n_flag;
    unsigned long long exact_n = 0, item_n = 0;
    for (uint32_t jo = blockIdx.x; jo < kcount; jo += gridDim.x) {
        const uint32_t kk = order[jo];
        const uint32_t k = k0 + kk;
        if (k >= nflag) continue;
        const uint32_t id = flag[k];
        const uint32_t f = best_lab[id], p = best_idx[id];
        if (window_skipped(d, L, theta, f, p)) continue;
        const float seed = best_lik[id];
        const float thr0 = fmaxf(seed, 0.f);
        const float* Gk = G + (uint64_t)kk * M * S2;
        const unsigned long long mf = chmask[f];
        __syncthreads();
        // ---- phase A: window quantities.  The window's energy per channel gives,
        // per template, the norm of the window over that template's channels: a
        // template's products touch no other channel, so its part of the bound
        // (Cauchy-Schwarz over its support) needs no more
        for (uint32_t c = warp; c < d.C; c += nwarps) {
            float e2 = 0.f;
            for (uint32_t j = lane; j < W; j += 32) {
                const float v = V[(uint64_t)c * d.N + p + j];
                e2 = fmaf(v, v, e2);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, off);
            if (lane == 0) vc2[c] = e2;
        }
        for (uint32_t x = threadIdx.x; x < S2; x += blockDim.x) {
            const uint64_t xp = (uint64_t)x + p;
            const bool inb = xp >= S && xp < (uint64_t)d.N - W + S;
            fa[x] = inb ? ((L[(uint64_t)f * d.N + xp - S] > 0.f) ? 3 : 1) : 0;
        }
        for (uint32_t t = threadIdx.x; t < M; t += blockDim.x) nx[t] = mx[(uint64_t)f * M + t];
        if (threadIdx.x == 0) {
            sh.best = 0ull;
            sh.nrows = 0;
            sh.ncand = 0;
            sh.gfull = 0;
        }
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < M; t += blockDim.x) {
            const unsigned long long mt = chmask[t];   // all ones above 64 channels
            float e2 = 0.f;
            for (uint32_t c = 0; c < d.C; ++c)
                if (c >= 64 || ((mt >> c) & 1ull)) e2 += vc2[c];
            nvt[t] = sqrtf(e2) * 1.001f;
        }
        __syncthreads();
        const float nvf = nvt[f];
        float ma2 = -INFINITY;
        for (uint32_t x = threadIdx.x; x < S2; x += blockDim.x) {
            const float2 ea = Etab[(uint64_t)f * S2 + x];
            const float al = K * fmaf(nvf, ea.y, ea.x);
            const float g = Gk[(uint64_t)f * S2 + x];
            const uint8_t fl = fa[x];
            const float au = (fl & 1) ? g + al : -INFINITY, alo = (fl & 1) ? g - al : -INFINITY;
            Au[x] = au;
            Al[x] = alo;
            Au2[x] = fl == 1 ? au : -INFINITY;
            Al2[x] = fl == 1 ? alo : -INFINITY;
            if (fl == 1) ma2 = fmaxf(ma2, au);
        }
#pragma unroll 4
        for (uint32_t e = threadIdx.x; e < M * S2; e += blockDim.x) {
            const uint32_t t = e / S2, x = e - t * S2;
            const uint64_t xp = (uint64_t)x + p;
            const bool inb = xp >= S && xp < (uint64_t)d.N - W + S;
            const float2 eb = Etab[e];
            const float be = K * fmaf(nvt[t], eb.y, eb.x);
            const float g = Gk[e];
            Bu[e] = inb ? g + be : -INFINITY;
            Bl[e] = inb ? g - be : -INFINITY;
            pt[e] = (inb && L[(uint64_t)t * d.N + xp - S] > 0.f) ? 1 : 0;
        }
        {
            const float m2 = RF(tmp.rf).Reduce(ma2, cub::Max());
            if (threadIdx.x == 0) sh.maxau2 = m2;
        }
        __syncthreads();   // Bu/Bl (global scratch too: the block's own writes) visible
        for (uint32_t t = warp; t < M; t += nwarps) {
            float m = -INFINITY;
            for (uint32_t x = lane; x < S2; x += 32) m = fmaxf(m, Bu[(uint64_t)t * S2 + x]);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
            if (lane == 0) gmaxu[t] = m;
        }
        // A+ list in ascending order
        {
            uint32_t base = 0;
            for (uint32_t x0 = 0; x0 < S2; x0 += blockDim.x) {
                const uint32_t x = x0 + threadIdx.x;
                const uint32_t fl = (x < S2 && fa[x] == 3) ? 1u : 0u;
                uint32_t off, tot;
                SC(tmp.sc).ExclusiveSum(fl, off, tot);
                if (fl) alist[base + off] = x;
                base += tot;
                __syncthreads();
            }
            if (threadIdx.x == 0) sh.nA = base;
        }
        __syncthreads();
        const uint32_t nA = sh.nA;
        const float maxau2 = sh.maxau2;
        const uint32_t rows1 = nA * M, rows_all = rows1 + M * S2;
        // row r -> bound of every item in it (phase B), and its scan description
        auto row_bound = [&](uint32_t r) -> float {
            if (r < rows1) {
                const uint32_t t = r % M;
                return (Au[alist[r / M]] + gmaxu[t]) + nx[t];
            }
            const uint32_t e = r - rows1;
            if (!pt[e]) return -INFINITY;
            return (Bu[e] + maxau2) + nx[e / S2];
        };
        auto describe = [&](uint32_t r, ScreenRow& R) {
            if (r < rows1) {
                const uint32_t a = alist[r / M], t = r % M;
                R.fixed_a = true;
                R.t = t;
                R.y = a;
                R.uf = Au[a];
                R.lf = Al[a];
                R.ua = Bu + (size_t)t * S2;
                R.la = Bl + (size_t)t * S2;
                R.xr = (mf & chmask[t]) ? XT + (((uint64_t)f * M + t) * S2 + a) * S2 : nullptr;
            } else {
                const uint32_t e = r - rows1, t = e / S2, b = e - t * S2;
                R.fixed_a = false;
                R.t = t;
                R.y = b;
                R.uf = Bu[e];
                R.lf = Bl[e];
                R.ua = Au2;
                R.la = Al2;
                R.xr = (mf & chmask[t]) ? XTT + (((uint64_t)f * M + t) * S2 + b) * S2 : nullptr;
            }
            R.lo = max(0, (int)R.y - (int)W);
            R.hi = min((int)S2, (int)R.y + (int)W + 1);
        };
        // scan of up to two rows by one warp: cross terms of both rows loaded
        // together, then (listing == false) LB/UB maxima, or (listing) candidates
        auto scan2 = [&](const ScreenRow (&R)[2], bool listing, float thr, float (&lbm)[2], float (&ubm)[2]) {
            const int span = max(R[0].hi - R[0].lo, R[1].hi - R[1].lo);
            for (int c0 = 0; c0 < span; c0 += 32 * kScanQ) {
                float xv[2][kScanQ];
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int q = 0; q < kScanQ; ++q) {
                        const int x = R[i].lo + c0 + (int)lane + 32 * q;
                        xv[i][q] = (x < R[i].hi && R[i].xr) ? __ldg(R[i].xr + x) : 0.f;
                    }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
#pragma unroll
                    for (int q = 0; q < kScanQ; ++q) {
                        const int x = R[i].lo + c0 + (int)lane + 32 * q;
                        if (x >= R[i].hi) continue;
                        const float ub = (R[i].uf + R[i].ua[x]) - xv[i][q];
                        if (!listing) {
                            const float lb = (R[i].lf + R[i].la[x]) - xv[i][q];
                            lbm[i] = fmaxf(lbm[i], lb);
                            ubm[i] = fmaxf(ubm[i], ub);
                            continue;
                        }
                        if (!(ub >= thr)) continue;
                        const uint32_t a = R[i].fixed_a ? R[i].y : (uint32_t)x;
                        const uint32_t b = R[i].fixed_a ? (uint32_t)x : R[i].y;
                        const uint32_t slot = atomicAdd(&sh.ncand, 1u);
                        if (slot < (uint32_t)kCandCap) {
                            cand[3 * slot] = a;
                            cand[3 * slot + 1] = R[i].t;
                            cand[3 * slot + 2] = b;
                        } else {
                            const uint32_t g = atomicAdd(&status->cand_count, 1u);
                            if (g < gcand_cap)
                                gcand[g] = ((unsigned long long)kk << 32) | ((unsigned long long)R[i].t << 20) |
                                           ((unsigned long long)a << 10) | (unsigned long long)b;
                            else
                                sh.gfull = 1;
                        }
                    }
                }
            }
        };
        // ---- phase B: row bounds, keep rows that can reach the seed
        for (uint32_t r = threadIdx.x; r < rows_all; r += blockDim.x) {
            const float ub = row_bound(r);
            if (!(ub >= thr0)) continue;
            const uint32_t slot = atomicAdd(&sh.nrows, 1u);
            if (slot < (uint32_t)kRowCap) { rows[slot] = r; rowmax[slot] = ub; }
        }
        __syncthreads();
        uint32_t nrows = sh.nrows;
        const bool overflow = nrows > (uint32_t)kRowCap;
        if (overflow) nrows = rows_all;
        // ---- phase B2: a quick lower bound from the highest-bound row of each
        // warp's share, then keep only rows whose bound reaches it
        float lb = -INFINITY;
        if (!overflow && nrows > 0) {
            float bu = -INFINITY;
            uint32_t bi = 0xFFFFFFFFu;
            for (uint32_t i = warp + nwarps * lane; i < nrows; i += nwarps * 32)
                if (rowmax[i] > bu) { bu = rowmax[i]; bi = i; }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float ou = __shfl_xor_sync(0xffffffffu, bu, off);
                const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, off);
                if (ou > bu || (ou == bu && oi < bi)) { bu = ou; bi = oi; }
            }
            if (bi != 0xFFFFFFFFu) {
                ScreenRow R[2];
                describe(rows[bi], R[0]);
                R[1].lo = R[1].hi = 0;
                float lbm[2] = {-INFINITY, -INFINITY}, ubm[2] = {-INFINITY, -INFINITY};
                scan2(R, false, 0.f, lbm, ubm);
                lb = lbm[0];
            }
        }
        {
            const float lb1 = RF(tmp.rf).Reduce(lb, cub::Max());
            if (threadIdx.x == 0) sh.lb = lb1;
            __syncthreads();
            const float thr1 = fmaxf(sh.lb, thr0);
            if (!overflow) {
                // compact the rows reaching thr1 (order kept), reusing the row arrays in place
                uint32_t base = 0;
                for (uint32_t i0 = 0; i0 < nrows; i0 += blockDim.x) {
                    const uint32_t i = i0 + threadIdx.x;
                    const bool keep = i < nrows && rowmax[i] >= thr1;
                    const uint32_t r = keep ? rows[i] : 0u;
                    uint32_t off, tot;
                    SC(tmp.sc).ExclusiveSum(keep ? 1u : 0u, off, tot);
                    __syncthreads();
                    if (keep) rows[base + off] = r;
                    base += tot;
                    __syncthreads();
                }
                nrows = base;
            }
        }
        // a kept row (or, after an overflow, any row whose bound reaches thr),
        // else an empty range
        auto describe_kept = [&](uint32_t i, float thr, bool use_rowmax, ScreenRow& R) {
            R.lo = R.hi = 0;
            if (i >= nrows) return;
            const uint32_t r = overflow ? i : rows[i];
            if (overflow ? !(row_bound(r) >= thr) : (use_rowmax && !(rowmax[i] >= thr))) return;
            describe(r, R);
        };
        // ---- phase C: lower bound and per-row upper bounds, two rows per warp at a time
        {
            uint64_t scanned = 0;
            for (uint32_t i = 2 * warp; i < nrows; i += 2 * nwarps) {
                ScreenRow R[2];
                describe_kept(i, thr0, false, R[0]);
                describe_kept(i + 1, thr0, false, R[1]);
                scanned += (uint64_t)(R[0].hi - R[0].lo) + (uint64_t)(R[1].hi - R[1].lo);
                float lbm[2] = {-INFINITY, -INFINITY}, ubm[2] = {-INFINITY, -INFINITY};
                scan2(R, false, 0.f, lbm, ubm);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    float m = ubm[q];
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
                    ubm[q] = m;
                    lb = fmaxf(lb, lbm[q]);
                }
                if (!overflow && lane == 0) {
                    rowmax[i] = ubm[0];
                    if (i + 1 < nrows) rowmax[i + 1] = ubm[1];
                }
            }
            if (lane == 0) item_n += scanned;
        }
        const float lbs = RF(tmp.rf).Reduce(lb, cub::Max());
        if (threadIdx.x == 0) sh.lb = lbs;
        __syncthreads();
        const float thr = fmaxf(fmaxf(sh.lb, seed), 0.f);
        // ---- phase D: candidate list from the rows reaching thr, two per warp at a time
        for (uint32_t i = 2 * warp; i < nrows; i += 2 * nwarps) {
            ScreenRow R[2];
            describe_kept(i, thr, true, R[0]);
            describe_kept(i + 1, thr, true, R[1]);
            if (R[0].hi == R[0].lo && R[1].hi == R[1].lo) continue;
            float lbm[2], ubm[2];
            scan2(R, true, thr, lbm, ubm);
        }
        __syncthreads();
        const uint32_t ncand = sh.ncand;
        unsigned long long kbest = 0ull;
        // hand the listed candidates to the scoring kernel (the listing already
        // spilled past kCandCap straight into the global list)
        const uint32_t nlisted = min(ncand, (uint32_t)kCandCap);
        if (threadIdx.x == 0) s_gbase = atomicAdd(&status->cand_count, nlisted);
        __syncthreads();
        const uint32_t gbase = s_gbase;
        const bool handed = (uint64_t)gbase + nlisted <= gcand_cap && !sh.gfull;
        if (handed) {
            for (uint32_t i = threadIdx.x; i < nlisted; i += blockDim.x)
                gcand[gbase + i] = ((unsigned long long)kk << 32) | ((unsigned long long)cand[3 * i + 1] << 20) |
                                   ((unsigned long long)cand[3 * i] << 10) | (unsigned long long)cand[3 * i + 2];
        } else {
            // the global list is full: mark this window's slots in it empty and
            // score every item of the reaching rows here
            for (uint64_t i = (uint64_t)gbase + threadIdx.x; i < gcand_cap && i < (uint64_t)gbase + nlisted;
                 i += blockDim.x)
                gcand[i] = ~0ull;
            for (uint32_t i = threadIdx.x; i < nrows; i += blockDim.x) {
                const uint32_t r = overflow ? i : rows[i];
                if (!(row_bound(r) >= thr)) continue;
                ScreenRow R;
                describe(r, R);
                for (int x = R.lo; x < R.hi; ++x) {
                    const float xv = R.xr ? R.xr[x] : 0.f;
                    const float ub = (R.uf + R.ua[x]) - xv;
                    if (!(ub >= thr)) continue;
                    const uint32_t a = R.fixed_a ? R.y : (uint32_t)x, b = R.fixed_a ? (uint32_t)x : R.y;
                    const float v = pair_exact_g(d, T, V, f, R.t, p, a, b, mf | chmask[R.t]);
                    ++exact_n;
                    if (!(v > 0.f)) continue;
                    const uint64_t rr0 = (uint64_t)R.t + (uint64_t)M * a + (uint64_t)M * S2 * b;
                    uint32_t pr = item_priority(rr0, d.WG, lbits);
                    for (uint64_t rr = rr0 + items; rr < slots; rr += items) {
                        const uint32_t p2 = item_priority(rr, d.WG, lbits);
                        pr = p2 < pr ? p2 : pr;
                    }
                    const unsigned long long key =
                        ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xFFFFFFFFu - pr);
                    kbest = key > kbest ? key : kbest;
                }
            }
        }
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

// Screening order of a batch of flagged windows: grouped by best label f (a
// counting sort), so CTAs running at the same time read the same template's
// cross-term slices from L2.  Windows past the flagged count go last.
__global__ void __launch_bounds__(1024) label_order_kernel(Dims d, const uint32_t* __restrict__ flag,
                                                           const DevStatus* status,
                                                           const uint32_t* __restrict__ best_lab, uint32_t k0,
                                                           uint32_t kc, uint32_t* order)
{
    extern __shared__ uint32_t hist[];   // [M + 1]
    const uint32_t nflag = status->n_flag, M = d.M;
    for (uint32_t i = threadIdx.x; i <= M; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < kc; j += blockDim.x) {
        const uint32_t f = k0 + j < nflag ? min(best_lab[flag[k0 + j]], M) : M;
        atomicAdd(&hist[f], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t i = 0; i <= M; ++i) { const uint32_t c = hist[i]; hist[i] = run; run += c; }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < kc; j += blockDim.x) {
        const uint32_t f = k0 + j < nflag ? min(best_lab[flag[k0 + j]], M) : M;
        order[atomicAdd(&hist[f], 1u)] = j;
    }
}

// Exact scores of the listed candidates, one thread each: entry = window slot
// kk (32 bits) | t (12) | a (10) | b (10).  Folds the canonical winner key into
// keys[k0 + kk].
__global__ void __launch_bounds__(256) score_kernel(Dims d, const float* __restrict__ V, const float* __restrict__ T,
                                                    const uint32_t* __restrict__ flag, uint32_t k0,
                                                    const uint32_t* __restrict__ best_lab,
                                                    const uint32_t* __restrict__ best_idx,
                                                    const unsigned long long* __restrict__ gcand, uint32_t cap,
                                                    DevStatus* status, unsigned long long* keys,
                                                    const unsigned long long* __restrict__ chmask)
{
    const uint32_t n = min(status->cand_count, cap);
    const uint32_t S2 = 2 * d.S + 1, M = d.M;
    const uint64_t items = (uint64_t)S2 * S2 * M;
    const uint64_t nloc = (items - 1) / d.WG + 1;
    const uint64_t slots = nloc * d.WG;
    uint32_t lbits = 0;
    while ((1u << lbits) < d.WG) ++lbits;
    uint32_t done = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long e = gcand[i];
        if (e == ~0ull) continue;
        const uint32_t kk = (uint32_t)(e >> 32);
        const uint32_t t = (uint32_t)(e >> 20) & 0xFFFu, a = (uint32_t)(e >> 10) & 0x3FFu, b = (uint32_t)e & 0x3FFu;
        if ((uint64_t)k0 + kk >= status->n_flag || t >= M || a >= S2 || b >= S2) continue;
        const uint32_t id = flag[k0 + kk];
        const uint32_t f = best_lab[id], p = best_idx[id];
        const float acc = pair_exact_g(d, T, V, f, t, p, a, b, chmask[f] | chmask[t]);
        ++done;
        if (!(acc > 0.f)) continue;
        const uint64_t r = (uint64_t)t + (uint64_t)M * a + (uint64_t)M * S2 * b;
        uint32_t pr = item_priority(r, d.WG, lbits);
        for (uint64_t rr = r + items; rr < slots; rr += items) {
            const uint32_t p2 = item_priority(rr, d.WG, lbits);
            pr = p2 < pr ? p2 : pr;
        }
        atomicMax(&keys[k0 + kk],
                  ((unsigned long long)__float_as_uint(acc) << 32) | (unsigned long long)(0xFFFFFFFFu - pr));
    }
    if (done) atomicAdd(&status->n_pair_exact, done);
}

}  // namespace

struct PcConfig {
    int Q = 0;
    size_t smem = 0;
};

// The partial-correlation launch shape of the calling thread's current chunk:
// launch_overlap_tables sets it and launch_overlap_fast reads it, both inside the
// same fbp_pursue_chunk call on that thread, so no other call can come between them.
PcConfig& pc_config()
{
    static thread_local PcConfig c;
    return c;
}

int launch_overlap_tables(const Dims& d, const Work& w, const float* T, cudaStream_t st)
{
    const Layout& L = *w.lay;
    if (!L.screened) return FBP_OK;
    const uint32_t S2 = 2 * d.S + 1;
    count_launch(4);
    energy_table_kernel<<<(d.M * S2 + 255) / 256, 256, 0, st>>>(d, T, w.at<float2>(L.off_et));
    const size_t smem = (size_t)2 * d.C * d.W * 4 + 8 + (size_t)kLagChunk * (d.W + 1) * 8;
    if (smem > 200 * 1024) return fail(FBP_E_ARG, "template too large for the pair table kernel");
    FBP_CUDA(allow_max_dyn_smem(cross_table_kernel));
    cross_table_kernel<<<d.M * d.M, 256, smem, st>>>(d, T, w.at<float>(L.off_xt), w.at<float>(L.off_xtt),
                                                     w.at<float>(L.off_mx));
    energy_max_kernel<<<(d.M + 127) / 128, 128, 0, st>>>(d, w.at<float2>(L.off_et), w.at<float>(L.off_mx) + (size_t)d.M * d.M);
    template_order_kernel<<<1, 256, d.M * 4, st>>>(d, T, w.at<uint32_t>(L.off_perm),
                                                  reinterpret_cast<unsigned long long*>(w.at<uint32_t>(L.off_perm) + ((d.M + 1) & ~1u)));
    FBP_CUDA(cudaGetLastError());
    // channel unions of the template groups decide how many templates a
    // partial-correlation CTA can stage: read the order and masks back once
    std::vector<uint32_t> perm(d.M);
    std::vector<unsigned long long> mask(d.M);
    FBP_CUDA(cudaMemcpyAsync(perm.data(), w.at<uint32_t>(L.off_perm), d.M * 4, cudaMemcpyDeviceToHost, st));
    FBP_CUDA(cudaMemcpyAsync(mask.data(), w.at<uint32_t>(L.off_perm) + ((d.M + 1) & ~1u), d.M * 8,
                             cudaMemcpyDeviceToHost, st));
    FBP_CUDA(cudaStreamSynchronize(st));
    PcConfig& pc = pc_config();
    pc.Q = 0;
    // group size: least estimated work, sum over groups of Q x (union channels),
    // weighted by the measured cost per multiply-add of each group size (two
    // strip loads feed Q templates; below 4 the shared-memory loads dominate)
    double best = 0.0;
    const int want_q = (int)tuning().pc_group;
    for (int Q = 8; Q >= 1; Q >>= 1) {
        if (want_q && Q > want_q) continue;
        // measured time per unit of work relative to Q = 4: Q = 8 0.72 (64 ch, 200
        // templates, 60 s) and 0.84 (16 ch, 40 templates, 10 min), Q = 2 1.0-1.2, Q = 1 1.3-1.4
        const double eff = Q >= 8 ? 0.78 : (Q == 4 ? 1.0 : (Q == 2 ? 1.2 : 1.6));
        uint32_t cu_max = 0;
        double work = 0.0;
        for (uint32_t g0 = 0; g0 < d.M; g0 += Q) {
            unsigned long long m = 0ull;
            for (uint32_t q = 0; q < (uint32_t)Q && g0 + q < d.M; ++q) m |= mask[perm[g0 + q]];
            uint32_t cu = 0;
            for (uint32_t c = 0; c < d.C; ++c) cu += (c >= 64 || ((m >> c) & 1ull)) ? 1u : 0u;
            cu_max = cu > cu_max ? cu : cu_max;
            work += (double)Q * cu;
        }
        const size_t smem = pc_smem_bytes(d, cu_max, Q);
        if (!(smem <= 110 * 1024 || (Q == 1 && smem <= 200 * 1024))) continue;
        if (want_q) {   // the caller's group size, or the largest feasible one below it
            pc.Q = Q;
            pc.smem = smem;
            break;
        }
        if (pc.Q == 0 || work * eff < best) {
            pc.Q = Q;
            pc.smem = smem;
            best = work * eff;
        }
    }
    return FBP_OK;
}

int launch_overlap_fast(const Dims& d, const Work& w, const float* V, const float* T, const float* theta,
                        uint32_t nflag_max, cudaStream_t st)
{
    const Layout& L = *w.lay;
    if (!L.screened) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    if (nflag_max == 0) return FBP_OK;
    const uint32_t S2 = 2 * d.S + 1;
    if (S2 > 1024 || d.C > 256 || d.M > 4096) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    FBP_CUDA(cudaMemsetAsync(w.keys(), 0, sizeof(unsigned long long) * nflag_max, st));
    const PcConfig pc = pc_config();
    const int Q = pc.Q;
    const size_t smem_a = pc.smem;
    if (Q == 0) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    const uint32_t pc_threads = 32u * std::min<uint32_t>((S2 + 15) / 16, kPcMaxWarps);
    const bool bstaged = (uint64_t)d.M * S2 * 8 <= kBStage;
    const size_t smem_b = screen_smem_bytes(d.M, S2, bstaged);
    if (smem_b > 200 * 1024) return launch_overlap_plain(d, w, V, T, theta, nflag_max, st);
    FBP_CUDA(allow_max_dyn_smem(screen_kernel));
    const uint32_t groups = (d.M + Q - 1) / Q;
    float* G = w.at<float>(L.off_g);
    const float2* Et = w.at<float2>(L.off_et);
    const float* XT = w.at<float>(L.off_xt);
    const uint32_t* perm = w.at<uint32_t>(L.off_perm);
    const unsigned long long* chm = reinterpret_cast<const unsigned long long*>(perm + ((d.M + 1) & ~1u));
    for (uint32_t k0 = 0; k0 < nflag_max; k0 += (uint32_t)L.gbatch) {
        const uint32_t kc = (uint32_t)((nflag_max - k0) < L.gbatch ? (nflag_max - k0) : L.gbatch);
        count_launch(3);
        {
        KScope ks(&fbp_chunk_stats::ms_partial_corr, st);
        // persistent over the windows: as many CTAs as fit resident, split over the template groups
#define FBP_PC(QQ)                                                                                            \
    case QQ: {                                                                                                \
        FBP_CUDA(allow_max_dyn_smem(partial_corr_kernel<QQ>));                                                          \
        int per_sm = 1;                                                                                       \
        FBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, partial_corr_kernel<QQ>,              \
                                                               (int)pc_threads, smem_a));                 \
        const uint32_t want = (uint32_t)((148u * (per_sm > 0 ? per_sm : 1) + groups - 1) / groups);           \
        const uint32_t slices = std::min<uint32_t>((kc + kPcWin - 1) / kPcWin, want);                         \
        partial_corr_kernel<QQ><<<dim3(slices, groups), pc_threads, smem_a, st>>>(                          \
            d, V, T, w.L(), theta, Et, perm, chm, w.flag(), w.status(), w.best_lab(), w.best_idx(), k0, kc, G); \
        break;                                                                                                \
    }
        switch (Q) {
            FBP_PC(8)
            FBP_PC(4)
            FBP_PC(2)
            FBP_PC(1)
        }
#undef FBP_PC
        }
        const uint32_t gb = kc < kScreenGrid ? kc : kScreenGrid;
        uint32_t* order = w.at<uint32_t>(L.off_order);
        count_launch();
        label_order_kernel<<<1, 1024, (d.M + 1) * 4, st>>>(d, w.flag(), w.status(), w.best_lab(), k0, kc, order);
        FBP_CUDA(cudaMemsetAsync(&w.status()->cand_count, 0, 4, st));
        unsigned long long* gcand = w.at<unsigned long long>(L.off_cand);
        {
        KScope ks(&fbp_chunk_stats::ms_screen, st);
        screen_kernel<<<gb, kScrThreads, smem_b, st>>>(d, V, T, w.L(), theta, Et, XT, w.at<float>(L.off_xtt), G, k0, kc,
                                                       w.flag(), w.status(), w.best_lab(), w.best_idx(), w.best_lik(),
                                                       w.keys(), w.at<float>(L.off_mx), gcand, (uint32_t)L.cand_cap, chm,
                                                       bstaged ? nullptr : w.at<float>(L.off_bscr), order);
        }
        KScope ks(&fbp_chunk_stats::ms_score, st);
        score_kernel<<<148 * 8, 256, 0, st>>>(d, V, T, w.flag(), k0, w.best_lab(), w.best_idx(), gcand,
                                              (uint32_t)L.cand_cap, w.status(), w.keys(), chm);
        FBP_CUDA(cudaGetLastError());
    }
    return FBP_OK;
}

}  // namespace fbp
