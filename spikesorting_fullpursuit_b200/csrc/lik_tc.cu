// lik_tc.cu -- template-by-voltage likelihood on the 5th-generation tensor cores.
//
// L[t][s] = bias[t] + sum_c sum_j T[t][c][j] V[c][s+j]  (compute_full_likelihood,
// binary_pursuit.cl:216-300) as a GEMM over K = (tap j, channel c):
//   A[s][(j,c)] = V[c][s+j]   -- a Hankel matrix of the voltage
//   B[(j,c)][t] = T[t][c][j]
// with tcgen05.mma kind::tf32, M = 128 samples per tile, N = templates, K = 8
// channels per instruction, FP32 accumulators in TMEM.
//
// The voltage is kept on the device as Vq[Cp/4][rows][4] (four channels per
// 16-byte row).  A tile's strip of rows [s0, s0+128+W-1) is copied into shared
// memory once with cp.async.bulk; the UMMA operand for tap j is the same strip
// seen from row j, i.e. the shared-memory descriptor's start address advanced by
// 16*j bytes (canonical K-major layout without swizzle: 8-row core matrices of
// 16-byte rows).  No Hankel expansion is ever materialised.  Templates are
// pre-arranged as Tq[j][Cp/8][2][Np][4] and streamed per (tap, channel pair)
// through a ring of shared-memory stages.
//
// Exactness.  The pursuit reads a likelihood either for its sign or, when it is
// positive, for its value.  The epilogue bounds |estimate - reference float
// result| rigorously (TF32 operand truncation, FP32 accumulation, the
// reference's own sequential rounding), stores the estimate wherever
// estimate + bound <= 0, and queues every other sample for an exact FP32
// recomputation in the reference order (fixup kernel).  The stored likelihood
// therefore equals the reference's wherever the reference's is positive and is
// <= 0 wherever the reference's is <= 0.
//
// Roles of the 6 warps of a CTA: warp 0 lane 0 issues the bulk copies, warp 1
// allocates TMEM and lane 0 issues the MMAs, warps 2-5 run the epilogue (warp w
// reads TMEM lanes 32*(w%4) .. +32).  Every mbarrier wait is bounded; on a
// timeout the kernel records an error in the status word and returns after
// draining its own operations.
#include <cub/cub.cuh>

#include <algorithm>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

constexpr int kTile = 128;         // samples per UMMA tile (M)
constexpr int kThreads = 192;
constexpr uint64_t kWaitNs = 250ull * 1000ull * 1000ull;   // longest mbarrier wait (global timer)
constexpr uint32_t kFixCap = 512;   // queued 32-row entries recomputed in the CTA itself; more go to the global queue
// windows one tile of 128 consecutive samples can touch
__host__ __device__ __forceinline__ uint32_t win_slots(uint32_t W) { return (kTile + W - 1) / W + 1; }

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: false once the phase has not completed within kWaitNs of
// device time (the global nanosecond timer), checked every 64 polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    // canonical K-major, no swizzle; version 1 (sm_100) at bit 46
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Issues the MMAs of k-steps [k0, k0 + nk) for NT tiles.  k-step k is (tap j,
// channel pair qp) = (k / nqp, k % nqp); A of tile i is its strip seen from row j
// of channel block 2 qp, B the staged template k-step.  The descriptors advance
// in their start-address field (16-byte units): shared addresses stay below
// 256 KB, so the 14-bit field never carries into the next one.  The tile loop is
// unrolled: one issuing thread's dependent address arithmetic, not the tensor
// core, otherwise sets the MMA rate at these sizes.
template <int NT>
__device__ __forceinline__ void issue_ksteps_n(uint32_t d_tmem, uint32_t Np, uint64_t adesc0, uint32_t tile_units,
                                               uint32_t qp_units, uint64_t bdesc0, uint32_t kstep_units, uint32_t k0,
                                               uint32_t nk, uint32_t nqp, uint32_t idesc)
{
    uint32_t j = k0 / nqp, qp = k0 - j * nqp;
    uint64_t bd = bdesc0;
    uint32_t dd[NT];
    uint64_t ao[NT];
#pragma unroll
    for (int i = 0; i < NT; ++i) {
        dd[i] = d_tmem + i * Np;
        ao[i] = (uint64_t)i * tile_units;
    }
    for (uint32_t kq = 0; kq < nk; ++kq) {
        const uint64_t ad = adesc0 + j + qp * qp_units;
        const uint32_t acc = (k0 + kq) > 0 ? 1u : 0u;
#pragma unroll
        for (int i = 0; i < NT; ++i) umma_tf32(dd[i], ad + ao[i], bd, idesc, acc);
        bd += kstep_units;
        if (++qp == nqp) {
            qp = 0;
            ++j;
        }
    }
}

__device__ __forceinline__ void issue_ksteps(uint32_t d_tmem, uint32_t Np, uint32_t ntl, uint64_t adesc0,
                                             uint32_t tile_units, uint32_t qp_units, uint64_t bdesc0,
                                             uint32_t kstep_units, uint32_t k0, uint32_t nk, uint32_t nqp,
                                             uint32_t idesc)
{
    switch (ntl) {
        case 1: issue_ksteps_n<1>(d_tmem, Np, adesc0, tile_units, qp_units, bdesc0, kstep_units, k0, nk, nqp, idesc); break;
        case 2: issue_ksteps_n<2>(d_tmem, Np, adesc0, tile_units, qp_units, bdesc0, kstep_units, k0, nk, nqp, idesc); break;
        case 3: issue_ksteps_n<3>(d_tmem, Np, adesc0, tile_units, qp_units, bdesc0, kstep_units, k0, nk, nqp, idesc); break;
        default: issue_ksteps_n<4>(d_tmem, Np, adesc0, tile_units, qp_units, bdesc0, kstep_units, k0, nk, nqp, idesc); break;
    }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

struct TcParams {
    Dims d;
    const float* V;       // [C][N] (exact recomputation)
    const float* T;       // [M][C][W]
    const float* Vq;      // [Cq][rows][4]
    const float* Tq;      // [W][Cq/2][2][Np][4]
    const float* bias;    // [M]
    const float* tnorm;   // [M][C] channel norms of the templates
    const unsigned long long* tchm;   // [M] channels c < 64 where template t is not all zero (C <= 64)
    const float* Tp;      // [M][C][Wp] templates, taps padded to a multiple of 4 (exact recomputation)
    const uint32_t* list; // listed windows (mode 1) or null (mode 0: contiguous tiles)
    uint32_t nitems;      // tiles (mode 0) or listed windows (mode 1)
    uint32_t tile0;       // mode 0: first tile of the range (tile k covers samples [128 (tile0 + k), +128))
    uint32_t rows;        // rows of each Vq channel block
    uint32_t Cq, Np, ntiles, R8, stages, ncols, group;   // group: k-steps per template stage
    float* L;
    unsigned long long* fix;
    uint32_t fix_cap;
    DevStatus* status;
    float k_a, k_b;       // bound = k_a * sum_c |T_tc| |V_c strip| + k_b * |bias_t|
    // lazy exactness (pursuit): only samples whose sign is uncertain and the
    // contenders for each window's maximum are recomputed exactly; every other
    // positive sample keeps its estimate and its (window, template) row is flagged
    uint32_t lazy;
    unsigned long long* wkey;   // [nw] window maximum: see window_key()
    uint8_t* wpos;              // [nw] 1 if the window holds a positive likelihood
    uint8_t* wflag;             // [nw][M] 1: the window's row of template t holds estimates
    uint32_t wslots;            // win_slots(W): window slots per tile in shared memory
};

// Key of a positive likelihood v at (template t, sample s) of window w:
// larger for a larger value, then for a smaller t, then for a smaller s -- the
// order in which compute_template_maximum_likelihood (binary_pursuit.cl:395-408)
// keeps the first maximum.  Needs W <= 1024 and t < 2^22.
__device__ __forceinline__ unsigned long long window_key(float v, uint32_t t, uint32_t local_s)
{
    return ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xFFFFFFFFu - ((t << 10) | local_s));
}

// The reference's sum, skipping template channels that are entirely zero
// (tnorm == 0): there it adds 0 * v terms, which leave a nonzero sum unchanged
// (and a zero sum zero, up to the sign of zero, which no decision reads).
__device__ float exact_likelihood(const Dims& d, const float* __restrict__ V, const float* __restrict__ T,
                                  float b, uint32_t t, uint32_t s, const float* __restrict__ tnorm)
{
    float acc = b;
    for (uint32_t c = 0; c < d.C; ++c) {
        if (tnorm[(uint64_t)t * d.C + c] == 0.f) continue;
        const float* tr = T + ((uint64_t)t * d.C + c) * d.W;
        const float* vr = V + (uint64_t)c * d.N + s;
        for (uint32_t j = 0; j < d.W; ++j) acc = __fadd_rn(acc, __fmul_rn(tr[j], vr[j]));
    }
    return acc;
}


// TMEM -> registers: 4 consecutive accumulator columns of the warp's 32 lanes.
// The wait is a separate statement that names the destination registers, so no
// use of them is scheduled before it and a load can be in flight while the
// previous group is processed (no function call may come between the two).
__device__ __forceinline__ void tmem_ld4_issue(uint32_t taddr, uint32_t (&r)[4])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait4(uint32_t (&r)[4])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])::"memory");
}

// Shared-memory state of a likelihood CTA's epilogue for its current tiles.
// Queued runs: mask << 32 | t << 5 | tile << 2 | quarter -- rows 32 quarter + k of
// the tile for the set bits k of the mask.
struct Epi {
    const uint32_t* t_s0;    // [tiles] first sample
    const uint32_t* t_rows;  // [tiles] rows in use
    const uint32_t* t_w0;    // [tiles] first window
    const float* sbias;      // [M]
    const float* bnd;        // [tiles][M] error bound of the estimates
    int* s_mlb;              // [tiles][wslots] largest lower bound (float bits)
    uint32_t* s_pos;         // [tiles][wslots] a positive value seen
    unsigned long long* s_key;   // [tiles][wslots] window maximum key
    uint8_t* s_inex;         // [tiles][wslots][M] row holds estimates
    unsigned long long* fq;  // [kFixCap]
    uint32_t* nfq;
    uint32_t wslots;
};

// Queueing of the warp's flagged samples of one template (ballot m != 0), out of
// line: one entry for the warp's 32 rows in the CTA's list; when that is full,
// runs of 4 rows in the global queue; when that is full too, computed right here.
// Returns the sample's exact value if computed here (and sets *here), else `out`.
__device__ __noinline__ float queue_runs(const Dims d, uint32_t m, bool need, uint32_t t, uint32_t i, uint32_t row,
                                         uint32_t s, float b, float out, bool* here, unsigned long long* fq,
                                         uint32_t* nfq, DevStatus* status, unsigned long long* fix, uint32_t fix_cap,
                                         const float* V, const float* T, const float* tnorm)
{
    const uint32_t lane = threadIdx.x & 31;
    uint32_t slot = 0;
    if (lane == 0) slot = atomicAdd(nfq, 1u);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (slot < kFixCap) {
        if (lane == 0) fq[slot] = ((unsigned long long)m << 32) | (t << 5) | (i << 2) | (row >> 5);
        return out;
    }
    const uint32_t nib = (m >> (4 * (lane >> 2))) & 0xFu;
    uint32_t g = 0;
    if (nib && (lane & 3u) == 0) {
        g = atomicAdd(&status->n_fix, 1u);
        if (g < fix_cap) fix[g] = ((unsigned long long)t << 40) | ((unsigned long long)nib << 32) | s;
    }
    g = __shfl_sync(0xffffffffu, g, lane & ~3u);   // all lanes: the run's first lane holds g
    if (need && g >= fix_cap) {
        *here = true;
        return exact_likelihood(d, V, T, b, t, s, tnorm);
    }
    return out;
}

__device__ __forceinline__ float enqueue(const TcParams& P, const Epi& E, bool need, uint32_t t, uint32_t i,
                                         uint32_t row, uint32_t s, float b, float out, bool* here)
{
    *here = false;
    const uint32_t m = __ballot_sync(0xffffffffu, need);
    if (m == 0u) return out;
    return queue_runs(P.d, m, need, t, i, row, s, b, out, here, E.fq, E.nfq, P.status, P.fix, P.fix_cap, P.V, P.T,
                      P.tnorm);
}

// an exact positive value v at (t, s) of tile i: the window's maximum key and positive flag
__device__ __forceinline__ void note_exact(const Dims& d, const Epi& E, float v, uint32_t t, uint32_t i, uint32_t s)
{
    if (!(v > 0.f)) return;
    const uint32_t w = s / d.W, slot = i * E.wslots + (w - E.t_w0[i]);
    atomicMax(&E.s_key[slot], window_key(v, t, s - w * d.W));
    E.s_pos[slot] = 1u;
}

// The same for the exact values of the lanes with `has`, one atomic per window
// slot the warp's rows meet.
__device__ __forceinline__ void warp_note_exact(const Dims& d, const Epi& E, bool has, float v, uint32_t t,
                                                uint32_t i, uint32_t s)
{
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31;
    has = has && v > 0.f;
    uint32_t pend = __ballot_sync(full, has);
    if (pend == 0u) return;
    const uint32_t w = s / d.W, slot = i * E.wslots + (w - E.t_w0[i]);
    const unsigned long long key = has ? window_key(v, t, s - w * d.W) : 0ull;
    while (pend) {
        const uint32_t lead = __ffs(pend) - 1;
        const uint32_t sl = __shfl_sync(full, slot, lead);
        const bool mine = has && slot == sl;
        unsigned long long k = mine ? key : 0ull;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_xor_sync(full, k, off);
            k = o > k ? o : k;
        }
        if (lane == lead) {
            atomicMax(&E.s_key[sl], k);
            E.s_pos[sl] = 1u;
        }
        pend &= ~__ballot_sync(full, mine);
    }
}

// Each row's largest certain lower bound (mlb > 0 where pos) into its window
// slot.  The warp's rows are consecutive, so for W >= 32 they meet at most two
// windows: two warp reductions and at most two shared atomics.
__device__ __forceinline__ void warp_window_mlb(const Epi& E, uint32_t W, uint32_t wslot, float mlb, bool pos)
{
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31;
    const uint32_t pm = __ballot_sync(full, pos);
    if (pm == 0u) return;
    if (W < 32) {
        if (pos) {
            atomicMax(&E.s_mlb[wslot], __float_as_int(mlb));
            E.s_pos[wslot] = 1u;
        }
        return;
    }
    const uint32_t lead = __ffs(pm) - 1;
    const uint32_t wa = __shfl_sync(full, wslot, lead);
    const bool in_a = pos && wslot == wa, in_b = pos && wslot != wa;
    const int ma = __reduce_max_sync(full, in_a ? __float_as_int(mlb) : 0);
    const int mb = __reduce_max_sync(full, in_b ? __float_as_int(mlb) : 0);
    const uint32_t bm = __ballot_sync(full, in_b);
    if (lane == lead) {
        atomicMax(&E.s_mlb[wa], ma);
        E.s_pos[wa] = 1u;
    }
    if (bm != 0u && lane == __ffs(bm) - 1) {
        atomicMax(&E.s_mlb[wslot], mb);
        E.s_pos[wslot] = 1u;
    }
}

// Pass 1 of the epilogue over `ntiles` tiles (TMEM columns tbase + i * Np, this
// thread's row) for the template groups t0 = tfirst, tfirst + tstep, ... (4
// templates each): estimates stored; samples of uncertain sign (lazy) or that
// can be positive (not lazy) queued; each window slot's largest certain lower
// bound.  The TMEM load of the next group is in flight while a group is
// evaluated; it completes before any queueing call.
__device__ __forceinline__ void epi_pass1(const TcParams& P, const Epi& E, uint32_t tbase, uint32_t ntiles,
                                          uint32_t row, bool lazy, uint32_t tfirst, uint32_t tstep)
{
    const Dims& d = P.d;
    for (uint32_t i = 0; i < ntiles; ++i) {
        const uint32_t s = E.t_s0[i] + row;
        const bool valid = row < E.t_rows[i];
        const bool live = valid && (uint64_t)s + d.W < d.N;
        const uint32_t wslot = valid ? i * E.wslots + (s / d.W - E.t_w0[i]) : 0u;
        const float* bnd = E.bnd + i * d.M;
        float mlb = 0.f;
        bool pos = false;
        uint32_t r[4];
        if (tfirst < d.M) {
            tmem_ld4_issue(tbase + i * P.Np + tfirst, r);
            tmem_wait4(r);
        }
#pragma unroll 1
        for (uint32_t t0 = tfirst; t0 < d.M; t0 += tstep) {
            float est[4];
            bool need[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) est[e] = __uint_as_float(r[e]);
            const bool more = t0 + tstep < d.M;
            if (more) tmem_ld4_issue(tbase + i * P.Np + t0 + tstep, r);
            bool any = false;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t t = t0 + e;
                need[e] = false;
                if (t >= d.M) break;   // the same for every lane
                est[e] += E.sbias[t];
                const float bd = bnd[t];
                const bool certain = lazy && live && est[e] - bd > 0.f;
                need[e] = live && !(est[e] + bd <= 0.f) && !certain;
                if (certain) {
                    mlb = fmaxf(mlb, est[e] - bd);
                    pos = true;
                }
                if (!live) est[e] = 0.f;
                if (valid && !need[e]) P.L[(uint64_t)t * d.N + s] = est[e];
                any |= need[e];
            }
            any = __any_sync(0xffffffffu, any);
            if (more) tmem_wait4(r);
            if (any) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const uint32_t t = t0 + e;
                    if (t >= d.M) break;
                    bool here = false;
                    const float out = enqueue(P, E, need[e], t, i, row, s, E.sbias[t], est[e], &here);
                    if (here && lazy) note_exact(d, E, out, t, i, s);
                    if (need[e]) P.L[(uint64_t)t * d.N + s] = out;
                }
            }
        }
        if (lazy) warp_window_mlb(E, d.W, wslot, mlb, pos);
    }
}

// Pass 2 (lazy): contenders for each window slot's maximum (upper bound reaching
// its largest lower bound) are queued; the other certainly positive samples keep
// their estimate and flag their (window, template) row.
__device__ __forceinline__ void epi_pass2(const TcParams& P, const Epi& E, uint32_t tbase, uint32_t ntiles,
                                          uint32_t row, uint32_t tfirst, uint32_t tstep)
{
    const Dims& d = P.d;
    for (uint32_t i = 0; i < ntiles; ++i) {
        const uint32_t s = E.t_s0[i] + row;
        const bool valid = row < E.t_rows[i];
        const bool live = valid && (uint64_t)s + d.W < d.N;
        const uint32_t wslot = valid ? i * E.wslots + (s / d.W - E.t_w0[i]) : 0u;
        const float mlb = __int_as_float(E.s_mlb[wslot]);
        const float* bnd = E.bnd + i * d.M;
        uint8_t* inex = E.s_inex + (size_t)wslot * d.M;
        uint32_t r[4];
        if (tfirst < d.M) {
            tmem_ld4_issue(tbase + i * P.Np + tfirst, r);
            tmem_wait4(r);
        }
#pragma unroll 1
        for (uint32_t t0 = tfirst; t0 < d.M; t0 += tstep) {
            float est[4];
            bool cont[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) est[e] = __uint_as_float(r[e]);
            const bool more = t0 + tstep < d.M;
            if (more) tmem_ld4_issue(tbase + i * P.Np + t0 + tstep, r);
            bool any = false;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t t = t0 + e;
                cont[e] = false;
                if (t >= d.M) break;
                est[e] += E.sbias[t];
                const float bd = bnd[t];
                const bool certain = live && est[e] - bd > 0.f;
                cont[e] = certain && est[e] + bd >= mlb;
                if (certain && !cont[e]) inex[t] = 1;
                any |= cont[e];
            }
            any = __any_sync(0xffffffffu, any);
            if (more) tmem_wait4(r);
            if (any) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const uint32_t t = t0 + e;
                    if (t >= d.M) break;
                    bool here = false;
                    const float out = enqueue(P, E, cont[e], t, i, row, s, E.sbias[t], est[e], &here);
                    if (here) {
                        note_exact(d, E, out, t, i, s);
                        P.L[(uint64_t)t * d.N + s] = out;
                    }
                }
            }
        }
    }
}

// Exact recomputation of the queued runs, one warp per entry (warps w0, w0 +
// wstride, ...): lane k carries the sum of row 32 quarter + k, adding its
// products one at a time in the reference order (channel-major, taps ascending)
// over the template's non-zero channels (an all-zero channel adds exact zeros);
// the template row of the next such channel is loaded while the current one is
// summed and staged in the warp's shared scratch (2 x 128 floats).  Lanes whose
// row is not in the entry's mask compute a value nobody reads.  Vt: the strips
// transposed to channel-major rows (channel c of tile i at (i Cp + c) R8).
__device__ __forceinline__ void recompute_runs(const TcParams& P, const Epi& E, const float* Vt, uint32_t nq,
                                               uint32_t w0, uint32_t wstride, float* scratch, bool lazy)
{
    const Dims& d = P.d;
    const uint32_t lane = threadIdx.x & 31, W = d.W, Wp = (W + 3) & ~3u, Cp = P.Cq * 4;
    float* tw = scratch;   // this warp's [2][128]
    for (uint32_t qi = w0; qi < nq; qi += wstride) {
        const unsigned long long e = E.fq[qi];
        const uint32_t mask = (uint32_t)(e >> 32), lo = (uint32_t)e;
        const uint32_t t = lo >> 5, i = (lo >> 2) & 7u, r = (lo & 3u) * 32u + lane;
        float acc = E.sbias[t];
        const float* tb = P.Tp + (uint64_t)t * d.C * Wp;
        const float* tnr = P.tnorm + (uint64_t)t * d.C;
        // the template's non-zero channels in order: from its mask (C <= 64), else by norms
        const bool bym = d.C <= 64;
        const unsigned long long chm = bym ? P.tchm[t] : 0ull;
        auto next_chan = [&](uint32_t from) -> uint32_t {
            if (bym) {
                const unsigned long long rest = from < 64 ? chm & (~0ull << from) : 0ull;
                return rest ? (uint32_t)(__ffsll((long long)rest) - 1) : d.C;
            }
            uint32_t c = from;
            while (c < d.C && tnr[c] == 0.f) ++c;
            return c;
        };
        uint32_t c = next_chan(0);
        float tn[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t x = lane + 32u * q;
            tn[q] = (c < d.C && x < W) ? __ldg(tb + (uint64_t)c * Wp + x) : 0.f;
        }
        uint32_t buf = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) tw[lane + 32u * q] = tn[q];
        __syncwarp();
        while (c < d.C) {
            const uint32_t cn = next_chan(c + 1);
            if (cn < d.C) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t x = lane + 32u * q;
                    tn[q] = x < W ? __ldg(tb + (uint64_t)cn * Wp + x) : 0.f;
                }
            }
            const float* tr = tw + buf * 128u;
            const float* vr = Vt + ((size_t)i * Cp + c) * P.R8 + r;
#pragma unroll 8
            for (uint32_t j = 0; j < W; ++j) acc = __fadd_rn(acc, __fmul_rn(tr[j], vr[j]));
            if (cn < d.C) {
#pragma unroll
                for (int q = 0; q < 4; ++q) tw[(buf ^ 1u) * 128u + lane + 32u * q] = tn[q];
            }
            __syncwarp();
            buf ^= 1u;
            c = cn;
        }
        const bool mine = (mask >> lane) & 1u;
        const uint32_t sk = E.t_s0[i] + r;
        if (mine) P.L[(uint64_t)t * d.N + sk] = acc;
        if (lazy) warp_note_exact(d, E, mine, acc, t, i, sk);
        __syncwarp();
    }
}

// In-place transposition of `ntq` 4-channel blocks of R8 16-byte rows into
// channel-major rows of R8 floats.  A block's rows stay within its own bytes, so
// one warp transposes a whole block (warps w0, w0 + nwarps, ...) with warp
// synchronisation only; the caller synchronises the threads afterwards.
__device__ __forceinline__ void transpose_strips(unsigned char* A, uint32_t ntq, uint32_t R8, uint32_t w0,
                                                 uint32_t nwarps)
{
    const uint32_t lane = threadIdx.x & 31;
    const float4* src = reinterpret_cast<const float4*>(A);
    float* dst = reinterpret_cast<float*>(A);
    for (uint32_t tq = w0; tq < ntq; tq += nwarps) {
        float4 vv[8];   // R8 <= 256 rows
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
            const uint32_t r = k * 32 + lane;
            vv[k] = r < R8 ? src[(size_t)tq * R8 + r] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
            const uint32_t r = k * 32 + lane;
            if (r >= R8) continue;
            float* o = dst + (size_t)4 * tq * R8 + r;
            o[0] = vv[k].x;
            o[R8] = vv[k].y;
            o[2 * R8] = vv[k].z;
            o[3 * R8] = vv[k].w;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kThreads, 4) lik_tc_kernel(TcParams P)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const Dims& d = P.d;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t strip_bytes = P.R8 * 16;                  // one 4-channel block of a tile strip
    const uint32_t tile_bytes = P.Cq * strip_bytes;
    const uint32_t kstep_bytes = P.Np * 32;                  // one (tap, channel pair) of templates
    const uint32_t stage_bytes = P.group * kstep_bytes;      // P.group consecutive k-steps per bulk copy
    unsigned char* A = smem;
    unsigned char* B = A + P.ntiles * tile_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(B + P.stages * stage_bytes);
    uint64_t* a_full = bars;
    uint64_t* acc_full = bars + 1;
    uint64_t* b_full = bars + 2;
    uint64_t* b_empty = b_full + P.stages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(b_empty + P.stages);
    uint32_t* err = tmem_slot + 1;
    uint32_t* t_s0 = err + 1;                                // [ntiles]
    uint32_t* t_rows = t_s0 + P.ntiles;                      // [ntiles]
    float* snorm = reinterpret_cast<float*>(t_rows + P.ntiles);   // [ntiles][C]
    float* bnd = snorm + P.ntiles * d.C;                          // [ntiles][M]
    float* sbias = bnd + P.ntiles * d.M;                          // [M]
    unsigned long long* fq = reinterpret_cast<unsigned long long*>(
        (reinterpret_cast<uintptr_t>(sbias + d.M) + 7) & ~(uintptr_t)7);   // [kFixCap] queued runs
    uint32_t* nfq = reinterpret_cast<uint32_t*>(fq + kFixCap);
    uint32_t* t_w0 = nfq + 1;                                      // [ntiles] first window of each tile
    int* s_mlb = reinterpret_cast<int*>(t_w0 + P.ntiles);          // [ntiles][wslots] max lower bound (float bits)
    uint32_t* s_pos = reinterpret_cast<uint32_t*>(s_mlb + P.ntiles * P.wslots);   // [ntiles][wslots]
    unsigned long long* s_key = reinterpret_cast<unsigned long long*>(
        (reinterpret_cast<uintptr_t>(s_pos + P.ntiles * P.wslots) + 7) & ~(uintptr_t)7);   // [ntiles][wslots]
    uint8_t* s_inex = reinterpret_cast<uint8_t*>(s_key + P.ntiles * P.wslots);   // [ntiles][wslots][M]

    const uint32_t ksteps = d.W * (P.Cq / 2);
    const uint32_t ngroups = (ksteps + P.group - 1) / P.group;
    if (threadIdx.x == 0) {
        mbar_init(a_full, 1);
        mbar_init(acc_full, 1);
        for (uint32_t s = 0; s < P.stages; ++s) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        *err = 0;
        *nfq = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < P.ntiles) {
        const uint32_t i = threadIdx.x;
        const uint64_t item = (uint64_t)blockIdx.x * P.ntiles + i;
        uint32_t s0 = 0, rows = 0;
        if (P.list == nullptr) {
            const uint64_t st = ((uint64_t)P.tile0 + item) * kTile;
            if (item < P.nitems && st < d.N) { s0 = (uint32_t)st; rows = (uint32_t)(d.N - st < (uint64_t)kTile ? d.N - st : (uint64_t)kTile); }
        } else if (item < P.nitems) {
            const uint64_t st = (uint64_t)P.list[item] * d.W;
            if (st < d.N) { s0 = (uint32_t)st; rows = (uint32_t)(d.N - st < (uint64_t)d.W ? d.N - st : (uint64_t)d.W); }
        }
        t_s0[i] = s0;
        t_rows[i] = rows;
        t_w0[i] = s0 / d.W;
    }
    for (uint32_t e = threadIdx.x; e < P.ntiles * P.wslots; e += blockDim.x) {
        s_mlb[e] = 0;
        s_pos[e] = 0;
        s_key[e] = 0ull;
    }
    if (P.lazy)
        for (uint32_t e = threadIdx.x; e < P.ntiles * P.wslots * d.M; e += blockDim.x) s_inex[e] = 0;
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(P.ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // voltage strips, one bulk copy per tile and 4-channel block
            mbar_expect_tx(a_full, P.ntiles * tile_bytes);
            for (uint32_t i = 0; i < P.ntiles; ++i)
                for (uint32_t q = 0; q < P.Cq; ++q)
                    bulk_g2s(A + i * tile_bytes + q * strip_bytes,
                             P.Vq + ((uint64_t)q * P.rows + t_s0[i]) * 4, strip_bytes, a_full);
            // templates, one stage per P.group consecutive (tap, channel pair) steps
            for (uint32_t g = 0; g < ngroups; ++g) {
                const uint32_t st = g % P.stages, round = g / P.stages;
                if (round > 0 && !mbar_wait(&b_empty[st], (round - 1) & 1)) { atomicOr(err, 1u); break; }
                const uint32_t k0 = g * P.group, nk = min(P.group, ksteps - k0);
                mbar_expect_tx(&b_full[st], nk * kstep_bytes);
                bulk_g2s(B + st * stage_bytes, P.Tq + (uint64_t)k0 * P.Np * 8, nk * kstep_bytes, &b_full[st]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((P.Np >> 3) << 17) | ((kTile >> 4) << 24);
            bool ok = mbar_wait(a_full, 0);
            const uint32_t a_base = smem_u32(A), b_base = smem_u32(B);
            uint32_t issued = 0;
            for (uint32_t g = 0; ok && g < ngroups; ++g) {
                const uint32_t st = g % P.stages, round = g / P.stages;
                if (!mbar_wait(&b_full[st], round & 1)) { ok = false; break; }
                tc_fence_after();
                const uint32_t k0 = g * P.group, nk = min(P.group, ksteps - k0);
                issue_ksteps(tmem, P.Np, P.ntiles, umma_desc(a_base, strip_bytes, 128), tile_bytes >> 4,
                             (2 * strip_bytes) >> 4, umma_desc(b_base + st * stage_bytes, P.Np * 16, 128),
                             kstep_bytes >> 4, k0, nk, P.Cq / 2, idesc);
                umma_commit(&b_empty[st]);
                ++issued;
            }
            if (!ok) atomicOr(err, 2u);
            umma_commit(acc_full);   // arrives once every MMA issued above has completed
        }
    } else {
        // epilogue warps 2..5
        const uint32_t et = threadIdx.x - 64;
        const bool a_ok = mbar_wait(a_full, 0);
        if (a_ok) {
            // per-tile channel norms of the voltage strip (rows [0, rows+W-1))
            for (uint32_t e = et; e < P.ntiles * d.C; e += 128) {
                const uint32_t i = e / d.C, c = e % d.C;
                const float* col = reinterpret_cast<const float*>(A + i * tile_bytes + (c / 4) * strip_bytes) + (c % 4);
                const uint32_t nr = t_rows[i] ? t_rows[i] + d.W - 1 : 0;
                float acc = 0.f;
                for (uint32_t r = 0; r < nr; ++r) acc = fmaf(col[r * 4], col[r * 4], acc);
                snorm[e] = sqrtf(acc) * 1.0001f;
            }
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");
        for (uint32_t t = et; t < d.M; t += 128) sbias[t] = P.bias[t];
        for (uint32_t e = et; e < P.ntiles * d.M; e += 128) {
            const uint32_t i = e / d.M, t = e % d.M;
            float a = 0.f;
            for (uint32_t c = 0; c < d.C; ++c) a = fmaf(P.tnorm[t * d.C + c], snorm[i * d.C + c], a);
            bnd[e] = P.k_a * a * 1.0001f + P.k_b * fabsf(P.bias[t]);
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");
        const bool acc_ok = a_ok && mbar_wait(acc_full, 0);
        tc_fence_after();
        if (!acc_ok) {
            if (et == 0) atomicOr(err, 4u);
        } else {
            const uint32_t qd = warp & 3;
            const uint32_t row = qd * 32 + lane;
            const Epi E{t_s0, t_rows, t_w0, sbias, bnd, s_mlb, s_pos, s_key, s_inex, fq, nfq, P.wslots};
            const uint32_t tbase = tmem + ((qd * 32) << 16);
            epi_pass1(P, E, tbase, P.ntiles, row, P.lazy != 0, 0u, 4u);
            if (P.lazy) {
                asm volatile("bar.sync 1, 128;" ::: "memory");
                epi_pass2(P, E, tbase, P.ntiles, row, 0u, 4u);
            }
        }
        tc_fence_before();
    }
    __syncthreads();
    if (threadIdx.x == 0 && *err) atomicOr(&P.status->error, 0x100u | *err);
    if (warp == 1) {
        // drain: the accumulator barrier completes once all issued MMAs are done
        if (lane == 0 && (*err & 4u)) mbar_wait(acc_full, 0);
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P.ncols));
    }
    // exact recomputation of this CTA's queued runs, all warps, from the strips
    // transposed in place to channel-major rows; each warp stages template rows in
    // its share of the (now idle) template ring
    const uint32_t nq = min(*nfq, kFixCap);
    if (threadIdx.x == 0 && nq) atomicAdd(&P.status->n_fix_local, nq);
    if (nq == 0 && !P.lazy) return;
    const uint32_t W = d.W;
    if (nq > 0) {
        // the strips were written by bulk copies and read by the MMAs (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        transpose_strips(A, P.ntiles * P.Cq, P.R8, warp, blockDim.x >> 5);
        __syncthreads();
        const Epi E{t_s0, t_rows, t_w0, sbias, bnd, s_mlb, s_pos, s_key, s_inex, fq, nfq, P.wslots};
        recompute_runs(P, E, reinterpret_cast<const float*>(A), nq, warp, blockDim.x >> 5,
                       reinterpret_cast<float*>(B) + warp * 256u, P.lazy != 0);
    }
    __syncthreads();
    if (!P.lazy) return;
    // publish each touched window's maximum key and positive flag: a listed window
    // belongs to this CTA alone (stored); a tile of the whole-chunk pass shares its
    // edge windows with the neighbouring tiles (combined with atomics on zeroed arrays)
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < P.ntiles * P.wslots; e += blockDim.x) {
        const uint32_t i = e / P.wslots, j = e - i * P.wslots;
        if (t_rows[i] == 0 || j > (t_s0[i] + t_rows[i] - 1) / W - t_w0[i]) continue;
        const uint32_t w = t_w0[i] + j;
        if (P.list != nullptr) {
            P.wkey[w] = s_key[e];
            P.wpos[w] = (uint8_t)(s_pos[e] ? 1 : 0);
        } else {
            if (s_key[e]) atomicMax(&P.wkey[w], s_key[e]);
            if (s_pos[e]) P.wpos[w] = 1;
        }
    }
    // estimate flags of the windows' template rows: a listed window's are all
    // written; the whole-chunk pass sets them on zeroed flags
    for (uint32_t e = threadIdx.x; e < P.ntiles * P.wslots * d.M; e += blockDim.x) {
        const uint32_t slot = e / d.M, t = e - slot * d.M;
        const uint32_t i = slot / P.wslots, j = slot - i * P.wslots;
        if (t_rows[i] == 0 || j > (t_s0[i] + t_rows[i] - 1) / W - t_w0[i]) continue;
        const uint8_t f = s_inex[e];
        if (P.list != nullptr || f) P.wflag[(uint64_t)(t_w0[i] + j) * d.M + t] = f;
    }
}

// ---------------------------------------------------------------------------
// Persistent tensor-core likelihood (the pursuit's passes, lazy exactness).
//
// One CTA per SM walks batches of B tiles.  The voltage strips and the TMEM
// accumulators are double-buffered, so while the epilogue warps finish batch k
// (estimates, bounds, window maxima, exact recomputation of the queued runs
// from the strips, window keys), the bulk-copy warp and the MMA warp already run
// batch k+1; and each pass of the template ring feeds B tiles (as many as one
// TMEM buffer of 256 columns holds) instead of one CTA's two.  NE warpgroups run
// the epilogue: warpgroup g evaluates the template groups 4g, 4g + 4 NE, ... of
// all 128 rows (each of its warps reads its TMEM lane quarter), so every SM
// sub-partition has NE epilogue warps to interleave.
//   barriers: a_full[s]   strips (and the batch's tile list) of buffer s loaded
//             a_empty[s]  the epilogue is done with buffer s's strips
//             acc_full[s] the MMAs of buffer s's batch completed (tcgen05.commit)
//             acc_empty[s] the epilogue has read TMEM buffer s
//             b_full/b_empty  the template ring, stage counter running across batches
// The results are those of lik_tc_kernel in lazy mode.
// ---------------------------------------------------------------------------
template <uint32_t N>
__device__ __forceinline__ void epi_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory");
}

// True on every epilogue thread (named barrier 1, N threads) iff p holds on all
// of them: the epilogue's loop decisions stay uniform, so no thread leaves a
// loop whose named barriers the others still wait at.
template <uint32_t N>
__device__ __forceinline__ bool epi_all(bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p), "n"(N)
        : "memory");
    return r != 0;
}

struct PersistParams {
    TcParams P;          // sizes, tensors, bounds, outputs (P.ntiles = tiles per batch)
    uint32_t nbatches;
};

constexpr uint32_t persist_threads(int ne) { return 96u + 128u * (uint32_t)ne; }

template <int NE>
__global__ void __launch_bounds__(persist_threads(NE), 1) lik_tc_persist_kernel(PersistParams Q)
{
    constexpr uint32_t EPI = 128u * NE;   // epilogue threads
    extern __shared__ __align__(1024) unsigned char smem[];
    const TcParams& P = Q.P;
    const Dims& d = P.d;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t B = P.ntiles;
    const uint32_t strip_bytes = P.R8 * 16;
    const uint32_t tile_bytes = P.Cq * strip_bytes;
    const uint32_t kstep_bytes = P.Np * 32;
    const uint32_t stage_bytes = P.group * kstep_bytes;
    unsigned char* A = smem;                                       // [2][B][tile]
    unsigned char* R = A + 2 * B * tile_bytes;                     // template ring
    uint64_t* bars = reinterpret_cast<uint64_t*>(R + P.stages * stage_bytes);
    uint64_t* a_full = bars;          // [2]
    uint64_t* a_empty = bars + 2;     // [2]
    uint64_t* acc_full = bars + 4;    // [2]
    uint64_t* acc_empty = bars + 6;   // [2]
    uint64_t* drain = bars + 8;       // [2] each MMA warp's last commit, on an error
    uint64_t* b_full = bars + 10;
    uint64_t* b_empty = b_full + P.stages;
    unsigned long long* fq = reinterpret_cast<unsigned long long*>(b_empty + P.stages);   // [kFixCap] queued runs
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fq + kFixCap);
    uint32_t* err = tmem_slot + 1;
    uint32_t* nfq = err + 1;
    uint32_t* meta = nfq + 1;                                      // [2][3][B]: s0, rows, first window
    float* snorm = reinterpret_cast<float*>(meta + 6 * B);         // [B][C]
    float* bnd = snorm + B * d.C;                                  // [B][M]
    float* sbias = bnd + B * d.M;                                  // [M]
    int* s_mlb = reinterpret_cast<int*>(sbias + d.M);              // [B][wslots]
    uint32_t* s_pos = reinterpret_cast<uint32_t*>(s_mlb + B * P.wslots);
    unsigned long long* s_key = reinterpret_cast<unsigned long long*>(
        (reinterpret_cast<uintptr_t>(s_pos + B * P.wslots) + 7) & ~(uintptr_t)7);
    uint8_t* s_inex = reinterpret_cast<uint8_t*>(s_key + B * P.wslots);   // [B][wslots][M]
    float* scratch = reinterpret_cast<float*>(
        (reinterpret_cast<uintptr_t>(s_inex + B * P.wslots * d.M) + 15) & ~(uintptr_t)15);   // [4 NE warps][256]

    const uint32_t ksteps = d.W * (P.Cq / 2);
    const uint32_t ngroups = (ksteps + P.group - 1) / P.group;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&a_full[s], 1);
            mbar_init(&a_empty[s], 1);
            mbar_init(&acc_full[s], 2);   // one commit per MMA warp
            mbar_init(&acc_empty[s], 1);
            mbar_init(&drain[s], 1);
        }
        for (uint32_t s = 0; s < P.stages; ++s) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 2);    // one commit per MMA warp
        }
        *err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (uint32_t t = threadIdx.x; t < d.M; t += blockDim.x) sbias[t] = P.bias[t];
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t gtot = 0;
            for (uint32_t batch = blockIdx.x, it = 0; batch < Q.nbatches; batch += gridDim.x, ++it) {
                const uint32_t s = it & 1, use = it >> 1;
                if (*(volatile uint32_t*)err) break;
                if (use > 0 && !mbar_wait(&a_empty[s], (use - 1) & 1)) { atomicOr(err, 1u); break; }
                uint32_t* ms0 = meta + s * 3 * B;
                uint32_t* mrows = ms0 + B;
                uint32_t* mw0 = mrows + B;
                for (uint32_t i = 0; i < B; ++i) {
                    const uint64_t item = (uint64_t)batch * B + i;
                    uint32_t s0 = 0, rows = 0;
                    if (P.list == nullptr) {
                        const uint64_t st = ((uint64_t)P.tile0 + item) * kTile;
                        if (item < P.nitems && st < d.N) { s0 = (uint32_t)st; rows = (uint32_t)(d.N - st < (uint64_t)kTile ? d.N - st : (uint64_t)kTile); }
                    } else if (item < P.nitems) {
                        const uint64_t st = (uint64_t)P.list[item] * d.W;
                        if (st < d.N) { s0 = (uint32_t)st; rows = (uint32_t)(d.N - st < (uint64_t)d.W ? d.N - st : (uint64_t)d.W); }
                    }
                    ms0[i] = s0;
                    mrows[i] = rows;
                    mw0[i] = s0 / d.W;
                }
                unsigned char* Ab = A + s * B * tile_bytes;
                mbar_expect_tx(&a_full[s], B * tile_bytes);
                for (uint32_t i = 0; i < B; ++i)
                    for (uint32_t q = 0; q < P.Cq; ++q)
                        bulk_g2s(Ab + i * tile_bytes + q * strip_bytes, P.Vq + ((uint64_t)q * P.rows + ms0[i]) * 4,
                                 strip_bytes, &a_full[s]);
                bool ok = true;
                for (uint32_t g = 0; g < ngroups; ++g, ++gtot) {
                    const uint32_t st = gtot % P.stages, round = gtot / P.stages;
                    if (round > 0 && !mbar_wait(&b_empty[st], (round - 1) & 1)) { ok = false; break; }
                    const uint32_t k0 = g * P.group, nk = min(P.group, ksteps - k0);
                    mbar_expect_tx(&b_full[st], nk * kstep_bytes);
                    bulk_g2s(R + st * stage_bytes, P.Tq + (uint64_t)k0 * P.Np * 8, nk * kstep_bytes, &b_full[st]);
                }
                if (!ok) { atomicOr(err, 1u); break; }
            }
        }
    } else if (warp == 1 || warp == 2) {
        // two MMA warps: warp 1 the batch's first (B + 1) / 2 tiles, warp 2 the others
        // (one issuing thread is limited to about one MMA per 60 cycles)
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((P.Np >> 3) << 17) | ((kTile >> 4) << 24);
            const uint32_t r_base = smem_u32(R);
            const uint32_t B1 = (B + 1) / 2, t0 = warp == 1 ? 0u : B1, ntl = warp == 1 ? B1 : B - B1;
            const uint32_t ebit = warp == 1 ? 2u : 16u;
            uint32_t gtot = 0;
            for (uint32_t batch = blockIdx.x, it = 0; batch < Q.nbatches; batch += gridDim.x, ++it) {
                const uint32_t s = it & 1, use = it >> 1;
                if (*(volatile uint32_t*)err) break;
                if (!mbar_wait(&a_full[s], use & 1)) { atomicOr(err, ebit); break; }
                if (use > 0 && !mbar_wait(&acc_empty[s], (use - 1) & 1)) { atomicOr(err, ebit); break; }
                tc_fence_after();
                const uint32_t a_base = smem_u32(A + s * B * tile_bytes) + t0 * tile_bytes;
                const uint32_t dcol = tmem + s * 256u + t0 * P.Np;
                bool ok = true;
                for (uint32_t g = 0; g < ngroups; ++g, ++gtot) {
                    const uint32_t st = gtot % P.stages, round = gtot / P.stages;
                    if (!mbar_wait(&b_full[st], round & 1)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t k0 = g * P.group, nk = min(P.group, ksteps - k0);
                    if (ntl > 0)
                        issue_ksteps(dcol, P.Np, ntl, umma_desc(a_base, strip_bytes, 128), tile_bytes >> 4,
                                     (2 * strip_bytes) >> 4, umma_desc(r_base + st * stage_bytes, P.Np * 16, 128),
                                     kstep_bytes >> 4, k0, nk, P.Cq / 2, idesc);
                    umma_commit(&b_empty[st]);
                }
                umma_commit(&acc_full[s]);   // completes once every MMA this thread issued has
                if (!ok) { atomicOr(err, ebit); break; }
            }
        }
    } else {
        const uint32_t et = threadIdx.x - 96, ew = warp - 3;   // epilogue threads and warps
        const uint32_t qd = warp & 3, row = qd * 32 + lane, grp = ew >> 2;
        for (uint32_t batch = blockIdx.x, it = 0; batch < Q.nbatches; batch += gridDim.x, ++it) {
            const uint32_t s = it & 1, use = it >> 1;
            if (!epi_all<EPI>(*(volatile uint32_t*)err == 0)) break;
            if (!epi_all<EPI>(mbar_wait(&a_full[s], use & 1))) { if (et == 0) atomicOr(err, 4u); break; }
            const uint32_t* t_s0 = meta + s * 3 * B;
            const uint32_t* t_rows = t_s0 + B;
            const uint32_t* t_w0 = t_rows + B;
            unsigned char* Ab = A + s * B * tile_bytes;
            // per-batch scratch, norms of the strips (4 threads per tile channel) and the bounds
            if (et == 0) *nfq = 0;
            for (uint32_t e = et; e < B * P.wslots; e += EPI) {
                s_mlb[e] = 0;
                s_pos[e] = 0;
                s_key[e] = 0ull;
            }
            for (uint32_t e = et; e < B * P.wslots * d.M; e += EPI) s_inex[e] = 0;
            const uint32_t nsub = B * d.C * 4;
            for (uint32_t e0 = 0; e0 < nsub; e0 += EPI) {
                const uint32_t e = e0 + et;
                float acc = 0.f;
                if (e < nsub) {
                    const uint32_t ic = e >> 2, k = e & 3u, i = ic / d.C, c = ic - i * d.C;
                    const float* col = reinterpret_cast<const float*>(Ab + i * tile_bytes + (c / 4) * strip_bytes) + (c % 4);
                    const uint32_t nr = t_rows[i] ? t_rows[i] + d.W - 1 : 0;
                    for (uint32_t r = k; r < nr; r += 4) acc = fmaf(col[r * 4], col[r * 4], acc);
                }
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                if (e < nsub && (e & 3u) == 0) snorm[e >> 2] = sqrtf(acc) * 1.0001f;
            }
            epi_sync<EPI>();
            for (uint32_t e = et; e < B * d.M; e += EPI) {
                const uint32_t i = e / d.M, t = e % d.M;
                float a = 0.f;
                for (uint32_t c = 0; c < d.C; ++c) a = fmaf(P.tnorm[t * d.C + c], snorm[i * d.C + c], a);
                bnd[e] = P.k_a * a * 1.0001f + P.k_b * fabsf(sbias[t]);
            }
            epi_sync<EPI>();
            // one poller per warp; the barrier and the fence below order the TMEM reads after it
            if (!epi_all<EPI>(lane != 0 || mbar_wait(&acc_full[s], use & 1))) { if (et == 0) atomicOr(err, 8u); break; }
            tc_fence_after();
            const uint32_t tbase = tmem + ((qd * 32) << 16) + s * 256u;
            const Epi E{t_s0, t_rows, t_w0, sbias, bnd, s_mlb, s_pos, s_key, s_inex, fq, nfq, P.wslots};
            epi_pass1(P, E, tbase, B, row, true, 4u * grp, 4u * NE);
            epi_sync<EPI>();
            epi_pass2(P, E, tbase, B, row, 4u * grp, 4u * NE);
            // TMEM buffer s read: the MMAs of batch it+2 may use it
            tc_fence_before();
            epi_sync<EPI>();
            if (et == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[s])) : "memory");
            // exact recomputation of the queued runs from buffer s's strips, transposed in
            // place to channel-major rows (the MMAs of this batch are complete)
            const uint32_t nq = min(*nfq, kFixCap);
            if (et == 0 && nq) atomicAdd(&P.status->n_fix_local, nq);
            if (nq > 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                transpose_strips(Ab, B * P.Cq, P.R8, ew, 4u * NE);
                epi_sync<EPI>();
                recompute_runs(P, E, reinterpret_cast<const float*>(Ab), nq, ew, 4u * NE, scratch + ew * 256u, true);
            }
            const uint32_t W = d.W;
            epi_sync<EPI>();
            // publish the batch's window maxima, positive flags and estimate flags
            for (uint32_t e = et; e < B * P.wslots; e += EPI) {
                const uint32_t i = e / P.wslots, j = e - i * P.wslots;
                if (t_rows[i] == 0 || j > (t_s0[i] + t_rows[i] - 1) / W - t_w0[i]) continue;
                const uint32_t w = t_w0[i] + j;
                if (P.list != nullptr) {
                    P.wkey[w] = s_key[e];
                    P.wpos[w] = (uint8_t)(s_pos[e] ? 1 : 0);
                } else {
                    if (s_key[e]) atomicMax(&P.wkey[w], s_key[e]);
                    if (s_pos[e]) P.wpos[w] = 1;
                }
            }
            for (uint32_t e = et; e < B * P.wslots * d.M; e += EPI) {
                const uint32_t slot = e / d.M, t = e - slot * d.M;
                const uint32_t i = slot / P.wslots, j = slot - i * P.wslots;
                if (t_rows[i] == 0 || j > (t_s0[i] + t_rows[i] - 1) / W - t_w0[i]) continue;
                const uint8_t f = s_inex[e];
                if (P.list != nullptr || f) P.wflag[(uint64_t)(t_w0[i] + j) * d.M + t] = f;
            }
            // strips of buffer s (written through the generic proxy by the transposition)
            // go back to the bulk copies
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            epi_sync<EPI>();
            if (et == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&a_empty[s])) : "memory");
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *err) atomicOr(&P.status->error, 0x200u | *err);
    if ((warp == 1 || warp == 2) && lane == 0 && *err) {
        // this thread's MMAs may still be in flight: a last commit arrives once all are done
        umma_commit(&drain[warp - 1]);
        mbar_wait(&drain[warp - 1], 0);
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
    }
}

// With lazy exactness, each positive exact value also enters its window's key
// and positive flag (after the likelihood kernel has published the CTA's own).
__device__ __forceinline__ void note_window(const Dims& d, unsigned long long* wkey, uint8_t* wpos, float v,
                                            uint32_t t, uint32_t s)
{
    if (wkey == nullptr || !(v > 0.f)) return;
    const uint32_t w = s / d.W;
    atomicMax(&wkey[w], window_key(v, t, s - w * d.W));
    wpos[w] = 1;
}

// Exact recomputation of the queued runs (reference order, FP32).  An entry
// is (t << 40) | (mask << 32) | s0: samples s0 + k with bit k of the 4-bit mask
// set.  A thread carries the four samples' sequential sums side by side: per 4
// taps one 16-byte template load and 4 voltage loads feed 16 multiply-adds
// (each sum still adds its products one at a time, in the reference's order).
__global__ void fixup_kernel(Dims d, const float* __restrict__ V, const float* __restrict__ T,
                             const float* __restrict__ Tp, const float* __restrict__ bias,
                             const unsigned long long* __restrict__ fix, uint32_t cap, const DevStatus* status,
                             float* L, unsigned long long* wkey, uint8_t* wpos, const float* __restrict__ tnorm)
{
    const uint32_t n = min(status->n_fix, cap);
    const uint32_t W = d.W, Wp = (W + 3) & ~3u, W4 = W & ~3u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long e = fix[i];
        const uint32_t t = (uint32_t)(e >> 40), mask = (uint32_t)(e >> 32) & 0xFu, s0 = (uint32_t)e;
        const float b = bias[t];
        if ((uint64_t)s0 + W + 3 > d.N) {   // the run reaches the end of the chunk: one sample at a time
            for (uint32_t k = 0; k < 4; ++k)
                if ((mask >> k) & 1u) {
                    const float v = exact_likelihood(d, V, T, b, t, s0 + k, tnorm);
                    L[(uint64_t)t * d.N + s0 + k] = v;
                    note_window(d, wkey, wpos, v, t, s0 + k);
                }
            continue;
        }
        float a0 = b, a1 = b, a2 = b, a3 = b;
        for (uint32_t c = 0; c < d.C; ++c) {
            if (tnorm[(uint64_t)t * d.C + c] == 0.f) continue;   // an all-zero template channel adds 0
            const float* vr = V + (uint64_t)c * d.N + s0;
            const float* tr = Tp + ((uint64_t)t * d.C + c) * Wp;
            float w0 = __ldg(vr), w1 = __ldg(vr + 1), w2 = __ldg(vr + 2);   // V[s0 + j + 0..2]
            uint32_t j = 0;
            for (; j < W4; j += 4) {
                const float4 t4 = __ldg(reinterpret_cast<const float4*>(tr + j));
                const float w3 = __ldg(vr + j + 3), w4 = __ldg(vr + j + 4), w5 = __ldg(vr + j + 5),
                            w6 = __ldg(vr + j + 6);
                a0 = __fadd_rn(a0, __fmul_rn(t4.x, w0)); a1 = __fadd_rn(a1, __fmul_rn(t4.x, w1));
                a2 = __fadd_rn(a2, __fmul_rn(t4.x, w2)); a3 = __fadd_rn(a3, __fmul_rn(t4.x, w3));
                a0 = __fadd_rn(a0, __fmul_rn(t4.y, w1)); a1 = __fadd_rn(a1, __fmul_rn(t4.y, w2));
                a2 = __fadd_rn(a2, __fmul_rn(t4.y, w3)); a3 = __fadd_rn(a3, __fmul_rn(t4.y, w4));
                a0 = __fadd_rn(a0, __fmul_rn(t4.z, w2)); a1 = __fadd_rn(a1, __fmul_rn(t4.z, w3));
                a2 = __fadd_rn(a2, __fmul_rn(t4.z, w4)); a3 = __fadd_rn(a3, __fmul_rn(t4.z, w5));
                a0 = __fadd_rn(a0, __fmul_rn(t4.w, w3)); a1 = __fadd_rn(a1, __fmul_rn(t4.w, w4));
                a2 = __fadd_rn(a2, __fmul_rn(t4.w, w5)); a3 = __fadd_rn(a3, __fmul_rn(t4.w, w6));
                w0 = w4; w1 = w5; w2 = w6;
            }
            for (; j < W; ++j) {   // remaining taps; w0..w2 hold V[s0 + j + 0..2]
                const float tv = __ldg(tr + j);
                const float w3 = __ldg(vr + j + 3);
                a0 = __fadd_rn(a0, __fmul_rn(tv, w0)); a1 = __fadd_rn(a1, __fmul_rn(tv, w1));
                a2 = __fadd_rn(a2, __fmul_rn(tv, w2)); a3 = __fadd_rn(a3, __fmul_rn(tv, w3));
                w0 = w1; w1 = w2; w2 = w3;
            }
        }
        float* Lr = L + (uint64_t)t * d.N + s0;
        if (mask & 1u) { Lr[0] = a0; note_window(d, wkey, wpos, a0, t, s0); }
        if (mask & 2u) { Lr[1] = a1; note_window(d, wkey, wpos, a1, t, s0 + 1); }
        if (mask & 4u) { Lr[2] = a2; note_window(d, wkey, wpos, a2, t, s0 + 2); }
        if (mask & 8u) { Lr[3] = a3; note_window(d, wkey, wpos, a3, t, s0 + 3); }
    }
}

// Per-window argmax from the window keys (compute_template_maximum_likelihood,
// binary_pursuit.cl:350-441): the maximum over the 3-window span of listed window
// id is the best of the maxima of windows id-1, id and id+1, compared by value,
// then template, then sample (the span's first maximum in template-major order).
// The flags and outputs are those of argmax_kernel.
__global__ void argmax_lazy_kernel(Dims d, const uint32_t* __restrict__ list, uint32_t nlist,
                                   const unsigned long long* __restrict__ wkey, const uint8_t* __restrict__ wpos,
                                   float* best_lik, uint32_t* best_lab, uint32_t* best_idx, uint8_t* check,
                                   uint8_t* orech, uint32_t* ov_idx, uint32_t* ov_lab)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nlist; k += gridDim.x * blockDim.x) {
        const uint32_t id = list[k];
        const uint64_t start = (uint64_t)id * d.W, end = start + d.W;
        if (end >= (uint64_t)d.N - d.W) continue;
        bool have = false;
        float bv = 0.f;
        uint32_t bt = 0, bs = 0;
        const uint32_t x0 = id > 0 ? id - 1 : 0;
        for (uint32_t x = x0; x <= id + 1; ++x) {   // id + 1 < nw: end + W < N
            const unsigned long long key = wkey[x];
            if (key == 0ull) continue;
            const float v = __uint_as_float((uint32_t)(key >> 32));
            const uint32_t code = 0xFFFFFFFFu - (uint32_t)key;
            const uint32_t t = code >> 10, s = x * d.W + (code & 1023u);
            if (!have || v > bv || (v == bv && (t < bt || (t == bt && s < bs)))) {
                have = true; bv = v; bt = t; bs = s;
            }
        }
        if (wpos[id]) check[id] = 1;
        uint32_t lab = best_lab[id], idx = best_idx[id];
        float bl = 0.f;
        if (have) { bl = bv; lab = bt; idx = bs; }
        orech[id] = (bl > 0.f && idx >= start && idx < end) ? 1 : 0;
        best_lik[id] = bl;
        best_lab[id] = lab;
        best_idx[id] = idx;
        ov_idx[id] = idx;
        ov_lab[id] = lab;
    }
}

// Before a pass's residual: the positive values of flagged (window, template)
// rows -- rows that may hold estimates -- of windows whose voltage the residual
// changes and which the next pass does not recompute (check == 0 once the pass's
// flags are final) are replaced by their exact values from the voltage they were
// computed on, and the flags cleared, so that every estimate left in L can later
// be made exact from the current voltage.  One CTA per
// spike of the pass; a spike at s changes the likelihood of samples (s-W, s+W).
__global__ void lazy_fix_kernel(Dims d, const float* __restrict__ V, const float* __restrict__ T,
                                const float* __restrict__ bias, const uint32_t* __restrict__ pidx,
                                const DevStatus* status, const uint8_t* __restrict__ check, float* L,
                                uint8_t* wflag, const float* __restrict__ tnorm)
{
    const uint32_t n = status->n_spikes;
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const uint64_t s = pidx[k];
        const uint64_t lo = s + 1 >= d.W ? s + 1 - d.W : 0;
        const uint64_t hi = s + d.W < d.N ? s + d.W : d.N;   // samples [lo, hi)
        for (uint64_t x = lo / d.W; x * d.W < hi && x < d.nw; ++x) {
            if (check[x] != 0) continue;   // relisted: recomputed next pass before any read
            const uint64_t a = x * d.W, b = min((uint64_t)d.N, a + d.W);
            // positive values of flagged rows may be estimates: make them exact (the
            // others are certainly <= 0 and are read for their sign only)
            for (uint64_t e = threadIdx.x; e < (uint64_t)d.M * (b - a); e += blockDim.x) {
                const uint32_t t = (uint32_t)(e / (b - a));
                const uint32_t q = (uint32_t)(a + e % (b - a));
                if (!wflag[x * d.M + t]) continue;
                float* lp = L + (uint64_t)t * d.N + q;
                if (*lp > 0.f) *lp = exact_likelihood(d, V, T, bias[t], t, q, tnorm);
            }
            __syncthreads();
            for (uint32_t t = threadIdx.x; t < d.M; t += blockDim.x) wflag[x * d.M + t] = 0;
        }
    }
}

// Vq[q][r][e] = V[4q+e][r] for r < N (zero elsewhere and for padding channels).
// Vq rows [r0, r1) of every 4-channel block (rows past N are zeros).
__global__ void voltage_pack_kernel(Dims d, const float* __restrict__ V, uint32_t Cq, uint32_t rows, uint32_t r0,
                                    uint32_t r1, float4* Vq)
{
    const uint32_t span = r1 - r0;
    const uint64_t total = (uint64_t)Cq * span;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t q = (uint32_t)(i / span), r = r0 + (uint32_t)(i % span);
        float x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t c = 4 * q + e;
            x[e] = (r < d.N && c < d.C) ? V[(uint64_t)c * d.N + r] : 0.f;
        }
        Vq[(uint64_t)q * rows + r] = make_float4(x[0], x[1], x[2], x[3]);
    }
}

// Refresh Vq on the rows touched by the spikes of a pass.
__global__ void voltage_repack_kernel(Dims d, const float* __restrict__ V, uint32_t Cq, uint32_t rows,
                                      const uint32_t* __restrict__ idx, uint32_t n, float4* Vq)
{
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const uint32_t s = idx[k];
        for (uint32_t e2 = threadIdx.x; e2 < Cq * d.W; e2 += blockDim.x) {
            const uint32_t q = e2 / d.W, r = s + e2 % d.W;
            if (r >= d.N) continue;
            float x[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t c = 4 * q + e;
                x[e] = c < d.C ? V[(uint64_t)c * d.N + r] : 0.f;
            }
            Vq[(uint64_t)q * rows + r] = make_float4(x[0], x[1], x[2], x[3]);
        }
    }
}

// Tq[j][qp][h][n][e] = T[n][(2qp+h)*4+e][j]; Tp[t][c][j] = T[t][c][j] (zero for
// j >= W); tnorm[t][c] = |T[t][c][:]|.
__global__ void template_pack_kernel(Dims d, const float* __restrict__ T, uint32_t Cq, uint32_t Np, float* Tq,
                                     float* Tp, float* tnorm, unsigned long long* tchm)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < d.M; t += gridDim.x * blockDim.x) {
        unsigned long long m = 0ull;
        for (uint32_t c = 0; c < d.C && c < 64; ++c) {
            const float* r = T + ((uint64_t)t * d.C + c) * d.W;
            bool nz = false;
            for (uint32_t j = 0; j < d.W && !nz; ++j) nz = r[j] != 0.f;
            if (nz) m |= 1ull << c;
        }
        tchm[t] = m;
    }
    const uint32_t Wp = (d.W + 3) & ~3u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (uint64_t)d.M * d.C * Wp;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(i % Wp);
        const uint64_t tc = i / Wp;
        Tp[i] = j < d.W ? T[tc * d.W + j] : 0.f;
    }
    const uint64_t total = (uint64_t)d.W * Cq * Np * 4;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t e = i % 4;
        const uint32_t n = (i / 4) % Np;
        const uint32_t qh = (uint32_t)((i / 4 / Np) % Cq);   // = 2*qp + h
        const uint32_t j = (uint32_t)(i / 4 / Np / Cq);
        const uint32_t c = qh * 4 + e;
        Tq[i] = (n < d.M && c < d.C) ? T[((uint64_t)n * d.C + c) * d.W + j] : 0.f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < d.M * d.C; i += gridDim.x * blockDim.x) {
        const float* r = T + (uint64_t)i * d.W;
        double a = 0.0;
        for (uint32_t j = 0; j < d.W; ++j) a += (double)r[j] * r[j];
        tnorm[i] = (float)(sqrt(a) * (1.0 + 1e-6));
    }
}

struct TcConfig {
    uint32_t Cq, Np, ntiles, R8, stages, ncols, group;
    size_t smem;
};

bool tc_config(const Dims& d, TcConfig* c)
{
    if (d.W > (uint32_t)kTile || d.W == 0) return false;
    const uint32_t Cp = (d.C + 7) / 8 * 8;
    c->Cq = Cp / 4;
    c->Np = (d.M + 15) / 16 * 16;
    // one MMA (cta_group::1, M = 128) takes at most 256 template columns
    if (c->Np > 256) return false;
    c->R8 = (kTile + d.W - 1 + 7) / 8 * 8;
    // two tiles per CTA up to 128 template columns: up to 64 columns four CTAs fit an
    // SM (TMEM <= 128 columns and about 54 KB of shared memory each), so one CTA's
    // epilogue overlaps the others' MMAs (measured faster than four tiles in two CTAs,
    // or one tile); above 128 columns one tile per CTA and two CTAs per SM
    c->ntiles = c->Np <= 128 ? 2 : 1;
    const fbp_tuning& tu = tuning();
    if (tu.lik_tiles >= 1 && tu.lik_tiles <= 4 && tu.lik_tiles * c->Np <= 512) c->ntiles = tu.lik_tiles;
    for (;;) {
        const uint32_t cols = c->ntiles * c->Np;
        c->ncols = 32;
        while (c->ncols < cols) c->ncols <<= 1;
        // CTAs resident on one SM must not ask for more than its 512 TMEM columns
        // together (a blocked tcgen05.alloc would wait for another CTA to finish)
        const uint32_t fit = std::min<uint32_t>(4, 512 / c->ncols);
        const size_t strips = (size_t)c->ntiles * c->Cq * c->R8 * 16;
        const size_t kstep = (size_t)c->Np * 32;
        // template stages of about 6 KB (whole k-steps), three in the ring
        c->group = tu.lik_group ? tu.lik_group : (uint32_t)std::max<size_t>(1, (6 * 1024) / kstep);
        c->stages = tu.lik_stages ? tu.lik_stages : 3;
        while (c->group > 1 && strips + c->stages * c->group * kstep > 160 * 1024) c->group >>= 1;
        // after the MMAs the ring is the exact recomputation's scratch: 6 warps x 1 KB
        while (c->stages * c->group * kstep < 6 * 1024 + 256) ++c->group;
        const size_t misc = 8 + c->ntiles * 8 + (size_t)c->ntiles * (d.C + d.M) * 4 + (size_t)d.M * 4 +
                            (size_t)kFixCap * 8 + 8 + 4 + (size_t)c->ntiles * 4 + (size_t)c->ntiles * win_slots(d.W) * (16 + d.M) + 8 +
                            1024;
        auto total = [&](uint32_t stages) { return strips + stages * c->group * kstep + (2 + 2 * stages) * 8 + misc; };
        if (c->Np > 128 && !tu.lik_group && !tu.lik_stages) {
            // above 128 columns (one tile, two CTAs per SM): two stages of as many whole
            // k-steps as keep both CTAs resident.  Fewer, larger bulk copies and barrier
            // round trips per MMA; measured on 64 channels x 200 templates: 4 k-steps x 2
            // stages 249 ms per pursuit's likelihood, against 326 ms for 2 x 3 and 478 ms
            // for 1 x 7, and 382-513 ms for shapes that leave one CTA per SM
            const size_t budget = (228 * 1024) / fit - 2 * 1024;
            c->stages = 2;
            c->group = 1;
            while (total(2) <= budget && c->group < 64) {
                ++c->group;
                if (total(2) > budget) { --c->group; break; }
            }
        } else if (fit < 4 && !tu.lik_stages) {
            // fewer CTAs share the SM: a deeper ring keeps more template bytes in flight
            const size_t budget = (228 * 1024) / fit - 2 * 1024;
            while (c->stages < 8 && total(c->stages + 1) <= budget) ++c->stages;
        }
        c->smem = total(c->stages);
        // ask for enough shared memory that at most `fit` CTAs are resident on an SM
        if (fit < 4) c->smem = std::max<size_t>(c->smem, (228 * 1024) / (fit + 1) + 1024);
        if (c->smem <= 200 * 1024) return true;
        if (c->ntiles == 1) return false;
        --c->ntiles;
    }
}

}  // namespace

bool tc_supported(const Dims& d)
{
    TcConfig c;
    return tc_config(d, &c);
}

int launch_argmax_lazy(const Dims& d, const Work& w, const uint32_t* list, uint32_t nlist, cudaStream_t st)
{
    if (nlist == 0) return FBP_OK;
    const Layout& L = *w.lay;
    count_launch();
    const uint32_t grid = std::min<uint32_t>((nlist + 255) / 256, 148 * 16);
    argmax_lazy_kernel<<<grid, 256, 0, st>>>(d, list, nlist, w.at<unsigned long long>(L.off_wkey),
                                             w.at<uint8_t>(L.off_wpos), w.best_lik(), w.best_lab(), w.best_idx(),
                                             w.check(), w.orech(), w.ov_idx(), w.ov_lab());
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_lazy_fix(const Dims& d, const Work& w, const float* V, const float* T, const float* bias,
                    uint32_t nmax, cudaStream_t st)
{
    if (nmax == 0) return FBP_OK;
    const Layout& L = *w.lay;
    count_launch();
    lazy_fix_kernel<<<std::min<uint32_t>(nmax, 148 * 16), 256, 0, st>>>(
        d, V, T, bias, w.pidx(), w.status(), w.check(), w.L(), w.at<uint8_t>(L.off_wflag),
        w.at<float>(L.off_tnorm));
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_tc_prepare_templates(const Dims& d, const Work& w, const float* T, cudaStream_t st)
{
    TcConfig c;
    if (!tc_config(d, &c)) return FBP_OK;
    const Layout& L = *w.lay;
    count_launch();
    template_pack_kernel<<<256, 256, 0, st>>>(d, T, c.Cq, c.Np, w.at<float>(L.off_tt_hi), w.at<float>(L.off_tpad),
                                              w.at<float>(L.off_tnorm), w.at<unsigned long long>(L.off_tchm));
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_tc_update_voltage(const Dims& d, const Work& w, const float* V, const uint32_t* idx, const uint32_t* win,
                             uint32_t n, bool all, cudaStream_t st)
{
    (void)win;
    TcConfig c;
    if (!tc_config(d, &c)) return FBP_OK;
    const Layout& L = *w.lay;
    float4* Vq = w.at<float4>(L.off_vt_hi);
    count_launch();
    if (all) {
        voltage_pack_kernel<<<148 * 16, 256, 0, st>>>(d, V, c.Cq, (uint32_t)L.vq_rows, 0u, (uint32_t)L.vq_rows, Vq);
    } else if (n > 0) {
        voltage_repack_kernel<<<n < 65535u ? n : 65535u, 128, 0, st>>>(d, V, c.Cq, (uint32_t)L.vq_rows, idx, n, Vq);
    }
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_tc_pack_range(const Dims& d, const Work& w, const float* V, uint64_t r0, uint64_t r1, cudaStream_t st)
{
    TcConfig c;
    if (!tc_config(d, &c) || r1 <= r0) return FBP_OK;
    const Layout& L = *w.lay;
    count_launch();
    voltage_pack_kernel<<<148 * 16, 256, 0, st>>>(d, V, c.Cq, (uint32_t)L.vq_rows, (uint32_t)r0, (uint32_t)r1,
                                                  w.at<float4>(L.off_vt_hi));
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

// Rows of the voltage a whole-chunk likelihood tile reads: tile k needs samples up to
// 128 k + 128 + W - 1 (its strip, rounded up to 8 rows).
uint64_t tc_tile_rows(const Dims& d)
{
    TcConfig c;
    return tc_config(d, &c) ? c.R8 : 0;
}

// Persistent launch shape: tiles per batch (one TMEM buffer of 256 columns), the
// deepest template ring that fits the shared memory, and the epilogue
// warpgroups.  False when one buffer holds fewer than two tiles or the caller
// asked for a tile count.
struct PersistConfig {
    uint32_t B, stages, group, ne;
    size_t smem;
};

bool persist_config(const Dims& d, const TcConfig& c, PersistConfig* p)
{
    const fbp_tuning& tu = tuning();
    if (tu.lik_tiles != 0) return false;
    // an even tile count: the two MMA warps take half each
    uint32_t B = std::min<uint32_t>(8, 256 / c.Np) & ~1u;
    if (B < 2) return false;
    const uint32_t ne = tu.lik_epi ? tu.lik_epi : 4;
    const size_t tile = (size_t)c.Cq * c.R8 * 16, kstep = (size_t)c.Np * 32;
    const uint32_t ws = win_slots(d.W);
    for (; B >= 2; B -= 2) {
        const size_t misc = 10 * 8 + (size_t)kFixCap * 8 + 12 + 6 * B * 4 + (size_t)B * (d.C + d.M) * 4 +
                            (size_t)d.M * 4 + (size_t)B * ws * 8 + 8 + (size_t)B * ws * 8 + (size_t)B * ws * d.M +
                            16 + (size_t)4 * ne * 256 * 4 + 1024;
        const size_t budget = 220 * 1024;
        auto total = [&](uint32_t st, uint32_t g) { return 2 * B * tile + st * g * kstep + 2 * st * 8 + misc; };
        // template stages of up to 16 k-steps (fewer, longer MMA runs per stage), at least
        // three in flight; then as many stages as fit
        uint32_t group = tu.lik_group ? tu.lik_group : 16;
        while (group > 1 && total(3, group) > budget) group >>= 1;
        uint32_t stages = tu.lik_stages ? tu.lik_stages : 8;
        while (stages > 2 && total(stages, group) > budget) --stages;
        if (total(stages, group) > budget) continue;
        p->B = B;
        p->stages = stages;
        p->group = group;
        p->ne = ne;
        p->smem = std::max<size_t>(total(stages, group), 116 * 1024);   // one CTA per SM (it takes all TMEM)
        return true;
    }
    return false;
}

template <int NE>
static int launch_persist(const PersistParams& Q, uint32_t grid, size_t smem, cudaStream_t st)
{
    FBP_CUDA(allow_max_dyn_smem(lik_tc_persist_kernel<NE>));
    KScope ks(&fbp_chunk_stats::ms_lik_tc, st);
    lik_tc_persist_kernel<NE><<<grid, persist_threads(NE), smem, st>>>(Q);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

int launch_likelihood_tc(const Dims& d, const Work& w, const float* V, const float* T, const float* bias,
                         const uint32_t* list, uint32_t nlist, float* Lk, bool lazy, cudaStream_t st,
                         uint64_t* n_fix_out, uint64_t tile0, uint64_t tile_count)
{
    (void)n_fix_out;
    if (nlist == 0) return FBP_OK;
    TcConfig c;
    if (!tc_config(d, &c)) return fail(FBP_E_ARG, "tensor-core likelihood not supported for these sizes");
    const Layout& L = *w.lay;
    TcParams P;
    P.d = d;
    P.V = V;
    P.T = T;
    P.Vq = w.at<float>(L.off_vt_hi);
    P.Tq = w.at<float>(L.off_tt_hi);
    P.bias = bias;
    P.tnorm = w.at<float>(L.off_tnorm);
    P.tchm = w.at<unsigned long long>(L.off_tchm);
    P.Tp = w.at<float>(L.off_tpad);
    const bool all = nlist == d.nw;
    P.list = all ? nullptr : list;
    const uint64_t tiles = ((uint64_t)d.N + kTile - 1) / kTile;
    if (all && tile0 >= tiles) return FBP_OK;
    const uint64_t items = all ? std::min<uint64_t>(tile_count, tiles - tile0) : nlist;
    P.nitems = (uint32_t)items;
    P.tile0 = all ? (uint32_t)tile0 : 0u;
    P.rows = (uint32_t)L.vq_rows;
    P.Cq = c.Cq;
    P.Np = c.Np;
    P.ntiles = c.ntiles;
    P.R8 = c.R8;
    P.stages = c.stages;
    P.ncols = c.ncols;
    P.group = c.group;
    P.L = Lk;
    P.fix = w.at<unsigned long long>(L.off_fix);
    P.fix_cap = (uint32_t)L.n_fix_cap;
    P.status = w.status();
    // |tf32 operands| rel. error < 2^-10 each -> products < 2^-9; FP32 accumulation of n terms
    // (any order, truncating) < n 2^-22; the reference's sequential float sum < (n+1) 2^-24.
    const double n = (double)d.C * d.W;
    const double u24 = 1.0 / 16777216.0;
    P.k_a = (float)(1.1 * (1.0 / 512.0 + (2.0 * n + 8.0) * 4.0 * u24 + (n + 2.0) * u24));
    P.k_b = (float)(1.1 * (n + 8.0) * 4.0 * u24);
    P.lazy = lazy ? 1u : 0u;
    P.wkey = lazy ? w.at<unsigned long long>(L.off_wkey) : nullptr;
    P.wpos = lazy ? w.at<uint8_t>(L.off_wpos) : nullptr;
    P.wflag = lazy ? w.at<uint8_t>(L.off_wflag) : nullptr;
    P.wslots = win_slots(d.W);
    if (lazy && all && tile0 == 0) {
        FBP_CUDA(cudaMemsetAsync(P.wkey, 0, (size_t)d.nw * 8, st));
        FBP_CUDA(cudaMemsetAsync(P.wpos, 0, (size_t)d.nw, st));
        FBP_CUDA(cudaMemsetAsync(P.wflag, 0, (size_t)d.nw * d.M, st));
    }
    FBP_CUDA(cudaMemsetAsync(&w.status()->n_fix, 0, 4, st));
    PersistConfig pc;
    count_launch(2);
    if (lazy && persist_config(d, c, &pc)) {
        // the pursuit's passes: persistent CTAs over batches of tiles
        PersistParams Q;
        Q.P = P;
        Q.P.ntiles = pc.B;
        Q.P.stages = pc.stages;
        Q.P.group = pc.group;
        Q.nbatches = (uint32_t)((items + pc.B - 1) / pc.B);
        int dev = 0, sms = 148;
        FBP_CUDA(cudaGetDevice(&dev));
        FBP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const uint32_t grid = std::min<uint32_t>(Q.nbatches, (uint32_t)sms);
        switch (pc.ne) {
            case 1: FBP_TRY(launch_persist<1>(Q, grid, pc.smem, st)); break;
            case 3: FBP_TRY(launch_persist<3>(Q, grid, pc.smem, st)); break;
            case 2: FBP_TRY(launch_persist<2>(Q, grid, pc.smem, st)); break;
            default: FBP_TRY(launch_persist<4>(Q, grid, pc.smem, st)); break;
        }
    } else {
        FBP_CUDA(allow_max_dyn_smem(lik_tc_kernel));
        const uint32_t grid = (uint32_t)((items + c.ntiles - 1) / c.ntiles);
        KScope ks(&fbp_chunk_stats::ms_lik_tc, st);
        lik_tc_kernel<<<grid, kThreads, c.smem, st>>>(P);
    }
    KScope ks(&fbp_chunk_stats::ms_fixup, st);
    fixup_kernel<<<148 * 8, 256, 0, st>>>(d, V, T, P.Tp, bias, P.fix, P.fix_cap, w.status(), Lk, P.wkey, P.wpos,
                                          P.tnorm);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

}  // namespace fbp
