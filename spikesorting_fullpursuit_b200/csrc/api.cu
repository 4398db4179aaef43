// api.cu -- C ABI of libfbp.so and the per-chunk pursuit loop.
//
// fbp_pursue_chunk runs the loop of
// spikesorting_fullpursuit/overlap/binary_pursuit_parallel.py:907-1356 with all
// state resident on the device.  The reference copies three arrays to the host
// and back every pass and compacts window lists with np.nonzero
// (binary_pursuit_parallel.py:966-979, 1210-1251); here the lists are compacted
// on the device and the host reads one 48-byte status word per pass.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <utility>

#include "fbp_internal.cuh"

namespace fbp {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }

int fail(int status, const std::string& msg)
{
    g_err = msg;
    return status;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

fbp_tuning& tuning()
{
    static thread_local fbp_tuning t{};
    return t;
}

KernelClock& kclock()
{
    static thread_local KernelClock c;
    return c;
}

KScope::KScope(float fbp_chunk_stats::*field, cudaStream_t st) : st_(st)
{
    KernelClock& c = kclock();
    if (!c.stats) return;
    acc_ = &(c.stats->*field);
    cudaEventCreate(&ev_[0]);
    cudaEventCreate(&ev_[1]);
    cudaEventRecord(ev_[0], st_);
}

KScope::~KScope()
{
    if (!acc_) return;
    cudaEventRecord(ev_[1], st_);
    cudaEventSynchronize(ev_[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
    *acc_ += ms;
    cudaEventDestroy(ev_[0]);
    cudaEventDestroy(ev_[1]);
}

bool make_layout(const fbp_dims* d, uint32_t flags, Layout* L)
{
    if (!d || !L) return false;
    const uint64_t C = d->n_chans, N = d->n_samples, M = d->n_templates, W = d->template_len;
    const uint64_t S = d->n_max_shift, WG = d->work_group;
    if (C == 0 || M == 0 || W == 0 || N <= W || W > 1024) return false;
    if (WG == 0 || (WG & (WG - 1)) != 0 || WG > 1024) return false;
    const uint64_t S2 = 2 * S + 1;
    if (S2 * S2 * M + WG >= (1ull << 32)) return false;  // work-item ids are 32-bit in the reference
    if (N >= (1ull << 32)) return false;
    std::memset(L, 0, sizeof(*L));
    L->C = C; L->N = N; L->M = M; L->W = W; L->S = S; L->WG = WG;
    L->nw = (N + W - 1) / W;
    L->nwf = N / W;
    L->nblk = (L->nw + 1023) / 1024 + 2;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = align_up(off, 256);
        size_t o = off;
        off += bytes;
        return o;
    };
    const size_t nw = L->nw;
    L->off_L = take(M * N * 4);
    L->off_best_lik = take(nw * 4);
    L->off_best_lab = take(nw * 4);
    L->off_best_idx = take(nw * 4);
    L->off_ov_idx = take(nw * 4);
    L->off_ov_lab = take(nw * 4);
    L->off_check = take(nw);
    L->off_orech = take(nw);
    L->off_orech_fin = take(nw);
    L->off_list = take(nw * 4);
    L->off_list2 = take(nw * 4);
    L->off_flag = take(nw * 4);
    L->off_has = take(nw);
    L->off_newval = take(nw);
    L->off_pidx = take(nw * 4);
    L->off_plab = take(nw * 4);
    L->off_pwin = take(nw * 4);
    L->off_pconf = take(nw);
    L->off_keys = take(nw * 8);
    L->off_blk = take(L->nblk * 4);
    L->off_status = take(sizeof(DevStatus));
    if (!(flags & FBP_PLAIN_FP32)) {
        // tensor-core likelihood: the voltage sample-major in 4-channel rows
        // (channels padded to a multiple of 8), the templates in MMA order and
        // with taps padded to a multiple of 4, plus the queue of sample runs to
        // recompute exactly.
        L->Cp = (C + 7) / 8 * 8;
        L->Mp = (M + 15) / 16 * 16;
        L->vq_rows = N + 256 + 2 * W;
        L->off_vt_hi = take(L->vq_rows * L->Cp * 4);   // voltage as [Cp/4][rows][4] fp32
        L->off_tt_hi = take(L->Mp * W * L->Cp * 4);    // templates as [W][Cp/8][2][Mp][4] fp32
        L->off_tpad = take(M * C * ((W + 3) / 4 * 4) * 4);   // templates as [M][C][W rounded up to 4]
        L->off_tnorm = take(M * C * 4);
        L->off_tchm = take(M * 8);
        uint64_t cap = M * N / 4;
        if (cap > (32ull << 20)) cap = 32ull << 20;
        L->n_fix_cap = cap + 4096;
        L->off_fix = take(L->n_fix_cap * 8);
        L->off_wkey = take(nw * 8);
        L->off_wpos = take(nw);
        L->off_wflag = take(nw * M);
    }
    if (!(flags & FBP_PLAIN_FP32) && (flags & FBP_OVERLAP_RECHECK)) {
        const uint64_t xt = M * M * S2 * S2 * 4;
        if (xt <= (24ull << 30)) {  // larger template sets use the brute-force recheck
            L->screened = true;
            L->off_et = take(M * S2 * 8);
            L->off_xt = take(xt);
            L->off_xtt = take(xt);                      // the same table transposed: XTT[f][t][b][a]
            uint64_t per = M * S2 * 4;
            uint64_t gb = (1ull << 30) / per;
            if (gb < 256) gb = 256;
            if (gb > L->nw) gb = L->nw;
            L->gbatch = gb;
            L->off_g = take(gb * per);
            L->off_order = take(gb * 4);                // screening order of a batch (by best label)
            L->off_perm = take(M * 4 + 8 + M * 8);      // order, then (8-aligned) non-zero channel masks
            L->off_mx = take(M * M * 4 + 2 * M * 4);   // max -X_ft per pair; max sqrt(E), max E per template
            L->cand_cap = 16ull << 20;                  // exact-scoring candidates per batch
            L->off_cand = take(L->cand_cap * 8);
            // screening tables of each persistent screen CTA when they exceed shared memory
            L->off_bscr = (M * S2 * 8 > 96 * 1024) ? take(296 * M * S2 * 8) : 0;
        }
    }
    L->bytes = align_up(off, 256);
    return true;
}

namespace api_detail {

struct StageTimer {
    bool on = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    float* acc = nullptr;
    void start(bool enable, cudaStream_t s, float* a)
    {
        on = enable;
        st = s;
        acc = a;
        if (!on) return;
        cudaEventCreate(&ev[0]);
        cudaEventCreate(&ev[1]);
        cudaEventRecord(ev[0], st);
    }
    void stop()
    {
        if (!on) return;
        cudaEventRecord(ev[1], st);
        cudaEventSynchronize(ev[1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        *acc += ms;
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        on = false;
    }
};

}  // namespace api_detail

}  // namespace fbp

using namespace fbp;

extern "C" int fbp_abi_version(void) { return FBP_ABI_VERSION; }

extern "C" const char* fbp_last_error(void) { return g_err.c_str(); }

extern "C" int fbp_set_tuning(const fbp_tuning* t)
{
    g_err.clear();
    if (t == nullptr) {
        tuning() = fbp_tuning{};
        return FBP_OK;
    }
    if (t->lik_tiles > 4 || t->lik_epi > 4 || (t->lik_stages != 0 && (t->lik_stages < 2 || t->lik_stages > 8)) ||
        (t->pc_group != 0 && t->pc_group != 1 && t->pc_group != 2 && t->pc_group != 4 && t->pc_group != 8) ||
        t->lik_group > 64)
        return fail(FBP_E_ARG, "tuning value out of range");
    tuning() = *t;
    return FBP_OK;
}

extern "C" size_t fbp_workspace_bytes(const fbp_dims* dims, uint32_t flags)
{
    Layout L;
    if (!make_layout(dims, flags, &L)) return 0;
    return L.bytes;
}

namespace {

// Voltage ranges arriving on the device (fbp_pursue_chunk_staged); n == 0: all present.
struct Ready {
    void* const* events = nullptr;
    const uint32_t* upto = nullptr;
    const uint32_t* flags = nullptr;
    uint32_t n = 0;
};

// Host wait until the uploader has recorded event k, then the stream waits for it.
int wait_ready(const Ready& R, uint32_t k, cudaStream_t st)
{
    if (R.flags) {
        const auto t0 = std::chrono::steady_clock::now();
        while (__atomic_load_n(&R.flags[k], __ATOMIC_ACQUIRE) == 0u) {
            if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(120))
                return fail(FBP_E_ARG, "voltage range " + std::to_string(k) + " was never marked ready");
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
    FBP_CUDA(cudaStreamWaitEvent(st, static_cast<cudaEvent_t>(R.events[k]), 0));
    return FBP_OK;
}

int pursue_chunk(const fbp_dims* dims, uint32_t flags, float* voltage, const float* templates, const float* bias,
                 const float* theta, void* workspace, size_t workspace_bytes, uint32_t* spike_idx,
                 uint32_t* spike_lab, uint32_t capacity, uint32_t* n_spikes, fbp_chunk_stats* stats,
                 int32_t max_passes, const Ready& ready, void* stream)
{
    g_err.clear();
    Layout lay;
    if (!make_layout(dims, flags, &lay)) return fail(FBP_E_ARG, "invalid dims");
    if (ready.n > 0) {
        if (!ready.events || !ready.upto) return fail(FBP_E_ARG, "null ready-range argument");
        for (uint32_t k = 0; k < ready.n; ++k) {
            if (!ready.events[k]) return fail(FBP_E_ARG, "null ready event");
            if ((k > 0 && ready.upto[k] <= ready.upto[k - 1]) || ready.upto[k] > lay.N)
                return fail(FBP_E_ARG, "ready ranges must increase up to n_samples");
        }
        if (ready.upto[ready.n - 1] != lay.N) return fail(FBP_E_ARG, "the last ready range must end at n_samples");
    }
    if (!voltage || !templates || !bias || !theta || !workspace || !n_spikes)
        return fail(FBP_E_ARG, "null pointer argument");
    if (capacity > 0 && (!spike_idx || !spike_lab)) return fail(FBP_E_ARG, "null spike output");
    if (workspace_bytes < lay.bytes) return fail(FBP_E_WORKSPACE, "workspace too small");
    const bool plain = (flags & FBP_PLAIN_FP32) != 0;
    const bool overlap = (flags & FBP_OVERLAP_RECHECK) != 0;
    const bool timing = (flags & 0x4u) != 0;
    const bool use_tc = !plain && tc_supported(dims_of(lay));
    // tensor-core likelihood with lazy exactness: estimates kept where no
    // decision needs the exact value (see lik_tc.cu)
    const bool lazy = use_tc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fbp_chunk_stats local{};
    fbp_chunk_stats& S = stats ? *stats : local;
    std::memset(&S, 0, sizeof(S));
    kclock().stats = timing ? &S : nullptr;
    kclock().launches = 0;
    struct ClockReset {
        ~ClockReset() { kclock().stats = nullptr; }
    } clock_reset;
    Layout cur = lay;
    Work w{&cur, static_cast<unsigned char*>(workspace)};
    const Dims d = dims_of(lay);
    cudaEvent_t t_begin = nullptr, t_end = nullptr;
    if (timing) {
        FBP_CUDA(cudaEventCreate(&t_begin));
        FBP_CUDA(cudaEventCreate(&t_end));
        FBP_CUDA(cudaEventRecord(t_begin, st));
    }
    // per-window state starts at zero (binary_pursuit_parallel.py:595-654)
    FBP_CUDA(cudaMemsetAsync(w.base + lay.off_best_lik, 0, lay.off_list - lay.off_best_lik, st));
    FBP_CUDA(cudaMemsetAsync(w.status(), 0, sizeof(DevStatus), st));
    FBP_TRY(launch_iota(w.list(), d.nw, st));
    if (use_tc) {
        FBP_TRY(launch_tc_prepare_templates(d, w, templates, st));
        if (ready.n == 0) FBP_TRY(launch_tc_update_voltage(d, w, voltage, nullptr, nullptr, 0, true, st));
    }
    if (lazy) FBP_CUDA(cudaMemsetAsync(w.base + lay.off_wflag, 0, lay.nw * lay.M, st));
    if (!plain && overlap) FBP_TRY(launch_overlap_tables(d, w, templates, st));
    uint32_t nlist = d.nw, total = 0;
    api_detail::StageTimer tm;
    for (int32_t pass = 1;; ++pass) {
        if (max_passes > 0 && pass > max_passes) {
            S.n_spikes = total;
            S.launches = kclock().launches;
            *n_spikes = total;
            return fail(FBP_E_PASSES, "pass limit reached: pass " + std::to_string(max_passes) +
                                          " still added spikes (" + std::to_string(total) + " so far)");
        }
        S.passes = pass;
        S.listed += nlist;
        FBP_CUDA(cudaMemsetAsync(&w.status()->chain_overflow, 0, 8, st));
        tm.start(timing, st, &S.ms_likelihood);
        if (pass == 1 && ready.n > 0) {
            // first pass behind the upload: each arrived range is packed and the
            // tiles whose strips it completes are pursued
            const uint64_t R8 = use_tc ? tc_tile_rows(d) : 0, ntile = (lay.N + 127) / 128;
            uint64_t packed = 0, tdone = 0;
            for (uint32_t k = 0; k < ready.n; ++k) {
                FBP_TRY(wait_ready(ready, k, st));
                if (!use_tc) continue;
                const bool last = k + 1 == ready.n;
                const uint64_t r1 = last ? lay.vq_rows : ready.upto[k];
                FBP_TRY(launch_tc_pack_range(d, w, voltage, packed, r1, st));
                packed = r1;
                const uint64_t tready = last ? ntile : (r1 >= R8 ? (r1 - R8) / 128 + 1 : 0);
                if (tready > tdone) {
                    uint64_t nfix = 0;
                    FBP_TRY(launch_likelihood_tc(d, w, voltage, templates, bias, w.list(), nlist, w.L(), lazy, st,
                                                 &nfix, tdone, tready - tdone));
                    tdone = tready;
                }
            }
            if (!use_tc) FBP_TRY(launch_likelihood_exact(d, voltage, templates, bias, w.list(), nlist, w.L(), st));
        } else if (use_tc) {
            uint64_t nfix = 0;
            FBP_TRY(launch_likelihood_tc(d, w, voltage, templates, bias, w.list(), nlist, w.L(), lazy, st, &nfix));
        } else {
            FBP_TRY(launch_likelihood_exact(d, voltage, templates, bias, w.list(), nlist, w.L(), st));
        }
        tm.stop();
        tm.start(timing, st, &S.ms_argmax);
        if (lazy)
            FBP_TRY(launch_argmax_lazy(d, w, w.list(), nlist, st));
        else
            FBP_TRY(launch_argmax(d, w, w.list(), nlist, st));
        tm.stop();
        tm.start(timing, st, &S.ms_overlap);
        if (overlap) {
            FBP_TRY(launch_compact_flagged(d, w, nlist, st));
            if (plain)
                FBP_TRY(launch_overlap_plain(d, w, voltage, templates, theta, nlist, st));
            else
                FBP_TRY(launch_overlap_fast(d, w, voltage, templates, theta, nlist, st));
            FBP_TRY(launch_parse_reassign(d, w, theta, nlist, st, voltage, templates, bias, lazy));
        }
        tm.stop();
        tm.start(timing, st, &S.ms_accept);
        FBP_TRY(launch_accept(d, w, theta, nlist, st));
        if (lazy) FBP_TRY(launch_lazy_fix(d, w, voltage, templates, bias, nlist, st));
        FBP_TRY(launch_next_list(d, w, st));
        tm.stop();
        DevStatus hs;
        FBP_CUDA(cudaMemcpyAsync(&hs, w.status(), sizeof(hs), cudaMemcpyDeviceToHost, st));
        FBP_CUDA(cudaStreamSynchronize(st));
        if (hs.error) return fail(FBP_E_DEVICE, "device status error " + std::to_string(hs.error));
        if (overlap) S.flagged += hs.n_flag;
        S.fixups += 4ull * hs.n_fix;   // runs of 4 samples
        S.fixup_runs_queued += hs.n_fix;
        const uint32_t n = hs.n_spikes;
        S.pass_spikes[(pass - 1) % FBP_PASS_RING] = n;
        if (n == 0) break;
        if ((uint64_t)total + n > capacity) {
            S.n_spikes = total;
            *n_spikes = total + n;   // at least this many outputs are needed
            return fail(FBP_E_CAPACITY, "spike capacity exceeded");
        }
        FBP_CUDA(cudaMemcpyAsync(spike_idx + total, w.pidx(), (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
        FBP_CUDA(cudaMemcpyAsync(spike_lab + total, w.plab(), (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
        FBP_CUDA(cudaMemsetAsync(w.orech(), 0, d.nw, st));
        tm.start(timing, st, &S.ms_residual);
        FBP_TRY(launch_residual(d, w, voltage, templates, w.pidx(), w.plab(), w.pwin(), n, st));
        if (use_tc) FBP_TRY(launch_tc_update_voltage(d, w, voltage, w.pidx(), w.pwin(), n, false, st));
        tm.stop();
        total += n;
        std::swap(cur.off_list, cur.off_list2);
        nlist = hs.n_next;
    }
    if (timing) {
        FBP_CUDA(cudaEventRecord(t_end, st));
        FBP_CUDA(cudaEventSynchronize(t_end));
        FBP_CUDA(cudaEventElapsedTime(&S.ms_total, t_begin, t_end));
        cudaEventDestroy(t_begin);
        cudaEventDestroy(t_end);
    }
    DevStatus hs;
    FBP_CUDA(cudaMemcpyAsync(&hs, w.status(), sizeof(hs), cudaMemcpyDeviceToHost, st));
    FBP_CUDA(cudaStreamSynchronize(st));
    S.pair_exact = (plain || !lay.screened) ? hs.pair_items : hs.n_pair_exact;
    S.fixups += 4ull * hs.n_fix_local;
    S.pc_macs = hs.pc_macs;
    S.n_spikes = total;
    S.launches = kclock().launches;
    *n_spikes = total;
    return FBP_OK;
}

}  // namespace

extern "C" int fbp_pursue_chunk(const fbp_dims* dims, uint32_t flags, float* voltage,
                                const float* templates, const float* bias, const float* theta,
                                void* workspace, size_t workspace_bytes, uint32_t* spike_idx,
                                uint32_t* spike_lab, uint32_t capacity, uint32_t* n_spikes,
                                fbp_chunk_stats* stats, int32_t max_passes, void* stream)
{
    return pursue_chunk(dims, flags, voltage, templates, bias, theta, workspace, workspace_bytes, spike_idx,
                        spike_lab, capacity, n_spikes, stats, max_passes, Ready{}, stream);
}

extern "C" int fbp_pursue_chunk_staged(const fbp_dims* dims, uint32_t flags, float* voltage,
                                       const float* templates, const float* bias, const float* theta,
                                       void* workspace, size_t workspace_bytes, uint32_t* spike_idx,
                                       uint32_t* spike_lab, uint32_t capacity, uint32_t* n_spikes,
                                       fbp_chunk_stats* stats, int32_t max_passes, void* const* ready_events,
                                       const uint32_t* ready_upto, const uint32_t* ready_flags, uint32_t n_ready,
                                       void* stream)
{
    if (n_ready == 0) {
        g_err.clear();
        return fail(FBP_E_ARG, "no ready ranges");
    }
    Ready r;
    r.events = ready_events;
    r.upto = ready_upto;
    r.flags = ready_flags;
    r.n = n_ready;
    return pursue_chunk(dims, flags, voltage, templates, bias, theta, workspace, workspace_bytes, spike_idx,
                        spike_lab, capacity, n_spikes, stats, max_passes, r, stream);
}

extern "C" int fbp_adjusted_clips(const fbp_dims* dims, const float* residual, const float* templates,
                                  const uint32_t* spike_idx, const uint32_t* spike_lab, uint32_t n,
                                  float* clips, void* stream)
{
    g_err.clear();
    Layout lay;
    if (!make_layout(dims, FBP_PLAIN_FP32, &lay)) return fail(FBP_E_ARG, "invalid dims");
    if (n == 0) return FBP_OK;
    if (!residual || !templates || !spike_idx || !spike_lab || !clips) return fail(FBP_E_ARG, "null pointer argument");
    return launch_adjusted_clips(dims_of(lay), residual, templates, spike_idx, spike_lab, n, clips,
                                 static_cast<cudaStream_t>(stream));
}

extern "C" int fbp_likelihood(const fbp_dims* dims, int mode, const float* voltage, const float* templates,
                              const float* bias, const uint32_t* windows, uint32_t n_windows,
                              float* likelihood, void* workspace, size_t workspace_bytes, void* stream)
{
    g_err.clear();
    Layout lay;
    const uint32_t flags = mode == 0 ? FBP_PLAIN_FP32 : 0u;
    if (!make_layout(dims, flags, &lay)) return fail(FBP_E_ARG, "invalid dims");
    if (!voltage || !templates || !bias || !likelihood || !workspace) return fail(FBP_E_ARG, "null pointer argument");
    if (workspace_bytes < lay.bytes) return fail(FBP_E_WORKSPACE, "workspace too small");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Work w{&lay, static_cast<unsigned char*>(workspace)};
    const Dims d = dims_of(lay);
    const uint32_t* list = windows;
    uint32_t nlist = n_windows;
    if (!windows) {
        FBP_TRY(launch_iota(w.list(), d.nw, st));
        list = w.list();
        nlist = d.nw;
    }
    if (mode != 0 && tc_supported(d)) {
        FBP_CUDA(cudaMemsetAsync(w.status(), 0, sizeof(DevStatus), st));
        FBP_TRY(launch_tc_prepare_templates(d, w, templates, st));
        FBP_TRY(launch_tc_update_voltage(d, w, voltage, nullptr, nullptr, 0, true, st));
        uint64_t nfix = 0;
        return launch_likelihood_tc(d, w, voltage, templates, bias, list, nlist, likelihood, false, st, &nfix);
    }
    return launch_likelihood_exact(d, voltage, templates, bias, list, nlist, likelihood, st);
}

namespace fbp {
namespace api_kernels {
__global__ void window_of_kernel(const uint32_t* idx, uint32_t n, uint32_t W, uint32_t* win)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) win[i] = idx[i] / W;
}
}  // namespace api_kernels
}  // namespace fbp

extern "C" int fbp_residual(const fbp_dims* dims, float* voltage, const float* templates,
                            const uint32_t* spike_idx, const uint32_t* spike_lab, uint32_t n,
                            void* workspace, size_t workspace_bytes, void* stream)
{
    g_err.clear();
    Layout lay;
    if (!make_layout(dims, FBP_PLAIN_FP32, &lay)) return fail(FBP_E_ARG, "invalid dims");
    if (n == 0) return FBP_OK;
    if (!voltage || !templates || !spike_idx || !spike_lab || !workspace) return fail(FBP_E_ARG, "null pointer argument");
    if (workspace_bytes < lay.bytes) return fail(FBP_E_WORKSPACE, "workspace too small");
    if (n > lay.nw) return fail(FBP_E_ARG, "more spikes than windows in the chunk");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Work w{&lay, static_cast<unsigned char*>(workspace)};
    const Dims d = dims_of(lay);
    fbp::api_kernels::window_of_kernel<<<(n + 255) / 256, 256, 0, st>>>(spike_idx, n, d.W, w.pwin());
    FBP_CUDA(cudaGetLastError());
    return launch_residual(d, w, voltage, templates, spike_idx, spike_lab, w.pwin(), n, st);
}
