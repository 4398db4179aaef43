// fbp_internal.cuh -- shared definitions of libfbp.so (B200, sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>
#include <string>

#include "../../include/fbp.h"

namespace fbp {

// ---------------------------------------------------------------------------
// Error reporting
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

#define FBP_CUDA(expr)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return ::fbp::fail(FBP_E_CUDA, std::string(#expr " failed: ") + cudaGetErrorString(e_)); \
    } while (0)

#define FBP_TRY(expr)                  \
    do {                               \
        int rc_ = (expr);              \
        if (rc_ != FBP_OK) return rc_; \
    } while (0)

// Every launcher sets a kernel's dynamic shared-memory limit to the largest the
// device allows for that kernel (the block opt-in maximum less the kernel's
// static shared memory): the attribute belongs to the kernel in the whole
// process, and with one value per kernel, calls on other threads that launch the
// same kernel with other sizes never lower it under a launch in flight.
template <class Kernel>
inline cudaError_t allow_max_dyn_smem(Kernel kernel)
{
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, kernel);
    if (e != cudaSuccess) return e;
    int dev = 0, optin = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes);
}

// Launch shapes chosen by the caller (fbp_set_tuning), per thread; 0 = library choice.
fbp_tuning& tuning();

// ---------------------------------------------------------------------------
// Per-call instrumentation: kernel launch counts, and (with FBP_TIMING) device
// time per kernel family.  Thread-local; set up by the C-ABI entry points.
// ---------------------------------------------------------------------------
struct KernelClock {
    fbp_chunk_stats* stats = nullptr;  // non-null: time the launches
    uint64_t launches = 0;
};
KernelClock& kclock();

inline void count_launch(uint32_t n = 1) { kclock().launches += n; }

// Times the launches issued in its scope into *acc (if timing is on).
class KScope {
  public:
    KScope(float fbp_chunk_stats::*field, cudaStream_t st);
    ~KScope();

  private:
    float* acc_ = nullptr;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    cudaStream_t st_ = nullptr;
};

// ---------------------------------------------------------------------------
// Device status word: counters the kernels of one pass publish.
// ---------------------------------------------------------------------------
struct DevStatus {
    uint32_t n_flag;        // windows flagged for the overlap recheck this pass
    uint32_t n_spikes;      // spikes accepted this pass
    uint32_t n_next;        // windows listed for the next pass
    uint32_t chain_overflow;// a prune/reassign chain was longer than the walk limit
    uint32_t error;         // nonzero: a kernel detected an inconsistent state
    uint32_t n_fix;         // runs of 4 likelihood samples queued for exact recomputation
    uint32_t n_pair_exact;  // overlap items recomputed exactly
    uint32_t n_conf;        // spikes of this pass overlapping an earlier one
    unsigned long long pair_items;  // items evaluated by the overlap recheck
    uint32_t cand_count;    // candidates appended to the exact-scoring list (per batch)
    uint32_t n_fix_local;   // runs recomputed inside the likelihood kernel (whole call)
    unsigned long long pc_macs;   // multiply-adds done by the partial correlations (whole call)
};

// ---------------------------------------------------------------------------
// Workspace layout (all offsets 256-byte aligned)
// ---------------------------------------------------------------------------
struct Layout {
    uint64_t C, N, M, W, S, WG, nw, nwf, nblk;
    size_t off_L, off_best_lik, off_best_lab, off_best_idx, off_ov_idx, off_ov_lab;
    size_t off_check, off_orech, off_orech_fin, off_list, off_list2, off_flag;
    size_t off_has, off_newval, off_pidx, off_plab, off_pwin, off_pconf, off_keys;
    size_t off_blk, off_status;
    // tensor-core likelihood (mode 1)
    size_t off_vt_hi, off_tt_hi, off_tpad, off_fix, off_tnorm, off_tchm;
    uint64_t Cp, Mp, n_fix_cap, vq_rows;
    // lazy exactness of the tensor-core likelihood: per-window maximum keys and
    // positive flags, and per (window, template) "row holds estimates" flags
    size_t off_wkey, off_wpos, off_wflag;
    // screened overlap recheck: truncated energies Et[M][S2] (f64), pair cross
    // terms XT[M][M][S2][S2] (f32), partial correlations G[gbatch][M][S2] (f32),
    // template processing order perm[M]
    size_t off_et, off_xt, off_xtt, off_g, off_order, off_perm, off_mx, off_cand, off_bscr;
    uint64_t cand_cap;
    uint64_t gbatch;
    bool screened;
    size_t bytes;
};

bool make_layout(const fbp_dims* d, uint32_t flags, Layout* L);

struct Work {
    const Layout* lay;
    unsigned char* base;
    template <class T>
    T* at(size_t off) const { return reinterpret_cast<T*>(base + off); }
    float* L() const { return at<float>(lay->off_L); }
    float* best_lik() const { return at<float>(lay->off_best_lik); }
    uint32_t* best_lab() const { return at<uint32_t>(lay->off_best_lab); }
    uint32_t* best_idx() const { return at<uint32_t>(lay->off_best_idx); }
    uint32_t* ov_idx() const { return at<uint32_t>(lay->off_ov_idx); }
    uint32_t* ov_lab() const { return at<uint32_t>(lay->off_ov_lab); }
    uint8_t* check() const { return at<uint8_t>(lay->off_check); }
    uint8_t* orech() const { return at<uint8_t>(lay->off_orech); }
    uint8_t* orech_fin() const { return at<uint8_t>(lay->off_orech_fin); }
    uint32_t* list() const { return at<uint32_t>(lay->off_list); }
    uint32_t* list2() const { return at<uint32_t>(lay->off_list2); }
    uint32_t* flag() const { return at<uint32_t>(lay->off_flag); }
    uint8_t* has() const { return at<uint8_t>(lay->off_has); }
    uint8_t* newval() const { return at<uint8_t>(lay->off_newval); }
    uint32_t* pidx() const { return at<uint32_t>(lay->off_pidx); }
    uint32_t* plab() const { return at<uint32_t>(lay->off_plab); }
    uint32_t* pwin() const { return at<uint32_t>(lay->off_pwin); }
    uint8_t* pconf() const { return at<uint8_t>(lay->off_pconf); }
    unsigned long long* keys() const { return at<unsigned long long>(lay->off_keys); }
    uint32_t* blk() const { return at<uint32_t>(lay->off_blk); }
    DevStatus* status() const { return at<DevStatus>(lay->off_status); }
};

// Where the tensor-core likelihood left estimates (lazy exactness): readers of
// a positive likelihood value recompute it exactly when its window row is flagged.
struct LazyRef {
    const uint8_t* wflag;      // [nw][M] flags, or null: L is exact wherever read
    const float* tnorm;        // [M][C] template channel norms (0: an all-zero channel, skipped)
    const float* V;
    const float* T;
    const float* bias;
};

// Sizes passed by value to kernels.
struct Dims {
    uint32_t C, N, M, W, S, WG, nw, nwf;
};

inline Dims dims_of(const Layout& l)
{
    return Dims{(uint32_t)l.C, (uint32_t)l.N, (uint32_t)l.M, (uint32_t)l.W,
                (uint32_t)l.S, (uint32_t)l.WG, (uint32_t)l.nw, (uint32_t)l.nwf};
}

// ---------------------------------------------------------------------------
// Launchers (kernels_plain.cu)
// ---------------------------------------------------------------------------
int launch_iota(uint32_t* list, uint32_t n, cudaStream_t st);
int launch_likelihood_exact(const Dims& d, const float* V, const float* T, const float* bias,
                            const uint32_t* list, uint32_t nlist, float* L, cudaStream_t st);
int launch_argmax(const Dims& d, const Work& w, const uint32_t* list, uint32_t nlist,
                  cudaStream_t st);
int launch_compact_flagged(const Dims& d, const Work& w, uint32_t nlist, cudaStream_t st);
int launch_overlap_plain(const Dims& d, const Work& w, const float* V, const float* T,
                         const float* theta, uint32_t nflag_max, cudaStream_t st);
int launch_parse_reassign(const Dims& d, const Work& w, const float* theta, uint32_t nflag_max,
                          cudaStream_t st, const float* V = nullptr, const float* T = nullptr,
                          const float* bias = nullptr, bool lazy = false);
int launch_accept(const Dims& d, const Work& w, const float* theta, uint32_t nlist,
                  cudaStream_t st);
int launch_next_list(const Dims& d, const Work& w, cudaStream_t st);
int launch_residual(const Dims& d, const Work& w, float* V, const float* T,
                    const uint32_t* idx, const uint32_t* lab, const uint32_t* win, uint32_t n,
                    cudaStream_t st);
int launch_adjusted_clips(const Dims& d, const float* V, const float* T, const uint32_t* idx,
                          const uint32_t* lab, uint32_t n, float* clips, cudaStream_t st);

// Tensor-core likelihood (lik_tc.cu)
bool tc_supported(const Dims& d);
// nlist == d.nw: the whole chunk, tiles [tile0, tile0 + tile_count) of 128 samples
int launch_likelihood_tc(const Dims& d, const Work& w, const float* V, const float* T,
                         const float* bias, const uint32_t* list, uint32_t nlist, float* L,
                         bool lazy, cudaStream_t st, uint64_t* n_fix_out, uint64_t tile0 = 0,
                         uint64_t tile_count = ~0ull);
// Vq rows [r0, r1) from the voltage; the voltage rows a whole-chunk tile's strip reads
int launch_tc_pack_range(const Dims& d, const Work& w, const float* V, uint64_t r0, uint64_t r1, cudaStream_t st);
uint64_t tc_tile_rows(const Dims& d);
// Lazy exactness: per-window argmax from the window keys, and the exact
// recomputation of estimates whose voltage the coming residual changes in
// windows the next pass does not relist.
int launch_argmax_lazy(const Dims& d, const Work& w, const uint32_t* list, uint32_t nlist, cudaStream_t st);
int launch_lazy_fix(const Dims& d, const Work& w, const float* V, const float* T, const float* bias,
                    uint32_t nmax, cudaStream_t st);
int launch_tc_prepare_templates(const Dims& d, const Work& w, const float* T, cudaStream_t st);
int launch_tc_update_voltage(const Dims& d, const Work& w, const float* V, const uint32_t* idx,
                             const uint32_t* win, uint32_t n, bool all, cudaStream_t st);

// Screened overlap recheck (overlap_fast.cu)
int launch_overlap_tables(const Dims& d, const Work& w, const float* T, cudaStream_t st);
int launch_overlap_fast(const Dims& d, const Work& w, const float* V, const float* T,
                        const float* theta, uint32_t nflag_max, cudaStream_t st);

}  // namespace fbp
