/*
 * fbp.h -- C ABI of libfbp.so, the B200 (sm_100a) binary-pursuit library.
 *
 * Plain pointers and sizes only.  Device pointers are CUDA global-memory
 * addresses on the current device; `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream).  No call allocates device memory: the caller
 * owns every buffer, including the workspace sized by fbp_workspace_bytes().
 * Every call returns an fbp_status; the text of the last error of the calling
 * thread is available from fbp_last_error().
 *
 * Layouts (identical to the reference kernels,
 * spikesorting_fullpursuit/kernels/binary_pursuit.cl:11-29):
 *   voltage    float32 [C][N]     channel-major, N samples per channel
 *   templates  float32 [M][C][W]  W samples per channel, channel-major per template
 *   likelihood float32 [M][N]
 */
#ifndef FBP_H
#define FBP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FBP_ABI_VERSION 4

typedef enum fbp_status {
    FBP_OK = 0,
    FBP_E_ARG = -1,        /* bad shape, null pointer or size */
    FBP_E_WORKSPACE = -2,  /* workspace smaller than fbp_workspace_bytes() */
    FBP_E_CAPACITY = -3,   /* more spikes than the output capacity */
    FBP_E_PASSES = -4,     /* pass limit reached before convergence */
    FBP_E_CUDA = -5,       /* a CUDA call failed; see fbp_last_error() */
    FBP_E_DEVICE = -6      /* a kernel reported an error status word */
} fbp_status;

/* Option bits of fbp_pursue_chunk. */
#define FBP_OVERLAP_RECHECK 0x1u  /* sort_info["do_overlap_recheck"] */
#define FBP_PLAIN_FP32      0x2u  /* plain FP32 kernels: scalar likelihood, brute-force recheck */

/* Sizes of one chunk of the pursuit. */
typedef struct fbp_dims {
    uint32_t n_chans;      /* C */
    uint32_t n_samples;    /* N, samples per channel in the chunk (> W) */
    uint32_t n_templates;  /* M */
    uint32_t template_len; /* W, samples per channel of a template (window length) */
    uint32_t n_max_shift;  /* S, n_max_shift_inds of the overlap recheck */
    uint32_t work_group;   /* work-group size whose order the results follow (power of two, 256) */
} fbp_dims;

/* Passes whose spike counts fbp_chunk_stats keeps. */
#define FBP_PASS_RING 64

/* Counters of one fbp_pursue_chunk call. */
typedef struct fbp_chunk_stats {
    int32_t passes;          /* pursuit passes run (the last one adds no spike) */
    uint32_t n_spikes;       /* spikes written */
    uint64_t listed;         /* windows whose likelihood was (re)computed, summed over passes */
    uint64_t flagged;        /* windows given to the overlap recheck, summed over passes */
    uint64_t fixups;         /* likelihood samples recomputed exactly after the tensor-core product
                                (4 per queued run of consecutive samples) */
    uint64_t pair_exact;     /* overlap items whose pair likelihood was computed exactly */
    float ms_likelihood;     /* device time per stage, summed over passes (0 unless timing) */
    float ms_argmax;
    float ms_overlap;
    float ms_accept;
    float ms_residual;
    float ms_total;
    /* device time per kernel family, summed over passes (0 unless timing) */
    float ms_lik_tc;         /* tensor-core likelihood */
    float ms_fixup;          /* exact recomputation of queued likelihood samples */
    float ms_lik_exact;      /* plain FP32 likelihood */
    float ms_partial_corr;   /* partial correlations of the screened recheck */
    float ms_screen;         /* screening of the recheck items */
    float ms_score;          /* exact scoring of the recheck candidates */
    float ms_overlap_plain;  /* brute-force recheck */
    uint32_t fixup_runs_queued; /* runs recomputed by the separate fixup kernel (the others inside
                                   the likelihood kernel, from its staged voltage) */
    uint64_t launches;       /* kernels launched by the call */
    uint64_t pc_macs;        /* multiply-adds the screened recheck's partial correlations did */
    /* spikes added by each pass: pass p (1-based) at [(p - 1) % FBP_PASS_RING], so
       after more than FBP_PASS_RING passes the ring holds the most recent ones */
    uint32_t pass_spikes[FBP_PASS_RING];
} fbp_chunk_stats;

/* Option bit: record per-stage and per-kernel device times in the stats
 * (serialises the stream around each timed launch; for profiling). */
#define FBP_TIMING 0x4u

/* Launch shapes of the tensor-core likelihood and of the screened recheck's
 * partial correlations; 0 leaves a choice to the library.  Values the sizes do
 * not allow (shared memory, TMEM) fall back to the library's choice. */
typedef struct fbp_tuning {
    uint32_t lik_tiles;    /* 128-sample tiles per likelihood CTA: 1 to 4 */
    uint32_t lik_group;    /* (tap, channel pair) steps of templates per staged copy */
    uint32_t lik_stages;   /* staged template copies in flight: 2 to 8 */
    uint32_t pc_group;     /* templates per partial-correlation CTA: 1, 2, 4 or 8 */
    uint32_t lik_epi;      /* epilogue warpgroups of the persistent likelihood CTA: 1 to 4 */
} fbp_tuning;

/* Set the calling thread's launch shapes for its later calls (NULL: the
 * library's choices).  No counterpart in the reference (its work-group sizes are
 * the device's preferred ones, binary_pursuit_parallel.py:577-582). */
int fbp_set_tuning(const fbp_tuning* tuning);

/* Library ABI version (FBP_ABI_VERSION). */
int fbp_abi_version(void);

/* Text of the last error on the calling thread ("" if none). */
const char* fbp_last_error(void);

/* Bytes of device workspace fbp_pursue_chunk needs for these sizes and flags.
 * Returns 0 for invalid sizes. */
size_t fbp_workspace_bytes(const fbp_dims* dims, uint32_t flags);

/* One chunk of binary pursuit: the loop of
 * spikesorting_fullpursuit/overlap/binary_pursuit_parallel.py:907-1356 with the
 * kernels compute_full_likelihood, compute_template_maximum_likelihood,
 * overlap_recheck_indices, parse_overlap_recheck_indices,
 * check_overlap_reassignments, binary_pursuit and compute_residual
 * (binary_pursuit.cl:57-1063), run on the device until a pass adds no spike.
 *   voltage   in: the chunk's voltage; out: the residual (spikes subtracted)
 *   bias      float32[M], -0.5*template_SS (binary_pursuit_parallel.py:258)
 *   theta     float32[M], neuron_lower_thresholds (binary_pursuit_parallel.py:262)
 *   spike_idx, spike_lab  uint32[capacity]: spike onsets (chunk-relative) and
 *             template rows, pass by pass, each pass in window order
 *   n_spikes  host out: number of spikes written; after FBP_E_CAPACITY, a lower
 *             bound of the capacity the chunk needs (the voltage is then partly
 *             pursued: restore it before a retry)
 *   stats     host out, may be NULL
 *   max_passes  0 = no limit; otherwise the call fails with FBP_E_PASSES when pass
 *             max_passes still adds spikes (stats then hold the counters so far,
 *             including the spikes of the recent passes).  The reference's own
 *             loop has no limit (binary_pursuit_parallel.py:907); every pass adds
 *             at least one spike, so a pursuit of N samples and window W ends
 *             within ceil(N/W) * (spikes per window) passes.
 * The call synchronises with `stream` once per pass to read the pass's spike
 * count. */
int fbp_pursue_chunk(const fbp_dims* dims, uint32_t flags, float* voltage,
                     const float* templates, const float* bias, const float* theta,
                     void* workspace, size_t workspace_bytes,
                     uint32_t* spike_idx, uint32_t* spike_lab, uint32_t capacity,
                     uint32_t* n_spikes, fbp_chunk_stats* stats, int32_t max_passes,
                     void* stream);

/* fbp_pursue_chunk for a voltage that is still arriving on the device: the
 * first pass's packing and likelihood run range by range behind the upload.
 * ready_events[k] (a cudaEvent_t) completes once samples [0, ready_upto[k]) of
 * every channel are in `voltage`; ready_flags[k] turns non-zero (written by the
 * uploading host thread, read here with acquire ordering) once that event has
 * been recorded, and this call waits on the host for it (at most 120 s, then
 * FBP_E_ARG) before making `stream` wait for the event.  ready_upto strictly
 * increasing, the last equal to n_samples.  Results are those of
 * fbp_pursue_chunk.  No counterpart in the reference, whose host code uploads
 * the whole chunk before its first kernel (binary_pursuit_parallel.py:611-616). */
int fbp_pursue_chunk_staged(const fbp_dims* dims, uint32_t flags, float* voltage,
                            const float* templates, const float* bias, const float* theta,
                            void* workspace, size_t workspace_bytes,
                            uint32_t* spike_idx, uint32_t* spike_lab, uint32_t capacity,
                            uint32_t* n_spikes, fbp_chunk_stats* stats, int32_t max_passes,
                            void* const* ready_events, const uint32_t* ready_upto,
                            const uint32_t* ready_flags, uint32_t n_ready, void* stream);

/* Adjusted clips: clips[k][c][j] = residual[c][idx_k + j] + templates[lab_k][c][j]
 * for idx_k + j < N, else left untouched (get_adjusted_clips,
 * binary_pursuit.cl:1088-1130).  clips is float32 [n][C*W]. */
int fbp_adjusted_clips(const fbp_dims* dims, const float* residual, const float* templates,
                       const uint32_t* spike_idx, const uint32_t* spike_lab, uint32_t n,
                       float* clips, void* stream);

/* Likelihood of the listed windows (compute_full_likelihood,
 * binary_pursuit.cl:255-300): L[t][s] = bias[t] + sum_c sum_j T[t][c][j] V[c][s+j]
 * for s in [w*W, min((w+1)*W, N)), 0 where s+W >= N.  windows = NULL means all
 * ceil(N/W) windows.  mode 0: plain FP32 kernel; mode 1: tensor-core estimate
 * with exact FP32 recomputation of every sample that can be positive.  Both
 * give the reference's float32 result wherever it is > 0 and a value <= 0
 * wherever it is <= 0 (mode 0 is bit-exact everywhere).  workspace: as for
 * fbp_pursue_chunk (same dims, flags 0). */
int fbp_likelihood(const fbp_dims* dims, int mode, const float* voltage, const float* templates,
                   const float* bias, const uint32_t* windows, uint32_t n_windows, float* likelihood,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Residual subtraction of n spikes in order (compute_residual,
 * binary_pursuit.cl:57-102): voltage[c][idx_k + j] -= templates[lab_k][c][j].
 * Spikes whose ranges overlap are applied in list order. */
int fbp_residual(const fbp_dims* dims, float* voltage, const float* templates,
                 const uint32_t* spike_idx, const uint32_t* spike_lab, uint32_t n,
                 void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free residual subtraction.  No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc at all, such as a plug-in running
 * inside an acquisition or visualisation host that owns every byte of device
 * memory and forbids allocation while data stream, so it cannot hand this library
 * the workspace fbp_residual needs.  Same contract and results as fbp_residual;
 * the per-spike scratch (window ids, overlap flags, a counter) lives in one
 * file-scope static device array sized for FBP_NOALLOC_MAX_SPIKES spikes (about
 * 320 KB), which every GPU that loads the library holds until the process exits.
 *   - n > FBP_NOALLOC_MAX_SPIKES fails with FBP_E_ARG before any device work.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 *   - Every call shares the one array, which keeps the last call's contents:
 *     calls whose work overlaps on the GPU (other streams or threads without
 *     ordering between them) race on it and must be serialised by the caller.
 * It allocates no device memory and calls no allocating routine. */
#define FBP_NOALLOC_MAX_SPIKES 65536u
int fbp_residual_noalloc(const fbp_dims* dims, float* voltage, const float* templates,
                         const uint32_t* spike_idx, const uint32_t* spike_lab, uint32_t n,
                         void* stream);

/* Residual energy of a fixed spike assignment, for template refinement (no
 * counterpart in the reference):
 *   E = sum_{c,x} (v[c][x] - sum_k a_k T~_k[c][x - s_k])^2
 * with spike k at onset s_k = spike_idx[k] (ascending), template spike_lab[k],
 * amplitude a_k = amplitude[k] and fractional shift tau_k = shift[k] in (-1, 1)
 * samples: T~(c, j) = (1-|tau|) T[c][j] + |tau| T[c][j + dir], dir = -1 for
 * tau >= 0 and +1 for tau < 0, j in [-1, W], T = 0 outside [0, W); samples
 * outside [0, N) are not modelled.  Computed in FP64 from float32 inputs; *loss
 * is device memory. */
int fbp_adjoint_loss(const fbp_dims* dims, const float* voltage, const float* templates,
                     const uint32_t* spike_idx, const uint32_t* spike_lab, const float* amplitude,
                     const float* shift, uint32_t n_spikes, double* loss, void* stream);

/* scale * dE/d(templates, amplitude, shift) for fbp_adjoint_loss's E.  Residual
 * tiles are recomputed per spike (nothing kept from the loss call); sums in
 * FP64.  grad_templates64 is FP64 scratch [M][C][W] (overwritten),
 * grad_templates float32 [M][C][W], grad_amplitude and grad_shift float32 [n]. */
int fbp_adjoint_grad(const fbp_dims* dims, const float* voltage, const float* templates,
                     const uint32_t* spike_idx, const uint32_t* spike_lab, const float* amplitude,
                     const float* shift, uint32_t n_spikes, double scale, double* grad_templates64,
                     float* grad_templates, float* grad_amplitude, float* grad_shift, void* stream);

/* ---- the pursuit's templates and noise covariances (pre-pursuit) ---- */

/* Clips of n spikes on the listed channels (get_clips,
 * spikesorting_fullpursuit/processing/clip_utils.py:501-632, for indices whose
 * window lies inside the voltage): clips[k][i*win_len + j] =
 * voltage[chans[i]][event_indices[k] + win0 + j].  voltage float32 [n_chans][n_samples],
 * clips float32 [n][n_nbr*win_len]. */
int fbp_gather_clips(const float* voltage, uint32_t n_chans, uint64_t n_samples, const uint32_t* chans,
                     uint32_t n_nbr, const int64_t* event_indices, uint32_t n, int32_t win0,
                     uint32_t win_len, float* clips, void* stream);

/* Robust template of n clips (calculate_robust_template, clip_utils.py:202-248):
 * per clip sample, in float32, the median of the values within one MAD/0.6745 of
 * the median (strictly), else the median; medians as np.median. */
int fbp_robust_template(const float* clips, uint32_t n, uint32_t clip_len, float* tmpl, void* stream);

/* Per-channel noise covariances of clip-minus-template residuals
 * (get_channel_covariance_matrix, spikesorting_fullpursuit/overlap/full_binary_pursuit.py:863-923):
 * residual row r = clips[r] - templates[unit_of[r]] (float32); for each channel c,
 * over the rows listed in rows[c][0..n_rows) (int64 [n_chans][n_rows]: the
 * reference draws them per channel), cov[c] (float64 [W][W], W =
 * n_samples_per_chan) is np.cov of samples [c*W, (c+1)*W) with ddof 0. */
int fbp_residual_covariance(const float* clips, const float* templates, const uint32_t* unit_of,
                            const int64_t* rows, uint32_t n_rows, uint32_t clip_len, uint32_t n_chans,
                            uint32_t n_samples_per_chan, double* cov, void* stream);

/* ---- noise model of the thresholds (pre-pursuit) ---- */

/* compute_separability_metrics + set_bp_threshold
 * (spikesorting_fullpursuit/overlap/neuron_separability.py:113-195, 319-331) per
 * template, on the device: template_SS (np.sum(T**2) in the templates' type,
 * numpy's pairwise order), the FP64 likelihood variance sum_c T_c' Cov_c T_c,
 * lower_CI = 0.5 SS - sigma_bp_ci sqrt(var), the threshold -0.5 SS +
 * sigma_bp_noise sqrt(var) (then max(threshold, 0, lower_CI) when
 * apply_bp_threshold), the contamination norm.sf(threshold, -0.5 SS, sqrt(var))
 * and the peak channel argmax|T| / W.  templates [M][C][W] float32 or float64
 * (templates_f64), channel_cov float64 [C][W][W]; template_ss has the templates'
 * type; other outputs float64 [M], peak_channel int64 [M]. */
int fbp_separability(const void* templates, int templates_f64, const double* channel_cov,
                     uint32_t n_templates, uint32_t n_chans, uint32_t template_len, double sigma_bp_noise,
                     double sigma_bp_ci, int apply_bp_threshold, void* template_ss, double* variance,
                     double* lower_ci, double* threshold, double* contamination, int64_t* peak_channel,
                     void* stream);

/* pairwise_separability (spikesorting_fullpursuit/overlap/neuron_separability.py:348-444,
 * with optimal_align_templates(align_abs=True, zero_pad=True) of
 * spikesorting_fullpursuit/overlap/consolidate.py:10-93), all pairs at once.  For each
 * pair (n1, n2): the shift is the first arg-max over lags [-max_shift, max_shift] of the
 * absolute cross-correlation of the flattened templates; the templates are aligned per
 * channel by it and zero padded; pair_matrix[n1][n2] = P(N(E_diff, sd) < 0) with
 * E_diff = 0.5 SS[n1] - (P1.P2 - 0.5 SS[n2]) and sd^2 the FP64 quadratic form of P1 - P2
 * with each channel's covariance (0 where that variance is not positive).  Per n1:
 * noise_misses = P(N(0.5 SS, sd_n1) < threshold), noise_contamination =
 * P(N(-0.5 SS, sd_n1) > threshold) (NaN where the variance is 0, as scipy gives).
 * templates [M][C][W] float32 or float64 (templates_f64); template_ss [M] in the same
 * type; channel_cov float64 [C][W][W]; variance, threshold float64 [M]; pair_matrix
 * float64 [M][M]; noise_* float64 [M]; optimal_shift int32 [M][M] or NULL.  The
 * reference uses max_shift = template_len / 4 - 1. */
int fbp_pair_separability(const void* templates, int templates_f64, const void* template_ss,
                          const double* channel_cov, const double* variance, const double* threshold,
                          uint32_t n_templates, uint32_t n_chans, uint32_t template_len, int32_t max_shift,
                          double* pair_matrix, double* noise_contamination, double* noise_misses,
                          int32_t* optimal_shift, void* stream);

/* ---- post-pursuit duplicate removal (device-resident output) ---- */

/* Mean clip of one unit, np.mean(clips, axis=0) in float32 (rows summed in
 * order, then divided by n): the template WorkItemSummary.
 * remove_segment_binary_pursuit_duplicates passes
 * (spikesorting_fullpursuit/postprocessing.py:660-666).  clips float32 [n][clip_len]. */
int fbp_mean_clip(const float* clips, uint32_t n, uint32_t clip_len, float* mean, void* stream);

/* Device workspace bytes fbp_bp_duplicates needs for n spikes. */
size_t fbp_bp_duplicates_workspace(uint32_t n);

/* remove_binary_pursuit_duplicates (spikesorting_fullpursuit/analyze_spike_timing.py:148-193)
 * for the spikes of one unit: keep[i] = 0 where spike i is dropped.  Of two spikes
 * within tol_inds samples that binary pursuit both found (bp != 0), the one whose
 * clip has the larger float32 sum of squared differences from unit_template
 * (numpy's pairwise summation order) is dropped, walking the spikes in the given
 * order exactly as the reference does.  event_indices int64 [n], clips float32
 * [n][clip_len], unit_template float32 [clip_len], bp uint8 [n], keep uint8 [n]. */
int fbp_bp_duplicates(const int64_t* event_indices, const float* clips, const float* unit_template,
                      const uint8_t* bp, uint32_t n, uint32_t clip_len, int64_t tol_inds,
                      uint8_t* keep, void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FBP_H */
