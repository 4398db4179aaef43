/*
 * bp_oracle.c -- CPU restatement of Full Binary Pursuit's per-chunk pursuit.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * spikesorting_fullpursuit_b200/csrc.  Only tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py may load it.  The product never does.
 *
 * It restates, in plain C, the algorithm of
 *   spikesorting_fullpursuit/overlap/binary_pursuit_parallel.py:907-1356  (host loop)
 *   spikesorting_fullpursuit/kernels/binary_pursuit.cl:57-1130            (kernels)
 * with every order-dependent step fixed to the order the reference kernels
 * produce when their work-groups run one after another (the "canonical" order;
 * on a GPU the reference itself is non-deterministic at these points):
 *   - per-window argmax: templates ascending, samples ascending, strict '>';
 *   - overlap recheck: a work-group tree max (strict '>', lower slot keeps
 *     ties) followed by a strict '>' scan over the groups of one window;
 *   - check_overlap_reassignments: flagged windows in ascending order;
 *   - accept/prune: work-groups of WG list entries in order; inside a group
 *     all accepts first, then the prune rules entry by entry;
 *   - spike output and residual subtraction: window-list order.
 * Compile with -ffp-contract=off: every float product and sum is rounded on
 * its own, as the reference's scalar loops are.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    uint32_t C;   /* channels */
    uint32_t N;   /* samples per channel in this chunk */
    uint32_t M;   /* templates */
    uint32_t W;   /* template samples per channel (window length) */
    uint32_t S;   /* n_max_shift_inds */
    uint32_t WG;  /* work-group size the canonical order is defined with (power of 2) */
    int32_t do_overlap;
    int32_t threads;
} bpo_params;

typedef struct {
    int32_t passes;
    int32_t status;
    uint64_t spikes;
    uint64_t flagged;        /* flagged windows summed over passes */
    uint64_t overlap_items;  /* (a,t,b) items that were not skipped */
    uint64_t listed;         /* listed windows summed over passes */
} bpo_stats;

enum { BPO_OK = 0, BPO_EBADARG = -1, BPO_ENOMEM = -2, BPO_EPASSES = -3 };

/* compute_maximum_likelihood / compute_full_likelihood
 * (binary_pursuit.cl:216-252, 255-300): L[t,s] = b_t + sum_c sum_j T[t,c,j] V[c,s+j]
 * in channel-major, j-ascending order from one float accumulator; 0 when s+W >= N. */
static void lik_window(const bpo_params* P, const float* V, const float* T,
                       const float* bias, float* L, uint32_t id)
{
    const uint64_t N = P->N;
    uint64_t s0 = (uint64_t)id * P->W;
    uint64_t s1 = s0 + P->W;
    if (s1 > N) s1 = N;
    for (uint32_t t = 0; t < P->M; ++t) {
        float* Lt = L + (uint64_t)t * N;
        const float* Tt = T + (uint64_t)t * P->C * P->W;
        for (uint64_t s = s0; s < s1; ++s) {
            if (s + P->W >= N) { Lt[s] = 0.0f; continue; }
            float acc = bias[t];
            for (uint32_t c = 0; c < P->C; ++c) {
                const float* tc = Tt + (uint64_t)c * P->W;
                const float* vc = V + (uint64_t)c * N + s;
                for (uint32_t j = 0; j < P->W; ++j) acc = acc + tc[j] * vc[j];
            }
            Lt[s] = acc;
        }
    }
}

/* compute_template_maximum_likelihood (binary_pursuit.cl:350-441), the M host
 * launches of binary_pursuit_parallel.py:943-965 folded into one loop. */
static void argmax_window(const bpo_params* P, const float* L, uint32_t id,
                          float* best_lik, uint32_t* best_lab, uint32_t* best_idx,
                          uint8_t* check, uint8_t* orech, uint32_t* ov_idx, uint32_t* ov_lab)
{
    const uint64_t N = P->N, W = P->W;
    const uint64_t start_w = (uint64_t)id * W, end_w = start_w + W;
    if (end_w >= N - W) return;
    const uint64_t lo = (W > start_w) ? 0 : start_w - W;
    const uint64_t hi = (end_w + W > N) ? N : end_w + W;
    float bl = best_lik[id];
    uint32_t blab = best_lab[id], bidx = best_idx[id];
    int flag = 0;
    for (uint32_t t = 0; t < P->M; ++t) {
        if (t == 0) bl = 0.0f;
        const float* Lt = L + (uint64_t)t * N;
        for (uint64_t s = lo; s < hi; ++s) {
            float v = Lt[s];
            if (v > bl) { bl = v; blab = t; bidx = (uint32_t)s; }
            if (v > 0.0f && s >= start_w && s < end_w) flag = 1;
        }
    }
    if (flag) check[id] = 1;
    orech[id] = (bl > 0.0f && bidx >= start_w && bidx < end_w) ? 1 : 0;
    best_lik[id] = bl; best_lab[id] = blab; best_idx[id] = bidx;
    ov_idx[id] = bidx; ov_lab[id] = blab;
}

static inline uint32_t bitrev(uint32_t x, uint32_t bits)
{
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; ++i) { r = (r << 1) | (x & 1u); x >>= 1; }
    return r;
}

/* Pair likelihood of one (a, t, b) item of overlap_recheck_indices
 * (binary_pursuit.cl:578-632): the best template f shifted by a-S plus template
 * t shifted by b-S, truncated to the window [p, p+W), scored against the
 * residual as sum_c [ sum_j s_j v_j - 0.5 sum_j s_j^2 ]. */
static float pair_value(const bpo_params* P, const float* V, const float* T,
                        uint32_t f, uint32_t t, uint64_t p, uint32_t a, uint32_t b)
{
    const int64_t W = P->W, S = P->S;
    const int64_t fa = S - (int64_t)a, ta = S - (int64_t)b;  /* alignment offsets */
    float acc = 0.0f;
    for (uint32_t c = 0; c < P->C; ++c) {
        const float* fc = T + ((uint64_t)f * P->C + c) * P->W;
        const float* tc = T + ((uint64_t)t * P->C + c) * P->W;
        const float* vc = V + (uint64_t)c * P->N + p;
        float ss = 0.0f;
        for (int64_t j = 0; j < W; ++j) {
            int64_t xf = fa + j, xt = ta + j;
            float fv = (xf >= 0 && xf < W) ? fc[xf] : 0.0f;
            float tv = (xt >= 0 && xt < W) ? tc[xt] : 0.0f;
            float sv = fv + tv;
            ss = ss + sv * sv;
            acc = acc + sv * vc[j];
        }
        if (ss > 0.0f) acc = acc - 0.5f * ss;
    }
    return acc;
}

/* overlap_recheck_indices + max_local_reduction (binary_pursuit.cl:444-654,
 * 167-186) followed by the group scan of parse_overlap_recheck_indices
 * (binary_pursuit.cl:690-706).  The work-item of (a, t, b) has in-window
 * position r = t + M*a + M*(2S+1)*b; slots r >= items repeat item r - items
 * (binary_pursuit.cl:483-532).  Returns the winning value and r; a winner exists
 * only if some value beats the seed (the window's best likelihood). */
static int overlap_winner(const bpo_params* P, const float* V, const float* T,
                          const float* L, const float* theta, uint32_t id,
                          float seed, uint32_t f, uint32_t p,
                          float* win_val, uint64_t* win_r, uint64_t* n_items)
{
    const uint64_t N = P->N, W = P->W, S = P->S, M = P->M, S2 = 2ull * S + 1;
    const uint64_t items = S2 * S2 * M;
    const uint64_t WGs = P->WG;
    const uint64_t nloc = (items - 1) / WGs + 1;
    uint32_t lbits = 0;
    while ((1ull << lbits) < WGs) ++lbits;
    (void)id;
    *n_items = 0;
    if (L[(uint64_t)f * N + p] < theta[f]) return 0;
    if ((uint64_t)p >= N - W) return 0;
    int have = 0;
    float bv = 0.0f;
    uint64_t bprio = 0, br = 0;
    for (uint64_t b = 0; b < S2; ++b) {
        if (b + p < S || b + p >= N - W + S) continue;
        for (uint64_t a = 0; a < S2; ++a) {
            if (a + p < S || a + p >= N - W + S) continue;
            if ((a > b ? a - b : b - a) > W) continue;
            const float lf = L[(uint64_t)f * N + p + a - S];
            for (uint64_t t = 0; t < M; ++t) {
                const float lt = L[t * N + p + b - S];
                if (lf <= 0.0f && lt <= 0.0f) continue;
                float v = pair_value(P, V, T, f, (uint32_t)t, p, (uint32_t)a, (uint32_t)b);
                (*n_items)++;
                if (!(v > seed)) continue;
                /* every slot holding this item: r, r + items, ... below nloc*WG */
                for (uint64_t r = t + M * a + M * S2 * b; r < nloc * WGs; r += items) {
                    uint64_t g = r / WGs, l = r % WGs;
                    uint64_t prio = g * WGs + bitrev((uint32_t)l, lbits);
                    if (!have || v > bv || (v == bv && prio < bprio)) {
                        have = 1; bv = v; bprio = prio; br = r;
                    }
                }
            }
        }
    }
    if (have) { *win_val = bv; *win_r = br; }
    return have;
}

/* parse_overlap_recheck_indices accept rules (binary_pursuit.cl:707-814). */
static void parse_window(const bpo_params* P, const float* L, const float* theta, uint32_t id,
                         int have, float gv, uint64_t r,
                         float* best_lik, const uint32_t* best_lab, const uint32_t* best_idx,
                         uint8_t* orech, uint32_t* ov_idx, uint32_t* ov_lab)
{
    const uint64_t N = P->N, S = P->S, M = P->M, S2 = 2ull * S + 1;
    const uint64_t items = S2 * S2 * M;
    const float seed = best_lik[id];
    if (!have || gv <= seed || gv <= 0.0f) { orech[id] = 0; return; }
    if (r >= items) { orech[id] = 0; return; }
    const uint32_t f = best_lab[id], p = best_idx[id];
    const uint32_t t = (uint32_t)(r % M);
    const uint64_t a = (r / M) % S2, b = (r / (S2 * M)) % S2;
    const uint32_t afi = (uint32_t)(p + a - S), asi = (uint32_t)(p + b - S);
    const float l1 = L[(uint64_t)f * N + afi];
    const float l2 = L[(uint64_t)t * N + asi];
    if (gv < l1 || gv < l2) { orech[id] = 0; return; }
    if (l1 <= 0.0f || l2 <= 0.0f) { orech[id] = 0; return; }
    if (l1 >= l2 && l1 > theta[f]) { best_lik[id] = l1; ov_lab[id] = f; ov_idx[id] = afi; }
    else if (l2 > l1 && l2 > theta[t]) { best_lik[id] = l2; ov_lab[id] = t; ov_idx[id] = asi; }
    else if (l1 > theta[f]) { best_lik[id] = l1; ov_lab[id] = f; ov_idx[id] = afi; }
    else { ov_idx[id] = best_idx[id]; ov_lab[id] = best_lab[id]; orech[id] = 0; }
}

/* check_overlap_reassignments (binary_pursuit.cl:822-875), ascending order. */
static void reassign_window(const bpo_params* P, uint32_t id, uint32_t* best_idx, uint32_t* best_lab,
                            uint8_t* check, const uint32_t* ov_idx, const uint32_t* ov_lab,
                            uint8_t* orech)
{
    const uint64_t W = P->W;
    const uint64_t start_w = (uint64_t)id * W, end_w = start_w + W;
    if (orech[id] == 0) return;
    best_idx[id] = ov_idx[id];
    best_lab[id] = ov_lab[id];
    if (ov_idx[id] < start_w && id > 1) {
        if (orech[id - 2] == 1) {
            orech[id] = 0;
            best_idx[id] = 0;
            check[id - 1] = 2; check[id] = 2; check[id + 1] = 2;
        } else {
            check[id - 2] = 2;
        }
    }
    if (ov_idx[id] >= end_w && (uint64_t)id + 2 < P->N / W) check[id + 2] = 2;
}

/* binary_pursuit kernel (binary_pursuit.cl:918-1063) over the window list in
 * work-groups of WG entries; returns the number of spikes appended. */
static uint64_t accept_prune(const bpo_params* P, const float* theta, const uint32_t* list, uint64_t nlist,
                             const float* best_lik, const uint32_t* best_lab, const uint32_t* best_idx,
                             const uint8_t* orech, uint8_t* check,
                             uint32_t* sp_idx, uint32_t* sp_lab, uint8_t* has)
{
    const uint64_t N = P->N, W = P->W, WGs = P->WG;
    const uint64_t nwf = N / W;
    uint64_t count = 0;
    for (uint64_t g0 = 0; g0 < nlist; g0 += WGs) {
        uint64_t g1 = g0 + WGs < nlist ? g0 + WGs : nlist;   /* padding entries do nothing */
        for (uint64_t k = g0; k < g1; ++k) {
            uint32_t id = list[k];
            uint64_t start_w = (uint64_t)id * W, end_w = start_w + W;
            float ml = 0.0f; uint32_t lab = 0, idx = 0;
            if (end_w < N - W) { ml = best_lik[id]; lab = best_lab[id]; idx = best_idx[id]; }
            has[k - g0] = 0;
            if (ml > theta[lab] || orech[id] == 1) {
                if ((idx >= start_w && idx < end_w) || orech[id] == 1) {
                    has[k - g0] = 1;
                    check[id] = 3;
                    if (id > 0) check[id - 1] = 3;
                    if ((uint64_t)id + 1 < nwf) check[id + 1] = 3;
                }
            }
        }
        for (uint64_t k = g0; k < g1; ++k) {
            uint32_t id = list[k];
            uint64_t start_w = (uint64_t)id * W, end_w = start_w + W;
            if (!(end_w < N - W) || has[k - g0]) continue;
            float ml = best_lik[id]; uint32_t lab = best_lab[id], idx = best_idx[id];
            if (idx < start_w && check[id] == 1 && id > 0 && check[id - 1] == 0) check[id] = 0;
            if (idx >= end_w && check[id] == 1 && (uint64_t)id + 1 < nwf && check[id + 1] == 0) check[id] = 0;
            if (ml <= theta[lab] && check[id] < 3) check[id] = 0;
        }
        for (uint64_t k = g0; k < g1; ++k) {
            if (!has[k - g0]) continue;
            uint32_t id = list[k];
            sp_idx[count] = best_idx[id];
            sp_lab[count] = best_lab[id];
            ++count;
        }
    }
    return count;
}

/* compute_residual (binary_pursuit.cl:57-102), spikes in output order. */
static void residual(const bpo_params* P, float* V, const float* T,
                     const uint32_t* sp_idx, const uint32_t* sp_lab, uint64_t n)
{
    const uint64_t N = P->N, W = P->W;
    for (uint64_t k = 0; k < n; ++k) {
        uint64_t s = sp_idx[k];
        uint32_t l = sp_lab[k];
        if (l >= P->M) continue;
        for (uint32_t c = 0; c < P->C; ++c) {
            float* vc = V + (uint64_t)c * N;
            const float* tc = T + ((uint64_t)l * P->C + c) * W;
            for (uint64_t i = 0; i < W; ++i) {
                if (s + i >= N) break;
                vc[s + i] = vc[s + i] - tc[i];
            }
        }
    }
}

/* get_adjusted_clips (binary_pursuit.cl:1088-1130). */
void bpo_adjusted_clips(const bpo_params* P, const float* V, const float* T,
                        const uint32_t* sp_idx, const uint32_t* sp_lab, uint64_t n, float* clips)
{
    const uint64_t N = P->N, W = P->W, CW = (uint64_t)P->C * P->W;
    for (uint64_t k = 0; k < n; ++k) {
        uint64_t s = sp_idx[k];
        uint32_t l = sp_lab[k];
        if (l >= P->M) continue;
        for (uint32_t c = 0; c < P->C; ++c) {
            const float* vc = V + (uint64_t)c * N;
            const float* tc = T + ((uint64_t)l * P->C + c) * W;
            float* out = clips + k * CW + (uint64_t)c * W;
            for (uint64_t i = 0; i < W; ++i) {
                if (s + i >= N) break;
                out[i] = vc[s + i] + tc[i];
            }
        }
    }
}

/* Likelihood of every window of a chunk (one first-pass launch of
 * compute_full_likelihood); exported for kernel-level tests. */
void bpo_likelihood_all(const bpo_params* P, const float* V, const float* T, const float* bias, float* L)
{
    const uint64_t nw = ((uint64_t)P->N + P->W - 1) / P->W;
    #pragma omp parallel for schedule(dynamic, 64) num_threads(P->threads > 0 ? P->threads : 1)
    for (int64_t k = 0; k < (int64_t)nw; ++k) lik_window(P, V, T, bias, L, (uint32_t)k);
}

/* Pair likelihood of one item; exported for kernel-level tests. */
float bpo_pair_value(const bpo_params* P, const float* V, const float* T,
                     uint32_t f, uint32_t t, uint64_t p, uint32_t a, uint32_t b)
{
    return pair_value(P, V, T, f, t, p, a, b);
}

/* One chunk of the pursuit loop of binary_pursuit_parallel.py:907-1356.
 * V (C x N) is turned into the residual in place.  Spikes are appended to
 * sp_idx/sp_lab (capacity cap) pass by pass, each pass in window order. */
int bpo_pursue_chunk(const bpo_params* P, float* V, const float* T, const float* bias,
                     const float* theta, uint32_t* sp_idx, uint32_t* sp_lab, uint64_t cap,
                     uint64_t* n_out, int32_t max_passes, bpo_stats* st)
{
    if (!P || !V || !T || !bias || !theta || !n_out) return BPO_EBADARG;
    if (P->C == 0 || P->M == 0 || P->W == 0 || P->N <= P->W) return BPO_EBADARG;
    if (P->WG == 0 || (P->WG & (P->WG - 1))) return BPO_EBADARG;
    const uint64_t N = P->N, M = P->M, W = P->W;
    const uint64_t nw = (N + W - 1) / W;
    const int nth = P->threads > 0 ? P->threads : 1;
    memset(st, 0, sizeof(*st));
    float* L = (float*)calloc(M * N, sizeof(float));
    float* best_lik = (float*)calloc(nw, sizeof(float));
    uint32_t* best_lab = (uint32_t*)calloc(nw, 4);
    uint32_t* best_idx = (uint32_t*)calloc(nw, 4);
    uint32_t* ov_idx = (uint32_t*)calloc(nw, 4);
    uint32_t* ov_lab = (uint32_t*)calloc(nw, 4);
    uint8_t* check = (uint8_t*)calloc(nw, 1);
    uint8_t* orech = (uint8_t*)calloc(nw, 1);
    uint32_t* list = (uint32_t*)malloc(nw * 4);
    uint32_t* flag = (uint32_t*)malloc(nw * 4);
    uint32_t* pidx = (uint32_t*)malloc(nw * 4);
    uint32_t* plab = (uint32_t*)malloc(nw * 4);
    float* gval = (float*)malloc(nw * 4);
    uint64_t* gr = (uint64_t*)malloc(nw * 8);
    int* ghave = (int*)malloc(nw * sizeof(int));
    uint8_t* has = (uint8_t*)malloc(P->WG);
    int rc = BPO_OK;
    if (!L || !best_lik || !best_lab || !best_idx || !ov_idx || !ov_lab || !check || !orech ||
        !list || !flag || !pidx || !plab || !gval || !gr || !ghave || !has) { rc = BPO_ENOMEM; goto done; }
    uint64_t nlist = nw, total = 0;
    for (uint64_t k = 0; k < nw; ++k) list[k] = (uint32_t)k;
    for (int32_t pass = 1;; ++pass) {
        if (max_passes > 0 && pass > max_passes) { rc = BPO_EPASSES; break; }
        st->passes = pass;
        st->listed += nlist;
        #pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
        for (int64_t k = 0; k < (int64_t)nlist; ++k) lik_window(P, V, T, bias, L, list[k]);
        #pragma omp parallel for schedule(dynamic, 64) num_threads(nth)
        for (int64_t k = 0; k < (int64_t)nlist; ++k)
            argmax_window(P, L, list[k], best_lik, best_lab, best_idx, check, orech, ov_idx, ov_lab);
        uint64_t nflag = 0;
        for (uint64_t k = 0; k < nw; ++k) if (orech[k]) flag[nflag++] = (uint32_t)k;
        if (nflag > 0 && P->do_overlap) {
            st->flagged += nflag;
            uint64_t items_sum = 0;
            #pragma omp parallel for schedule(dynamic, 1) num_threads(nth) reduction(+:items_sum)
            for (int64_t k = 0; k < (int64_t)nflag; ++k) {
                uint32_t id = flag[k];
                uint64_t ni = 0;
                ghave[k] = overlap_winner(P, V, T, L, theta, id, best_lik[id], best_lab[id],
                                          best_idx[id], &gval[k], &gr[k], &ni);
                items_sum += ni;
            }
            st->overlap_items += items_sum;
            for (uint64_t k = 0; k < nflag; ++k)
                parse_window(P, L, theta, flag[k], ghave[k], gval[k], gr[k],
                             best_lik, best_lab, best_idx, orech, ov_idx, ov_lab);
            for (uint64_t k = 0; k < nflag; ++k)
                reassign_window(P, flag[k], best_idx, best_lab, check, ov_idx, ov_lab, orech);
        }
        uint64_t cnt = accept_prune(P, theta, list, nlist, best_lik, best_lab, best_idx,
                                    orech, check, pidx, plab, has);
        if (cnt == 0) break;
        memset(orech, 0, nw);
        nlist = 0;
        for (uint64_t k = 0; k < nw; ++k) if (check[k]) list[nlist++] = (uint32_t)k;
        memset(check, 0, nw);
        if (total + cnt > cap) { rc = BPO_EBADARG; break; }
        memcpy(sp_idx + total, pidx, cnt * 4);
        memcpy(sp_lab + total, plab, cnt * 4);
        total += cnt;
        residual(P, V, T, pidx, plab, cnt);
    }
    *n_out = total;
    st->spikes = total;
done:
    st->status = rc;
    free(L); free(best_lik); free(best_lab); free(best_idx); free(ov_idx); free(ov_lab);
    free(check); free(orech); free(list); free(flag); free(pidx); free(plab); free(gval);
    free(gr); free(ghave); free(has);
    return rc;
}
