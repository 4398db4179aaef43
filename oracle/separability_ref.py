"""CPU restatement of the pursuit's noise model (checker for csrc/separability.cu).

TEST INFRASTRUCTURE ONLY.  Restates compute_separability_metrics and
set_bp_threshold (spikesorting_fullpursuit/overlap/neuron_separability.py:113-195,
319-331): template energies summed by numpy in the templates' type, FP64
quadratic forms with each channel's noise covariance, thresholds, lower
confidence bounds, tail probabilities and peak channels; and pairwise_separability
(neuron_separability.py:348-444) with the template alignment it uses
(consolidate.optimal_align_templates, consolidate.py:10-93, align_abs=True,
zero_pad=True).
"""
from __future__ import annotations

import numpy as np
from scipy.stats import norm


def separability(templates, covs, sort_info):
    T = np.vstack(templates)
    n_chans = sort_info["n_channels"]
    W = sort_info["n_samples_per_chan"]
    M = T.shape[0]
    ss = np.sum(T ** 2, axis=1)
    var = np.zeros(M)
    for n in range(M):
        for c in range(n_chans):
            t = T[n, c * W:(c + 1) * W].astype(np.float64)
            var[n] += t @ covs[c] @ t
    expectation = 0.5 * ss
    lower_ci = expectation - sort_info["sigma_bp_CI"] * np.sqrt(var)
    thr = -1 * expectation + sort_info["sigma_bp_noise"] * np.sqrt(var)
    contamination = norm.sf(thr, -expectation, np.sqrt(var))
    peak = np.argmax(np.abs(T), axis=1) // W
    p_noise = (sort_info["n_samples"] - np.asarray(sort_info["n_threshold_crossings"])) / sort_info["n_samples"]
    thr = np.maximum(np.maximum(thr, 0), lower_ci)
    return {"template_SS": ss, "neuron_variances": var, "neuron_lower_CI": lower_ci,
            "neuron_lower_thresholds": thr, "contamination": contamination, "peak_channel": peak,
            "channel_p_noise": p_noise}


def align_pair(t1, t2, n_chans, max_shift):
    """Shift of t2 against t1 that maximises |cross-correlation| within
    +-max_shift lags (first maximum), and the two templates aligned per channel
    by it, zero padded to full length; with shift 0 the templates themselves
    (consolidate.py:27-44, 70-91)."""
    cc = np.abs(np.correlate(t1, t2, mode="full"))
    centre = cc.shape[0] // 2
    shift = int(np.argmax(cc[centre - max_shift:centre + max_shift + 1])) - max_shift
    if shift == 0:
        return t1, t2, 0
    W = t1.shape[0] // n_chans
    lo, hi = max(shift, 0), W + min(shift, 0)
    p1 = np.zeros(t1.shape[0])
    p2 = np.zeros(t2.shape[0])
    for c in range(n_chans):
        p1[c * W + lo:c * W + hi] = t1[c * W + lo:c * W + hi]
        p2[c * W + lo:c * W + hi] = t2[c * W + lo - shift:c * W + hi - shift]
    return p1, p2, shift


def pairwise(sm, sort_info):
    """(pair matrix, noise contamination, noise misses, shifts) as
    pairwise_separability computes them (neuron_separability.py:348-444)."""
    n_chans = sort_info["n_channels"]
    W = sm["bp_n_samples_per_chan"]
    max_shift = (W // 4) - 1
    T = sm["templates"]
    M = T.shape[0]
    ss = sm["template_SS"]
    covs = sm["channel_covariance_mats"]
    sd = np.sqrt(sm["neuron_variances"])
    thr = sm["neuron_lower_thresholds"]
    pair = np.zeros((M, M))
    shifts = np.zeros((M, M), dtype=np.int32)
    misses = np.zeros(M)
    contamination = np.zeros(M)
    for n1 in range(M):
        e1 = 0.5 * ss[n1]
        misses[n1] = norm.cdf(thr[n1], e1, sd[n1])
        contamination[n1] = norm.sf(thr[n1], -0.5 * ss[n1], sd[n1])
        for n2 in range(M):
            p1, p2, shifts[n1, n2] = align_pair(T[n1, :], T[n2, :], n_chans, max_shift)
            var_diff = 0
            for c in range(n_chans):
                d = p1[c * W:(c + 1) * W] - p2[c * W:(c + 1) * W]
                var_diff += d[None, :] @ covs[c] @ d[:, None]
            e_diff = e1 - (np.dot(p1, p2) - 0.5 * ss[n2])
            pair[n1, n2] = norm.cdf(0, e_diff, np.sqrt(var_diff)).item() if var_diff > 0 else 0
    return pair, contamination, misses, shifts
