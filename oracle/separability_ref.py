"""CPU restatement of the pursuit's noise model (checker for csrc/separability.cu).

TEST INFRASTRUCTURE ONLY.  Restates compute_separability_metrics and
set_bp_threshold (spikesorting_fullpursuit/overlap/neuron_separability.py:113-195,
319-331): template energies summed by numpy in the templates' type, FP64
quadratic forms with each channel's noise covariance, thresholds, lower
confidence bounds, tail probabilities and peak channels.
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
