"""CPU restatement of the pursuit's pre-processing (checker for csrc/preprocess.cu).

TEST INFRASTRUCTURE ONLY.  Restates get_clips (spikesorting_fullpursuit/processing/clip_utils.py:501-632,
edge checks :401-500), calculate_robust_template (clip_utils.py:202-248) and
get_channel_covariance_matrix (spikesorting_fullpursuit/overlap/full_binary_pursuit.py:863-923).
"""
from __future__ import annotations

import numpy as np


def _window(clip_width_s, fs):
    w = list(clip_width_s)
    if w[0] > 0:
        w[0] *= -1
    return [min(int(round(w[0] * fs)), 0), max(int(round(w[1] * fs)), 1) + 1]


def get_clips(probe, voltage, neighbors, event_indices, clip_width_s):
    window = _window(clip_width_s, probe["sampling_rate"])
    n = event_indices.size
    valid = np.ones(n, dtype=bool)
    start = 0
    while event_indices[start] + window[0] < 0:
        valid[start] = False
        start += 1
        if start == n:
            valid[:] = False
            return None, valid
    stop = n - 1
    while event_indices[stop] + window[1] > probe["n_samples"]:
        valid[stop] = False
        stop -= 1
        if stop < 0:
            valid[:] = False
            return None, valid
    wc = window[1] - window[0]
    clips = np.empty((stop + 1 - start, wc * len(neighbors)), dtype=probe["v_dtype"])
    for k, spk in enumerate(range(start, stop + 1)):
        for i, ch in enumerate(neighbors):
            clips[k, i * wc:(i + 1) * wc] = voltage[ch, event_indices[spk] + window[0]:event_indices[spk] + window[1]]
    return clips, valid


def robust_template(clips):
    if clips.shape[0] == 1 or clips.ndim == 1:
        return np.squeeze(clips)
    med = np.median(clips, axis=0)
    out = np.zeros(clips.shape[1], dtype=clips.dtype)
    for s in range(clips.shape[1]):
        mad = np.median(np.abs(clips[:, s] - med[s])) / 0.6745
        sel = np.logical_and(clips[:, s] > med[s] - mad, clips[:, s] < med[s] + mad)
        out[s] = med[s] if not np.any(sel) else np.median(clips[sel, s])
    return out


def channel_covariances(residuals, n_channels, W, n_cov_samples):
    R = np.vstack(residuals)
    out = []
    for c in range(n_channels):
        rows = np.arange(R.shape[0]) if n_cov_samples >= R.shape[0] else np.random.randint(0, R.shape[0], n_cov_samples)
        out.append(np.cov(R[rows, c * W:(c + 1) * W], rowvar=False, ddof=0))
    return out
