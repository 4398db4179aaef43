"""The pursuit's noise model on the GPU: bias and accept thresholds.

``compute_separability_metrics`` and ``set_bp_threshold`` have the signatures,
arguments and returned dictionary of
spikesorting_fullpursuit.overlap.neuron_separability (neuron_separability.py:113-195,
319-331); ``binary_pursuit`` reads ``templates``, ``template_SS`` and
``neuron_lower_thresholds`` from it.  The per-template work (the FP64 quadratic
forms of the templates with each channel's noise covariance, template energies,
thresholds, tail probabilities, peak channels) runs in libfbp.so
(csrc/separability.cu).  Template energies, expectations, peak channels are
bit-identical to the reference; variances and the values derived from them
agree to FP64 rounding (the reference sums its matrix products with BLAS).

``pairwise_separability`` (neuron_separability.py:348-444) estimates, for every
pair of units, the probability that a spike of one is taken for the other, and
per unit the probabilities of missing a spike or adding noise.  Each pair's
templates are aligned by the arg-max of their absolute cross-correlation
(consolidate.optimal_align_templates with align_abs=True, zero_pad=True) and
compared through the FP64 quadratic form of their difference with the channel
covariances; all pairs run at once on the device (csrc/separability.cu).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _native


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _device_metrics(templates, channel_covariance_mats, n_chans, W, sigma_noise, sigma_ci, apply_bp, device=None):
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    dev = (device if isinstance(device, torch.device)
           else torch.device("cuda", torch.cuda.current_device() if device is None else int(device)))
    T = np.ascontiguousarray(templates)
    f64 = T.dtype == np.float64
    if not f64 and T.dtype != np.float32:
        T = T.astype(np.float64)
        f64 = True
    M = T.shape[0]
    Td = torch.from_numpy(T.reshape(M, n_chans * W)).to(dev)
    cov = np.ascontiguousarray(np.stack([np.asarray(c, dtype=np.float64).reshape(W, W)
                                         for c in channel_covariance_mats[:n_chans]]))
    Cd = torch.from_numpy(cov).to(dev)
    ss = torch.empty(M, dtype=torch.float64 if f64 else torch.float32, device=dev)
    out = [torch.empty(M, dtype=torch.float64, device=dev) for _ in range(4)]
    peak = torch.empty(M, dtype=torch.int64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(_native.lib().fbp_separability(_ptr(Td), int(f64), _ptr(Cd), M, n_chans, W, float(sigma_noise),
                                                 float(sigma_ci), int(apply_bp), _ptr(ss), *[_ptr(o) for o in out],
                                                 _ptr(peak), stream))
    var, lower_ci, thr, contamination = (o.cpu().numpy() for o in out)
    return T, ss.cpu().numpy(), var, lower_ci, thr, contamination, peak.cpu().numpy()


def compute_separability_metrics(templates, channel_covariance_mats, sort_info, device=None):
    """neuron_separability.compute_separability_metrics on the GPU."""
    n_chans = sort_info["n_channels"]
    W = sort_info["n_samples_per_chan"]
    T = np.vstack(templates)
    M = T.shape[0]
    T, ss, var, lower_ci, thr, contamination, peak = _device_metrics(
        T, channel_covariance_mats, n_chans, W, sort_info["sigma_bp_noise"], sort_info["sigma_bp_CI"], False,
        device)
    sm = {
        "bp_n_samples_per_chan": W,
        "templates": np.vstack(templates),
        "template_SS": ss,
        "template_SS_by_chan": np.zeros((M, n_chans)),
        "channel_covariance_mats": channel_covariance_mats,
        "contamination": contamination,
        "peak_channel": peak,
        "channel_p_noise": np.zeros(n_chans),
        "neuron_variances": var,
        "neuron_lower_thresholds": thr,
        "neuron_lower_CI": lower_ci,
    }
    # per channel: fraction of samples without a threshold crossing (host scalars,
    # neuron_separability.py:141-153)
    for chan in range(n_chans):
        sm["channel_p_noise"][chan] = (sort_info["n_samples"] - sort_info["n_threshold_crossings"][chan]) \
            / sort_info["n_samples"]
    return sm


def set_bp_threshold(separability_metrics):
    """neuron_separability.set_bp_threshold: threshold = max(threshold, 0, lower CI)."""
    thr = separability_metrics["neuron_lower_thresholds"]
    ci = separability_metrics["neuron_lower_CI"]
    for n in range(ci.shape[0]):
        thr[n] = max(thr[n], 0)
        thr[n] = max(thr[n], ci[n])
    return separability_metrics


def bp_thresholds(templates, channel_covariance_mats, n_chans, W, sigma_bp_noise=3.719, sigma_bp_CI=np.inf,
                  device=None):
    """Both steps fused on the device: (template_SS, neuron_lower_thresholds) as
    binary_pursuit reads them (a NaN threshold becomes 0 here, where the
    reference's max() keeps it)."""
    _, ss, _, _, thr, _, _ = _device_metrics(np.vstack(templates), channel_covariance_mats, n_chans, W,
                                             sigma_bp_noise, sigma_bp_CI, True, device)
    return ss, thr


def _pair_metrics(separability_metrics, sort_info, device=None):
    """(pair matrix, noise contamination, noise misses, optimal shifts) of all pairs."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    dev = (device if isinstance(device, torch.device)
           else torch.device("cuda", torch.cuda.current_device() if device is None else int(device)))
    n_chans = sort_info["n_channels"]
    W = int(separability_metrics["bp_n_samples_per_chan"])
    max_shift = (W // 4) - 1
    T = np.ascontiguousarray(separability_metrics["templates"])
    if T.dtype not in (np.float32, np.float64):
        T = T.astype(np.float64)
    M = T.shape[0]
    if max_shift < 0:
        # the reference's arg-max over an empty lag range
        raise ValueError("attempt to get argmax of an empty sequence")
    if M == 0:
        return np.zeros((0, 0)), np.zeros(0), np.zeros(0), np.zeros((0, 0), dtype=np.int32)
    ss = np.ascontiguousarray(np.asarray(separability_metrics["template_SS"]).astype(T.dtype, copy=False))
    covs = separability_metrics["channel_covariance_mats"]
    cov = np.ascontiguousarray(np.stack([np.asarray(c, dtype=np.float64).reshape(W, W) for c in covs[:n_chans]]))
    var = np.ascontiguousarray(np.asarray(separability_metrics["neuron_variances"], dtype=np.float64))
    thr = np.ascontiguousarray(np.asarray(separability_metrics["neuron_lower_thresholds"], dtype=np.float64))
    Td = torch.from_numpy(T.reshape(M, n_chans * W)).to(dev)
    ssd, covd, vard, thrd = (torch.from_numpy(a).to(dev) for a in (ss, cov, var, thr))
    pair = torch.empty((M, M), dtype=torch.float64, device=dev)
    contamination = torch.empty(M, dtype=torch.float64, device=dev)
    misses = torch.empty(M, dtype=torch.float64, device=dev)
    shifts = torch.empty((M, M), dtype=torch.int32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(_native.lib().fbp_pair_separability(
        _ptr(Td), int(T.dtype == np.float64), _ptr(ssd), _ptr(covd), _ptr(vard), _ptr(thrd), M, n_chans, W,
        max_shift, _ptr(pair), _ptr(contamination), _ptr(misses), _ptr(shifts), stream))
    return pair.cpu().numpy(), contamination.cpu().numpy(), misses.cpu().numpy(), shifts.cpu().numpy()


def pairwise_separability(separability_metrics, sort_info, device=None):
    """neuron_separability.pairwise_separability on the GPU: returns
    (pair_separability_matrix, noise_contamination, noise_misses).
    pair_separability_matrix[n1, n2] is the probability that the likelihood of
    unit n2 exceeds that of unit n1 given an n1 spike; noise_misses[n] the
    probability that a spike of n stays below its threshold; noise_contamination[n]
    the probability that noise alone crosses it."""
    pair, contamination, misses, _ = _pair_metrics(separability_metrics, sort_info, device)
    return pair, contamination, misses
