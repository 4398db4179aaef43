"""The pursuit's templates and noise covariances built on the GPU.

full_binary_pursuit (spikesorting_fullpursuit/overlap/full_binary_pursuit.py:325-349)
prepares binary_pursuit's inputs from the sorted spikes of a segment: per
unit, its clips on all channels and their robust template; from all units'
clip-minus-template residuals, one noise covariance per channel
(get_channel_covariance_matrix, full_binary_pursuit.py:863-923).

``get_channel_covariance_matrix`` keeps the reference's signature and result;
``templates_and_covariances`` does the per-unit loop of full_binary_pursuit.py:325-349
with the clips, templates and residuals left on the device.  Rows for the
covariances are drawn with numpy's global generator exactly as the reference
draws them (one np.random.randint call per channel when there are more
residuals than ``n_cov_samples``), so with the same generator state the same
rows are used.  Covariances agree with numpy's to FP64 rounding.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _native
from ..processing import clip_utils


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _rows(total, n_channels, n_cov_samples):
    out = []
    for _ in range(n_channels):
        if n_cov_samples >= total:
            out.append(np.arange(0, total))
        else:
            out.append(np.random.randint(0, total, n_cov_samples))
    return np.ascontiguousarray(np.stack(out).astype(np.int64))


def _covariances(torch, dev, clips, templates, unit_of, rows, n_channels, W):
    C = n_channels
    cov = torch.empty((C, W, W), dtype=torch.float64, device=dev)
    rd = torch.from_numpy(rows).to(dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(_native.lib().fbp_residual_covariance(_ptr(clips), _ptr(templates), _ptr(unit_of), _ptr(rd),
                                                        rows.shape[1], clips.shape[1], C, W, _ptr(cov), stream))
    c = cov.cpu().numpy()
    return [c[i] for i in range(C)]


def get_channel_covariance_matrix(clip_template_residuals, n_channels, n_samples_per_chan, n_cov_samples, verbose,
                                  device=None):
    """Noise covariance per channel of the residuals (list of float32 arrays, one
    per unit), as full_binary_pursuit.get_channel_covariance_matrix returns it."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    dev = (device if isinstance(device, torch.device)
           else torch.device("cuda", torch.cuda.current_device() if device is None else int(device)))
    R = np.vstack(clip_template_residuals)
    if R.dtype != np.float32:
        raise TypeError("residuals must be float32, got %s" % R.dtype)
    if verbose:
        print("Computing clip noise covariance for each channel with", n_cov_samples, "clip samples")
    rows = _rows(R.shape[0], n_channels, n_cov_samples)
    Rd = torch.from_numpy(np.ascontiguousarray(R)).to(dev)
    zero = torch.zeros((1, R.shape[1]), dtype=torch.float32, device=dev)
    unit_of = torch.zeros(R.shape[0], dtype=torch.int32, device=dev)
    return _covariances(torch, dev, Rd, zero, unit_of, rows, n_channels, n_samples_per_chan)


def templates_and_covariances(clips_dict, voltage, all_chan_nbrs, spike_indices_per_unit, clip_width_s, n_channels,
                              n_samples_per_chan, n_cov_samples, device=None):
    """Robust templates (units x clip length, float32) and per-channel noise
    covariances of full_binary_pursuit.py:325-349, with the clips on the device.
    Each unit's spike indices must be ordered (get_clips' contract)."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    dev = (device if isinstance(device, torch.device)
           else torch.device("cuda", torch.cuda.current_device() if device is None else int(device)))
    Vd = voltage if isinstance(voltage, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(voltage, np.float32))
    Vd = Vd.to(dev)
    clips, templates, units = [], [], []
    for u, idx in enumerate(spike_indices_per_unit):
        cl, _ = clip_utils.get_clips(clips_dict, Vd, all_chan_nbrs, np.asarray(idx), clip_width_s, device=dev,
                                     device_out=True)
        if cl is None:
            raise ValueError("unit %d has no spike whose clip lies inside the voltage" % u)
        t = clip_utils.calculate_robust_template(cl, device=dev, device_out=True)
        clips.append(cl)
        templates.append(t.reshape(1, -1))
        units.append(torch.full((cl.shape[0],), u, dtype=torch.int32, device=dev))
    allc = torch.cat(clips).contiguous()
    T = torch.cat(templates).contiguous()
    rows = _rows(allc.shape[0], n_channels, n_cov_samples)
    covs = _covariances(torch, dev, allc, T, torch.cat(units).contiguous(), rows, n_channels, n_samples_per_chan)
    return T.cpu().numpy(), covs
