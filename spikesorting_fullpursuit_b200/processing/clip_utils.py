"""Clips and robust templates on the GPU (full_binary_pursuit's pre-processing).

``get_clips`` and ``calculate_robust_template`` keep the signatures, argument
meaning and results of spikesorting_fullpursuit.processing.clip_utils
(clip_utils.py:501-632 and 202-248); the work runs in libfbp.so
(csrc/preprocess.cu) and the results are bit-identical to the reference's
numpy code.  Differences: memory-mapped output (``use_memmap``) is not
offered (the clips stay in memory, or on the device with ``device_out``), and
clips are float32 (the pursuit's voltage type).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _native
from .conversions import time_window_to_samples


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _torch_dev(device):
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    return torch, (device if isinstance(device, torch.device)
           else torch.device("cuda", torch.cuda.current_device() if device is None else int(device)))


def _valid_range(event_indices, n_samples, window):
    """validate_first_indices / validate_last_indices (clip_utils.py:435-500) for
    ordered indices: the valid spikes are [start, stop]."""
    n = event_indices.size
    valid = np.ones(n, dtype=bool)
    start = 0
    while event_indices[start] + window[0] < 0:
        valid[start] = False
        start += 1
        if start == n:
            valid[:] = False
            break
    stop = n - 1
    while event_indices[stop] + window[1] > n_samples:
        valid[stop] = False
        stop -= 1
        if stop < 0:
            valid[:] = False
            break
    return valid, start, stop


def get_clips(probe_dict, voltage, neighbors, event_indices, clip_width_s, use_memmap=False, check_valid=True,
              device=None, device_out=False):
    """Clips of the (ordered) event indices on the ``neighbors`` channels; returns
    (clips, valid_event_indices) as the reference does.  ``voltage`` may be a
    numpy array or a CUDA tensor; with ``device_out`` the clips stay a CUDA tensor."""
    if use_memmap:
        raise ValueError("memory-mapped clips are not offered; the clips are returned in memory")
    torch, dev = _torch_dev(device)
    event_indices = np.asarray(event_indices)
    if event_indices.ndim > 1:
        raise ValueError("Event_indices must be one dimensional array of indices")
    window, _ = time_window_to_samples(clip_width_s, probe_dict["sampling_rate"])
    neighbors = np.asarray(neighbors, dtype=np.int64).reshape(-1)
    wc = window[1] - window[0]
    if len(event_indices) == 0:
        return np.zeros((0, wc * len(neighbors)), dtype=probe_dict["v_dtype"]), np.ones(0, dtype="bool")
    if check_valid:
        valid, start, stop = _valid_range(event_indices, probe_dict["n_samples"], window)
        if not np.any(valid):
            return None, valid
    else:
        valid, start, stop = np.ones(event_indices.size, dtype=bool), 0, event_indices.size - 1
    Vd = voltage if isinstance(voltage, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(voltage, np.float32))
    Vd = Vd.to(device=dev, dtype=torch.float32).contiguous()
    ev = torch.from_numpy(np.ascontiguousarray(event_indices[start:stop + 1], dtype=np.int64)).to(dev)
    ch = torch.from_numpy(neighbors.astype(np.int32)).to(dev)
    n = stop + 1 - start
    clips = torch.empty((n, wc * neighbors.size), dtype=torch.float32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(_native.lib().fbp_gather_clips(_ptr(Vd), Vd.shape[0], Vd.shape[1], _ptr(ch), neighbors.size,
                                                 _ptr(ev), n, window[0], wc, _ptr(clips), stream))
    if device_out:
        return clips, valid
    return clips.cpu().numpy().astype(probe_dict["v_dtype"], copy=False), valid


def calculate_robust_template(all_channel_clips, device=None, device_out=False):
    """Robust template of float32 clips [n, clip_len] (clip_utils.py:202-248)."""
    torch, dev = _torch_dev(device)
    c = all_channel_clips
    if (c.shape[0] == 1 if c.ndim > 1 else True):
        # only one clip: nothing to average over (the reference returns it squeezed)
        return c.reshape(-1) if device_out or not isinstance(c, torch.Tensor) else c.reshape(-1).cpu().numpy()
    if str(c.dtype).split(".")[-1] != "float32":
        raise TypeError("clips must be float32, got %s" % c.dtype)
    cd = c if isinstance(c, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(c))
    cd = cd.to(dev).contiguous()
    out = torch.empty(cd.shape[1], dtype=torch.float32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(_native.lib().fbp_robust_template(_ptr(cd), cd.shape[0], cd.shape[1], _ptr(out), stream))
    return out if device_out else out.cpu().numpy()
