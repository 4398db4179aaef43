"""Duplicate removal on the pursuit's output, on the GPU.

``remove_binary_pursuit_duplicates`` has the signature, argument meaning and
result of spikesorting_fullpursuit.analyze_spike_timing.remove_binary_pursuit_duplicates
(analyze_spike_timing.py:148-193): for the spikes of one unit, in the given
order, of two spikes within ``tol_inds`` samples that binary pursuit both found
the one whose clip is farther from ``unit_template`` (float32 sum of squared
differences) is dropped.  ``remove_segment_duplicates`` is the per-unit loop of
WorkItemSummary.remove_segment_binary_pursuit_duplicates
(postprocessing.py:646-675) for one channel and segment, with each unit's mean
clip as its template.

Inputs may be numpy arrays or CUDA tensors (the pursuit's output left on the
device); clips and templates must be float32, as the pursuit produces them.
The work runs in libfbp.so (csrc/postprocess.cu); results are bit-identical to
the reference's numpy code.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native


def _device(torch, device):
    """A CUDA torch.device from None (the current device), an index or a device."""
    if isinstance(device, torch.device):
        return device
    return torch.device("cuda", torch.cuda.current_device() if device is None else int(device))


def _dev_tensor(torch, x, dtype, dev):
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x)).to(device=dev, dtype=dtype).contiguous()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _check_float32(x, what):
    dt = getattr(x, "dtype", None)
    name = str(dt)
    if dt is not None and not name.endswith("float32"):
        raise TypeError("%s must be float32 (the pursuit's clip type), got %s" % (what, name))


def remove_binary_pursuit_duplicates(event_indices, clips, unit_template, binary_pursuit_bool, tol_inds,
                                     device=None):
    """Keep mask (numpy bool) of one unit's spikes; see the module docstring."""
    import torch

    _check_float32(clips, "clips")
    _check_float32(unit_template, "unit_template")
    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    dev = _device(torch, device)
    n = int(len(event_indices))
    if n == 0:
        return np.ones(0, dtype=bool)
    ev = _dev_tensor(torch, event_indices, torch.int64, dev)
    cl = _dev_tensor(torch, clips, torch.float32, dev).reshape(n, -1)
    tm = _dev_tensor(torch, unit_template, torch.float32, dev).reshape(-1)
    if tm.numel() != cl.shape[1]:
        raise ValueError("unit_template length differs from the clip length")
    bp = _dev_tensor(torch, binary_pursuit_bool, torch.uint8, dev)
    keep = torch.empty(n, dtype=torch.uint8, device=dev)
    L = _native.lib()
    ws = torch.empty(int(L.fbp_bp_duplicates_workspace(n)), dtype=torch.uint8, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(L.fbp_bp_duplicates(_ptr(ev), _ptr(cl), _ptr(tm), _ptr(bp), n, cl.shape[1], int(tol_inds),
                                      _ptr(keep), _ptr(ws), ws.numel(), stream))
    return keep.cpu().numpy().astype(bool)


def mean_clip(clips, device=None):
    """np.mean(clips, axis=0) of float32 clips, on the GPU (bit-identical)."""
    import torch

    _check_float32(clips, "clips")
    dev = _device(torch, device)
    cl = _dev_tensor(torch, clips, torch.float32, dev)
    n = int(cl.shape[0])
    cl = cl.reshape(n, -1)
    out = torch.empty(cl.shape[1], dtype=torch.float32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _native.check(_native.lib().fbp_mean_clip(_ptr(cl), n, cl.shape[1], _ptr(out), stream))
    return out


def remove_segment_duplicates(event_indices, neuron_labels, clips, binary_pursuit_bool, tol_inds, device=None):
    """Keep mask over all spikes of one channel and segment: per unit (labels in
    ascending order) the unit's spikes in their given order, its mean clip as the
    template (postprocessing.py:656-666)."""
    import torch

    labels = np.asarray(neuron_labels.cpu() if isinstance(neuron_labels, torch.Tensor) else neuron_labels)
    keep = np.ones(labels.size, dtype=bool)
    if labels.size == 0:
        return keep
    ev = np.asarray(event_indices.cpu() if isinstance(event_indices, torch.Tensor) else event_indices)
    bp = np.asarray(binary_pursuit_bool.cpu() if isinstance(binary_pursuit_bool, torch.Tensor)
                    else binary_pursuit_bool)
    dev = _device(torch, device)
    cl = clips if isinstance(clips, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(clips))
    _check_float32(cl, "clips")
    cl = cl.to(dev)
    for lab in np.unique(labels):
        sel = np.flatnonzero(labels == lab)
        ucl = cl[torch.as_tensor(sel, device=dev)]
        keep[sel] = remove_binary_pursuit_duplicates(ev[sel], ucl, mean_clip(ucl, dev), bp[sel], tol_inds, dev)
    return keep
