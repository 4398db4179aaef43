"""CPU oracle for Full Binary Pursuit's template-matching path.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
``__graft_entry__.smoke()`` and the cpu_baseline leg of ``bench.py`` import it.

``binary_pursuit`` restates the host function of
spikesorting_fullpursuit/overlap/binary_pursuit_parallel.py:175-1532 (chunk
planner, chunk loop, output assembly) over the C restatement of the per-chunk
pursuit in ``bp_oracle.c``.  ``plan_chunks`` restates the device-memory chunk
planner of binary_pursuit_parallel.py:389-507.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libbp_oracle.so")
_lib = None


class BpoParams(ctypes.Structure):
    _fields_ = [("C", ctypes.c_uint32), ("N", ctypes.c_uint32), ("M", ctypes.c_uint32),
                ("W", ctypes.c_uint32), ("S", ctypes.c_uint32), ("WG", ctypes.c_uint32),
                ("do_overlap", ctypes.c_int32), ("threads", ctypes.c_int32)]


class BpoStats(ctypes.Structure):
    _fields_ = [("passes", ctypes.c_int32), ("status", ctypes.c_int32),
                ("spikes", ctypes.c_uint64), ("flagged", ctypes.c_uint64),
                ("overlap_items", ctypes.c_uint64), ("listed", ctypes.c_uint64)]


def build(force: bool = False) -> str:
    """Compile bp_oracle.c into libbp_oracle.so next to it."""
    src = os.path.join(_HERE, "bp_oracle.c")
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(src)):
        return _LIB_PATH
    tmp = _LIB_PATH + ".tmp%d" % os.getpid()
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
                           "-fPIC", "-shared", "-o", tmp, src, "-lm"])
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        L.bpo_pursue_chunk.argtypes = [P(BpoParams), ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_uint64, P(ctypes.c_uint64),
                                       ctypes.c_int32, P(BpoStats)]
        L.bpo_pursue_chunk.restype = ctypes.c_int
        L.bpo_adjusted_clips.argtypes = [P(BpoParams), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                         ctypes.c_void_p]
        L.bpo_likelihood_all.argtypes = [P(BpoParams), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]
        L.bpo_pair_value.argtypes = [P(BpoParams), ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                     ctypes.c_uint32, ctypes.c_uint32]
        L.bpo_pair_value.restype = ctypes.c_float
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def time_window_to_samples(time_window_s, sampling_rate):
    """Restates spikesorting_fullpursuit/processing/conversions.py:4-39."""
    w = list(time_window_s)
    if w[0] > 0:
        w[0] *= -1
    s0 = min(int(round(w[0] * sampling_rate)), 0)
    s1 = max(int(round(w[1] * sampling_rate)), 1) + 1
    return [s0, s1], w


def plan_chunks(n_samples, n_chans, n_templates, template_samples_per_chan, sampling_rate,
                n_max_shift_inds, global_mem_size, max_gpu_memory=None, work_group_size=256,
                address_bits=64):
    """Chunk onsets and length (binary_pursuit_parallel.py:389-507)."""
    W = template_samples_per_chan
    gpu_memory_size = max(global_mem_size * 0.5, global_mem_size - (1024 * 1024 * 1024))
    if max_gpu_memory is not None:
        gpu_memory_size = min(gpu_memory_size, max_gpu_memory)
    assert gpu_memory_size > 0
    S = int(n_max_shift_inds)
    items_per_index = np.int64((2 * S + 1) * (2 * S + 1) * n_templates)
    n_local_ID = np.int64(((items_per_index - 1) / np.int64(work_group_size)) + 1)
    constant_memory_usage = n_templates * n_chans * W * 4 + n_templates * 4
    n_chans_u = np.uint32(n_chans)
    usage = n_chans_u * sampling_rate * 4
    usage += n_templates * sampling_rate * 4
    usage += (sampling_rate / W) * (4 + 4 + 4 + 4 + 4 + (n_local_ID / 3) * 4 + (n_local_ID / 3) * 4)
    seconds = (gpu_memory_size - constant_memory_usage) / usage
    max_addr_seconds = ((1 << address_bits) - 1) / (4 * sampling_rate * n_chans_u)
    seconds = min(seconds, np.floor(max_addr_seconds))
    chunk = int(np.floor(seconds * sampling_rate))
    if chunk < 4 * W:
        raise ValueError("Cannot fit enough data on GPU to run binary pursuit. "
                         "Decrease template samples or get a new GPU.")
    onsets = []
    cur = 0
    while cur < n_samples - W:
        onsets.append(cur)
        cur += chunk - 3 * W
    return onsets, chunk


def pursue_chunk(chunk_voltage, templates, bias, theta, W, S, do_overlap=True,
                 work_group_size=256, threads=None, max_passes=0):
    """Run the per-chunk pursuit on one float32 C x N chunk.

    Returns (spike_indices uint32, spike_labels uint32, residual, stats)."""
    V = np.ascontiguousarray(chunk_voltage, dtype=np.float32).copy()
    C, N = V.shape
    T = np.ascontiguousarray(templates, dtype=np.float32).reshape(-1)
    M = T.size // (C * W)
    b = np.ascontiguousarray(bias, dtype=np.float32)
    th = np.ascontiguousarray(theta, dtype=np.float32)
    nw = (N + W - 1) // W
    cap = max(64, nw * 64)
    idx = np.zeros(cap, dtype=np.uint32)
    lab = np.zeros(cap, dtype=np.uint32)
    p = BpoParams(C, N, M, W, S, work_group_size, 1 if do_overlap else 0,
                  threads or os.cpu_count() or 1)
    n = ctypes.c_uint64(0)
    st = BpoStats()
    rc = lib().bpo_pursue_chunk(ctypes.byref(p), _ptr(V), _ptr(T), _ptr(b), _ptr(th), _ptr(idx),
                                _ptr(lab), cap, ctypes.byref(n), int(max_passes), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle pursuit failed with status %d" % rc)
    return idx[:n.value].copy(), lab[:n.value].copy(), V, st


def adjusted_clips(residual_v, templates, spike_idx, spike_lab, W):
    V = np.ascontiguousarray(residual_v, dtype=np.float32)
    C, N = V.shape
    T = np.ascontiguousarray(templates, dtype=np.float32).reshape(-1)
    M = T.size // (C * W)
    si = np.ascontiguousarray(spike_idx, dtype=np.uint32)
    sl = np.ascontiguousarray(spike_lab, dtype=np.uint32)
    out = np.zeros((si.size, C * W), dtype=np.float32)
    p = BpoParams(C, N, M, W, 0, 256, 0, 1)
    lib().bpo_adjusted_clips(ctypes.byref(p), _ptr(V), _ptr(T), _ptr(si), _ptr(sl), si.size, _ptr(out))
    return out


def likelihood_all(chunk_voltage, templates, bias, W, threads=None):
    """First-pass likelihood L[M, N] of one chunk (compute_full_likelihood)."""
    V = np.ascontiguousarray(chunk_voltage, dtype=np.float32)
    C, N = V.shape
    T = np.ascontiguousarray(templates, dtype=np.float32).reshape(-1)
    M = T.size // (C * W)
    b = np.ascontiguousarray(bias, dtype=np.float32)
    L = np.zeros((M, N), dtype=np.float32)
    p = BpoParams(C, N, M, W, 0, 256, 0, threads or os.cpu_count() or 1)
    lib().bpo_likelihood_all(ctypes.byref(p), _ptr(V), _ptr(T), _ptr(b), _ptr(L))
    return L


def pair_value(chunk_voltage, templates, W, S, f, t, p, a, b):
    V = np.ascontiguousarray(chunk_voltage, dtype=np.float32)
    C, N = V.shape
    T = np.ascontiguousarray(templates, dtype=np.float32).reshape(-1)
    M = T.size // (C * W)
    prm = BpoParams(C, N, M, W, S, 256, 1, 1)
    return float(lib().bpo_pair_value(ctypes.byref(prm), _ptr(V), _ptr(T), f, t, p, a, b))


def binary_pursuit(voltage, v_dtype, sort_info, separability_metrics, n_max_shift_inds=None,
                   kernels_path=None, max_gpu_memory=None, *, global_mem_size=None,
                   work_group_size=256, threads=None, return_stats=False):
    """Restatement of binary_pursuit() (binary_pursuit_parallel.py:175-1532) on the CPU."""
    del kernels_path
    n_chans = int(voltage.shape[0])
    n_samples = int(voltage.shape[1])
    sampling_rate = sort_info["sampling_rate"]
    chan_win, _ = time_window_to_samples(sort_info["clip_width"], sampling_rate)
    W = int(sort_info["n_samples_per_chan"])
    templates = separability_metrics["templates"]
    if templates.ndim == 1:
        templates = np.reshape(templates, (1, -1))
    templates = np.float32(templates)
    M = templates.shape[0]
    clip_init_samples = int(np.abs(chan_win[0]))
    bias = np.float32(-0.5 * separability_metrics["template_SS"])
    theta = np.float32(separability_metrics["neuron_lower_thresholds"])
    if n_max_shift_inds is None or n_max_shift_inds < 0:
        n_max_shift_inds = W // 2
    S = int(np.uint32(n_max_shift_inds))
    if global_mem_size is None:
        global_mem_size = 8 * 1024 ** 3
    onsets, chunk = plan_chunks(n_samples, n_chans, M, W, sampling_rate, S, global_mem_size,
                                max_gpu_memory, work_group_size)
    idx_all, lab_all, bool_all, clips_all, stats = [], [], [], [], []
    for start in onsets:
        stop = int(np.uint32(min(n_samples, start + chunk)))
        cv = np.float32(voltage[:, start:stop])
        si, sl, resid, st = pursue_chunk(cv, templates, bias, theta, W, S,
                                         bool(sort_info["do_overlap_recheck"]),
                                         work_group_size, threads)
        stats.append(st)
        if si.size == 0:
            continue
        if sort_info["get_adjusted_clips"]:
            clips = adjusted_clips(resid, templates, si, sl, W)
        else:
            clips = []
        idx_all.append(si.astype(np.int64) + start)
        lab_all.append(sl)
        clips_all.append(clips)
        bool_all.append(np.ones(si.size, dtype=bool))
    if idx_all:
        event_indices = np.int64(np.hstack(idx_all))
        neuron_labels = np.int64(np.hstack(lab_all))
        adjusted = np.vstack(clips_all).astype(v_dtype)
        spike_bool = np.hstack(bool_all)
        event_indices += clip_init_samples
    else:
        event_indices, neuron_labels, spike_bool, adjusted = [], [], [], []
    separability_metrics["n_spikes"] = np.zeros(M)
    for n in range(M):
        separability_metrics["n_spikes"][n] = np.count_nonzero(np.asarray(neuron_labels) == n)
    out = (event_indices, neuron_labels, spike_bool, adjusted)
    if return_stats:
        return out, stats
    return out
