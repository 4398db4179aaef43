"""Launch-shape autotuner for the pursuit, cached per chunk shape and device.

The library picks its launch shapes from the sizes alone (include/fbp.h,
fbp_tuning): 128-sample tiles per tensor-core likelihood CTA, template steps
per staged copy, staged copies in flight, and templates per
partial-correlation CTA.  ``tune`` measures candidates on the caller's own
data -- a leading slice of the voltage with the real templates -- and keeps
the fastest: first the likelihood shapes, by the likelihood kernel's device
time within whole pursuits of the slice (the pass-by-pass window lists of a
real pursuit), then the partial-correlation group, by whole pursuits.  Results are cached in a JSON file
(``FBP_TUNE_CACHE``, else ~/.cache/spikesorting_fullpursuit_b200/tuning.json)
keyed by (channels, templates, window, shift, device name), so each shape is
measured once.  Launch shapes change speed only: every candidate gives the
same spikes.
"""
from __future__ import annotations

import ctypes
import json
import os
import threading

import numpy as np

from . import _native

_LOCK = threading.Lock()
FIELDS = ("lik_tiles", "lik_group", "lik_stages", "pc_group", "lik_epi")


def cache_path():
    p = os.environ.get("FBP_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "spikesorting_fullpursuit_b200", "tuning.json")


def _load():
    try:
        with open(cache_path()) as fp:
            return json.load(fp)
    except (OSError, ValueError):
        return {}


def _store(key, value):
    with _LOCK:
        d = _load()
        d[key] = value
        path = cache_path()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp%d" % os.getpid()
        with open(tmp, "w") as fp:
            json.dump(d, fp, indent=1, sort_keys=True)
        os.replace(tmp, path)


def key_of(C, M, W, S, device_name):
    return "C%d-M%d-W%d-S%d-%s" % (C, M, W, S, device_name)


def apply(tuning):
    """Set the calling thread's launch shapes (dict with FIELDS, or None)."""
    if tuning is None:
        _native.check(_native.lib().fbp_set_tuning(None))
        return
    t = _native.FbpTuning(*[int(tuning.get(f, 0)) for f in FIELDS])
    _native.check(_native.lib().fbp_set_tuning(ctypes.byref(t)))


def _ptr(x):
    return ctypes.c_void_p(x.data_ptr())


def _time(torch, fn, reps=3):
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = None
    for _ in range(reps):
        ev0.record()
        fn()
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        best = ms if best is None or ms < best else best
    return best


def lik_candidates(M):
    """Likelihood launch shapes to measure: the persistent kernel (lik_tiles 0)
    with 1 to 4 epilogue warpgroups, then per-CTA tile counts."""
    Np = (M + 15) // 16 * 16
    out = [{"lik_tiles": 0, "lik_epi": e, "lik_stages": st, "lik_group": 0, "pc_group": 0}
           for e in (2, 3, 1, 4) for st in (0, 4)]
    tiles = tuple(k for k in (2, 4, 1) if k * Np <= 512)
    for lt in tiles:
        for st in (0, 4, 6):
            for g in (0, 2, 8):
                out.append({"lik_tiles": lt, "lik_stages": st, "lik_group": g, "pc_group": 0, "lik_epi": 0})
    return out


def tune(voltage, templates, bias, theta, W, S, overlap=True, sample_s=None, sampling_rate=None, device=None,
         use_cache=True):
    """Fastest launch shapes for pursuing chunks of this shape (a dict of FIELDS).

    voltage: C x N array (host or CUDA); templates M x (C*W); bias, theta [M].
    The first ``sample_s`` seconds (default: up to 240,000 samples) are measured."""
    import torch

    dev = device if isinstance(device, torch.device) else torch.device(
        "cuda", torch.cuda.current_device() if device is None else int(device))
    C = int(voltage.shape[0])
    M = int(np.asarray(templates).shape[0])
    key = key_of(C, M, W, S, torch.cuda.get_device_name(dev))
    if use_cache:
        hit = _load().get(key)
        if hit is not None:
            return hit
    n = int(voltage.shape[1])
    if sample_s is not None and sampling_rate:
        n = min(n, max(4 * W, int(sample_s * sampling_rate)))
    else:
        n = min(n, 240000)
    V0 = voltage[:, :n] if isinstance(voltage, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(voltage[:, :n], dtype=np.float32))
    V0 = V0.to(dev, torch.float32).contiguous()
    T = torch.from_numpy(np.ascontiguousarray(templates, dtype=np.float32)).to(dev)
    b = torch.from_numpy(np.ascontiguousarray(bias, dtype=np.float32)).to(dev)
    th = torch.from_numpy(np.ascontiguousarray(theta, dtype=np.float32)).to(dev)
    L = _native.lib()
    d = _native.dims(C, n, M, W, S)
    flags = _native.FBP_OVERLAP_RECHECK if overlap else 0
    ws = torch.empty(_native.workspace_bytes(d, flags), dtype=torch.uint8, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    Vw = torch.empty_like(V0)
    cap = 8 * (n // W + 1) + 1024
    idx = torch.empty(cap, dtype=torch.int32, device=dev)
    lab = torch.empty(cap, dtype=torch.int32, device=dev)

    def run_pursuit(timing):
        Vw.copy_(V0)
        k = ctypes.c_uint32(0)
        st = _native.FbpChunkStats()
        _native.check(L.fbp_pursue_chunk(ctypes.byref(d), flags | (_native.FBP_TIMING if timing else 0), _ptr(Vw),
                                         _ptr(T), _ptr(b), _ptr(th), _ptr(ws), ws.numel(), _ptr(idx), _ptr(lab), cap,
                                         ctypes.byref(k), ctypes.byref(st), _native.MAX_PASSES, stream))
        return st

    best, best_ms = None, None
    try:
        for cand in lik_candidates(M):
            apply(cand)
            ms = min(run_pursuit(True).ms_lik_tc for _ in range(2))
            if best_ms is None or ms < best_ms:
                best, best_ms = dict(cand), ms
        if overlap:
            pbest, pbest_ms = None, None
            for q in (0, 8, 4, 2):
                cand = dict(best, pc_group=q)
                apply(cand)
                run_pursuit(False)
                ms = _time(torch, lambda: run_pursuit(False), reps=2)
                if pbest_ms is None or ms < pbest_ms:
                    pbest, pbest_ms = cand, ms
            best = pbest
    finally:
        apply(None)
    if use_cache:
        _store(key, best)
    return best
