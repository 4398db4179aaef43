"""Drop-in binary_pursuit() on a B200.

Same signature, arguments, return values and side effect as
spikesorting_fullpursuit.overlap.binary_pursuit_parallel.binary_pursuit
(binary_pursuit_parallel.py:175-1532):

    binary_pursuit(voltage, v_dtype, sort_info, separability_metrics,
                   n_max_shift_inds=None, kernels_path=None, max_gpu_memory=None)
      -> (event_indices int64[n], neuron_labels int64[n],
          binary_pursuit_spike_bool bool[n], adjusted_clips)

The pursuit of each chunk runs in libfbp.so (hand-written sm_100a CUDA behind
the C ABI of include/fbp.h) on PyTorch-owned device buffers.  Chunking follows
the reference's device-memory planner with this GPU's memory, so chunk
boundaries (and the duplicate spikes the reference leaves in the 3W chunk
overlaps) are the reference's.  Results equal the reference kernels run with
their work-groups in order: where the reference's outcome depends on which
work-item runs first, the outcome of in-order execution is the one reproduced.

Differences, all documented:
* ``kernels_path`` is accepted and ignored (there is no OpenCL source).
* If the first pass of a chunk flags no window for the overlap recheck the
  reference raises UnboundLocalError (binary_pursuit_parallel.py:1369-1371
  releases buffers it never created); this implementation returns the empty
  result it was meant to return.
* The reference's pass loop has no limit (binary_pursuit_parallel.py:907);
  here a chunk that still adds spikes after ``max_passes`` passes raises
  FbpError (status FBP_E_PASSES) instead of running on.
* Keyword-only extras: ``mode`` ("fast": tensor-core likelihood and screened
  overlap recheck, both exact; "plain": scalar FP32 kernels), ``device``,
  ``work_group_size`` (the reference's kernel work-group size, 256, whose
  execution order the results follow), ``max_passes``,
  ``dedupe_chunk_seams`` (drop a chunk's spikes that the previous chunk found
  with the same index and label in their 3-window overlap; off by default,
  where the output is the reference's, duplicates included), ``tuning``
  (launch shapes: None for the library's, "auto" to measure them on the first
  chunk with spikesorting_fullpursuit_b200.autotune, or a dict), ``verbose``,
  ``return_stats``.
"""
from __future__ import annotations

import ctypes
import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .. import _native, autotune
from ..processing.conversions import time_window_to_samples

WORK_GROUP_SIZE = 256
MAX_PASSES = _native.MAX_PASSES   # default pass limit of one chunk
MAX_CAPACITY_RETRIES = 4   # re-runs of a chunk whose spikes outgrew the output buffers
CAPACITY_PER_WINDOW = 16   # spike slots of a chunk's first attempt, per window ...
CAPACITY_EXTRA = 1024      # ... plus these


def plan_chunks(n_samples, n_chans, n_templates, template_samples_per_chan, sampling_rate,
                n_max_shift_inds, global_mem_size, max_gpu_memory=None,
                work_group_size=WORK_GROUP_SIZE, address_bits=64):
    """Chunk onsets and chunk length from the device-memory budget.

    Follows binary_pursuit_parallel.py:389-475 (budget per second of data:
    voltage, likelihood, per-window buffers and the overlap group buffers) and
    :498-507 (onsets overlap by 3 windows).  Arithmetic types follow the
    reference so the floor() lands on the same sample count."""
    W = int(template_samples_per_chan)
    budget = max(global_mem_size * 0.5, global_mem_size - (1024 * 1024 * 1024))
    if max_gpu_memory is not None:
        budget = min(budget, max_gpu_memory)
    assert budget > 0
    S = int(n_max_shift_inds)
    items = np.int64((2 * S + 1) * (2 * S + 1) * n_templates)
    groups = np.int64(((items - 1) / np.int64(work_group_size)) + 1)
    fixed = n_templates * n_chans * W * 4 + n_templates * 4
    chans = np.uint32(n_chans)
    per_second = chans * sampling_rate * 4
    per_second += n_templates * sampling_rate * 4
    per_second += (sampling_rate / W) * (5 * 4 + (groups / 3) * 4 + (groups / 3) * 4)
    seconds = (budget - fixed) / per_second
    seconds = min(seconds, np.floor(((1 << address_bits) - 1) / (4 * sampling_rate * chans)))
    chunk = int(np.floor(seconds * sampling_rate))
    if chunk < 4 * W:
        raise ValueError("Cannot fit enough data on GPU to run binary pursuit. "
                         "Decrease template samples or get a new GPU.")
    onsets = []
    onset = 0
    while onset < n_samples - W:
        onsets.append(onset)
        onset += chunk - 3 * W
    return onsets, chunk


def seam_duplicates(prev_idx, prev_lab, idx, lab, seam_start):
    """Which of a chunk's spikes the previous chunk already found.

    Chunks overlap by 3 windows (binary_pursuit_parallel.py:498-507) and the
    reference keeps the spikes both chunks find in the overlap
    (binary_pursuit_parallel.py:1491, left to later post-processing).  A spike of
    this chunk at or after ``seam_start`` (the chunk's onset) is a duplicate when
    the previous chunk has a spike with the same index and label.  Indices are
    absolute sample indices; returns a boolean mask over ``idx``."""
    idx = np.asarray(idx, dtype=np.int64)
    lab = np.asarray(lab, dtype=np.int64)
    prev_idx = np.asarray(prev_idx, dtype=np.int64)
    prev_lab = np.asarray(prev_lab, dtype=np.int64)
    dup = np.zeros(idx.size, dtype=bool)
    if idx.size == 0 or prev_idx.size == 0:
        return dup
    sel = prev_idx >= seam_start
    width = int(max(lab.max(initial=0), prev_lab.max(initial=0))) + 1
    prev_keys = np.unique(prev_idx[sel] * width + prev_lab[sel])
    mine = idx >= seam_start
    dup[mine] = np.isin(idx[mine] * width + lab[mine], prev_keys, assume_unique=False)
    return dup


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class _Uploader:
    """Host -> device copy of voltage chunks through pinned staging slabs.

    Host threads convert and copy pieces of the chunk (one channel row range
    each) into page-locked slabs while the copy engine moves the previous
    pieces to the device on a stream of its own; ``upload`` makes the caller's
    stream wait for the last piece.  The source may be any real dtype and any
    row-strided view: the float32 conversion happens in the slab copy."""

    SLAB_FLOATS = 2 << 20    # 8 MB per slab
    N_SLABS = 32
    N_THREADS = max(1, min(16, os.cpu_count() or 2))
    RANGE_SAMPLES = 2 << 20  # staged upload: samples of every channel per ready range

    def __init__(self, torch, dev):
        self.torch = torch
        self.dev = dev
        self.slabs = None
        self.events = [None] * self.N_SLABS
        self.stream = torch.cuda.Stream(dev)
        self.pool = ThreadPoolExecutor(self.N_THREADS)

    def upload(self, host, dst):
        torch = self.torch
        self._ensure_slabs()
        C, N = host.shape
        step = self.SLAB_FLOATS
        pieces = [(c, a, min(N, a + step)) for c in range(C) for a in range(0, N, step)]
        caller = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(caller)   # dst may still be read by earlier work
        half = self.N_SLABS // 2
        for w0 in range(0, len(pieces), half):
            wave = pieces[w0:w0 + half]
            slots = [((w0 // half) % 2) * half + k for k in range(len(wave))]
            for k in slots:
                if self.events[k] is not None:
                    self.events[k].synchronize()

            def fill(job):
                (c, a, b), k = job
                np.copyto(self.slabs[k].numpy()[:b - a], host[c, a:b], casting="unsafe")

            list(self.pool.map(fill, zip(wave, slots)))
            with torch.cuda.stream(self.stream):
                for (c, a, b), k in zip(wave, slots):
                    dst[c, a:b].copy_(self.slabs[k][:b - a], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(self.stream)
                    self.events[k] = ev
        caller.wait_stream(self.stream)

    def _ensure_slabs(self):
        if self.slabs is None:
            self.slabs = [self.torch.empty(self.SLAB_FLOATS, dtype=self.torch.float32, pin_memory=True)
                          for _ in range(self.N_SLABS)]

    def start_staged(self, host, dst):
        """Upload ``host`` on a host thread, time range by time range.

        Returns (events, upto, flags, finish): events[k] completes once samples
        [0, upto[k]) of every channel are in ``dst``; flags[k] turns 1 once events[k]
        is recorded (the library waits for it before waiting on the event);
        ``finish()`` joins the thread and re-raises its error, if any."""
        torch = self.torch
        self._ensure_slabs()
        C, N = host.shape
        span = min(self.RANGE_SAMPLES, self.SLAB_FLOATS)
        ranges = [(a, min(N, a + span)) for a in range(0, N, span)]
        events = [torch.cuda.Event() for _ in ranges]
        flags = np.zeros(len(ranges), dtype=np.uint32)
        upto = np.array([b for _, b in ranges], dtype=np.uint32)
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))   # dst may still be read by earlier work
        for ev in events:   # creates the CUDA events (torch makes them at the first record)
            ev.record(self.stream)
        half = self.N_SLABS // 2
        failure = []

        def run():
            try:
                with torch.cuda.device(self.dev):
                    wave_no = 0
                    for k, (a, b) in enumerate(ranges):
                        pieces = [(c, a, b) for c in range(C)]
                        for w0 in range(0, len(pieces), half):
                            wave = pieces[w0:w0 + half]
                            slots = [(wave_no % 2) * half + j for j in range(len(wave))]
                            wave_no += 1
                            for j in slots:
                                if self.events[j] is not None:
                                    self.events[j].synchronize()

                            def fill(job):
                                (c, x0, x1), j = job
                                np.copyto(self.slabs[j].numpy()[:x1 - x0], host[c, x0:x1], casting="unsafe")

                            list(self.pool.map(fill, zip(wave, slots)))
                            with torch.cuda.stream(self.stream):
                                for (c, x0, x1), j in zip(wave, slots):
                                    dst[c, x0:x1].copy_(self.slabs[j][:x1 - x0], non_blocking=True)
                                    ev = torch.cuda.Event()
                                    ev.record(self.stream)
                                    self.events[j] = ev
                        events[k].record(self.stream)
                        flags[k] = 1
            except BaseException as e:   # the library must not wait for ranges that never come
                failure.append(e)
                with torch.cuda.device(self.dev):
                    for k in range(len(ranges)):
                        if not flags[k]:
                            events[k].record(self.stream)
                            flags[k] = 1

        th = threading.Thread(target=run, daemon=True)
        th.start()

        def finish():
            th.join()
            torch.cuda.current_stream(self.dev).wait_stream(self.stream)
            if failure:
                raise failure[0]

        return events, upto, flags, finish

    def close(self):
        self.pool.shutdown(wait=True)


class _Pursuer:
    """Device buffers and the C-ABI calls for one binary_pursuit() call."""

    def __init__(self, torch, dev, n_chans, templates, bias, theta, W, S, max_chunk, flags,
                 work_group_size, max_passes, tuning=None):
        self.torch = torch
        self.dev = dev
        self.C, self.W, self.S = n_chans, W, S
        self.M = templates.shape[0]
        self.flags = flags
        self.wg = work_group_size
        self.max_passes = int(max_passes)
        self.T = torch.from_numpy(np.ascontiguousarray(templates, dtype=np.float32)).to(dev)
        self.bias = torch.from_numpy(np.ascontiguousarray(bias, dtype=np.float32)).to(dev)
        self.theta = torch.from_numpy(np.ascontiguousarray(theta, dtype=np.float32)).to(dev)
        d = _native.dims(n_chans, max_chunk, self.M, W, S, work_group_size)
        nbytes = _native.workspace_bytes(d, flags)
        if nbytes == 0:
            raise ValueError("invalid binary pursuit sizes for the GPU library")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.V = torch.empty((n_chans, max_chunk), dtype=torch.float32, device=dev)
        self.up = _Uploader(torch, dev)
        self.tuning = tuning
        self.stats = []

    def chunk(self, host_chunk, clips):
        """Pursue one chunk (``host_chunk``: C x N view of the caller's voltage)."""
        torch = self.torch
        C, N = host_chunk.shape
        d = _native.dims(C, N, self.M, self.W, self.S, self.wg)
        V = self.V[:, :N] if N == self.V.shape[1] else self.V.view(-1)[:C * N].view(C, N)
        # the first pass runs behind the upload unless the autotuner must see the voltage first
        ready = None
        if self.tuning == "auto":
            self.up.upload(host_chunk, V)
        else:
            ready = self.up.start_staged(host_chunk, V)
        nw = (N + self.W - 1) // self.W
        # every pass adds at most one spike per window; dense probes end with about five
        # spikes per window, so the first attempt holds 16 (8 B each, far below the
        # likelihood's 4*M*W bytes per window) and a capacity retry, which pursues the
        # chunk again, stays rare
        most = nw * self.max_passes if self.max_passes > 0 else 0xFFFFFFFF
        cap = min(CAPACITY_PER_WINDOW * nw + CAPACITY_EXTRA, most, 0xFFFFFFFF)
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        L = _native.lib()
        if self.tuning == "auto":
            self.tuning = autotune.tune(V, self.T.cpu().numpy(), self.bias.cpu().numpy(), self.theta.cpu().numpy(),
                                        self.W, self.S, overlap=bool(self.flags & _native.FBP_OVERLAP_RECHECK),
                                        device=self.dev)
        autotune.apply(self.tuning)
        try:
            return self._pursue(host_chunk, clips, V, d, N, nw, most, cap, stream, L, ready)
        finally:
            autotune.apply(None)

    def _pursue(self, host_chunk, clips, V, d, N, nw, most, cap, stream, L, ready=None):
        torch = self.torch
        C = V.shape[0]
        for attempt in range(MAX_CAPACITY_RETRIES + 1):
            idx = torch.empty(cap, dtype=torch.int32, device=self.dev)
            lab = torch.empty(cap, dtype=torch.int32, device=self.dev)
            n = ctypes.c_uint32(0)
            st = _native.FbpChunkStats()
            if ready is not None:
                events, upto, flags, finish = ready
                ready = None
                evp = (ctypes.c_void_p * len(events))(*[e.cuda_event for e in events])
                try:
                    rc = L.fbp_pursue_chunk_staged(ctypes.byref(d), self.flags, _ptr(V), _ptr(self.T),
                                                   _ptr(self.bias), _ptr(self.theta), _ptr(self.ws),
                                                   self.ws.numel(), _ptr(idx), _ptr(lab), cap, ctypes.byref(n),
                                                   ctypes.byref(st), self.max_passes, evp,
                                                   upto.ctypes.data_as(ctypes.c_void_p),
                                                   flags.ctypes.data_as(ctypes.c_void_p), len(events), stream)
                finally:
                    finish()
            else:
                rc = L.fbp_pursue_chunk(ctypes.byref(d), self.flags, _ptr(V), _ptr(self.T),
                                        _ptr(self.bias), _ptr(self.theta), _ptr(self.ws),
                                        self.ws.numel(), _ptr(idx), _ptr(lab), cap, ctypes.byref(n),
                                        ctypes.byref(st), self.max_passes, stream)
            if rc != _native.FBP_E_CAPACITY:
                break
            if cap >= min(most, 0xFFFFFFFF) or attempt == MAX_CAPACITY_RETRIES:
                _native.check(rc)
            # n holds a lower bound of what the chunk needs; the voltage was partly pursued
            cap = int(min(max(4 * cap, 2 * n.value), most, 0xFFFFFFFF))
            self.up.upload(host_chunk, V)
        self.stats.append(st.as_dict())
        _native.check(rc)
        k = n.value
        out_clips = []
        if clips and k > 0:
            cl = torch.zeros((k, C * self.W), dtype=torch.float32, device=self.dev)
            _native.check(L.fbp_adjusted_clips(ctypes.byref(d), _ptr(V), _ptr(self.T), _ptr(idx),
                                               _ptr(lab), k, _ptr(cl), stream))
            out_clips = cl.cpu().numpy()
        si = idx[:k].cpu().numpy().view(np.uint32)
        sl = lab[:k].cpu().numpy().view(np.uint32)
        return si, sl, out_clips

    def close(self):
        self.up.close()


def binary_pursuit(voltage, v_dtype, sort_info, separability_metrics, n_max_shift_inds=None,
                   kernels_path=None, max_gpu_memory=None, *, mode="fast", device=None,
                   work_group_size=WORK_GROUP_SIZE, max_passes=MAX_PASSES,
                   dedupe_chunk_seams=False, tuning=None, verbose=True, return_stats=False):
    """Find template spikes in ``voltage`` by binary pursuit on the GPU.

    See the module docstring for the contract; the arguments mean what they
    mean for the reference function (binary_pursuit_parallel.py:175-183)."""
    import torch

    del kernels_path
    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    _native.lib()
    dev = (device if isinstance(device, torch.device)
           else torch.device("cuda", torch.cuda.current_device() if device is None else int(device)))
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
    total_mem = torch.cuda.get_device_properties(dev).total_memory
    onsets, chunk_len = plan_chunks(n_samples, n_chans, M, W, sampling_rate, S, total_mem,
                                    max_gpu_memory, work_group_size)
    flags = _native.FBP_OVERLAP_RECHECK if sort_info["do_overlap_recheck"] else 0
    if mode == "plain":
        flags |= _native.FBP_PLAIN_FP32
    elif mode != "fast":
        raise ValueError("mode must be 'fast' or 'plain'")
    get_clips = bool(sort_info["get_adjusted_clips"])
    idx_all, lab_all, bool_all, clips_all = [], [], [], []
    pursuer = None
    if onsets:
        max_chunk = min(n_samples, chunk_len)
        pursuer = _Pursuer(torch, dev, n_chans, templates, bias, theta, W, S, max_chunk, flags,
                           work_group_size, max_passes, tuning)
    try:
        for start in onsets:
            stop = int(np.uint32(min(n_samples, start + chunk_len)))
            si, sl, clips = pursuer.chunk(voltage[:, start:stop], get_clips)
            if si.size == 0:
                continue
            ab = si.astype(np.int64) + start
            if dedupe_chunk_seams and idx_all:
                keep = ~seam_duplicates(idx_all[-1], lab_all[-1], ab, sl, start)
                ab, sl = ab[keep], sl[keep]
                if get_clips and len(clips):
                    clips = clips[keep]
                if ab.size == 0:
                    continue
            idx_all.append(ab)
            lab_all.append(sl)
            clips_all.append(clips)
            bool_all.append(np.ones(ab.size, dtype=bool))
    finally:
        if pursuer is not None:
            pursuer.close()
    if idx_all:
        event_indices = np.int64(np.hstack(idx_all))
        neuron_labels = np.int64(np.hstack(lab_all))
        adjusted_clips = np.vstack(clips_all).astype(v_dtype)
        spike_bool = np.hstack(bool_all)
        event_indices += clip_init_samples
        if verbose:
            print("Found a total of", np.count_nonzero(spike_bool), "secret spikes", flush=True)
    else:
        event_indices, neuron_labels, spike_bool, adjusted_clips = [], [], [], []
        if verbose:
            print("Found a total of ZERO secret spikes", flush=True)
    # side effect of add_n_spikes (neuron_separability.py:334-345)
    labels_arr = np.asarray(neuron_labels, dtype=np.int64)
    counts = np.bincount(labels_arr, minlength=M)[:M] if labels_arr.size else np.zeros(M, dtype=np.int64)
    separability_metrics["n_spikes"] = counts.astype(np.float64)
    out = (event_indices, neuron_labels, spike_bool, adjusted_clips)
    if return_stats:
        return out, (pursuer.stats if pursuer else [])
    return out
