"""The reference's OpenCL kernels on the host CPU, driven by a restated host loop.

TEST INFRASTRUCTURE ONLY: the CPU baseline of bench.py (``--impl reference``
and the cpu_baseline leg).  The kernels are the reference's own
(spikesorting_fullpursuit/kernels/binary_pursuit.cl compiled for the CPU into
oracle/_ref/libbp_ref.so by build_ref.py).  The reference's Python host
function cannot be shipped with this repository, so its per-chunk loop
(spikesorting_fullpursuit/overlap/binary_pursuit_parallel.py:486-1500) is
restated here with the same buffers, launch sizes and host steps
(np.nonzero window lists, per-pass readbacks).  Work-groups run on all host
threads except where the reference's work-items race (fake_pyopencl).
"""
from __future__ import annotations

import os

import numpy as np

import fake_pyopencl as cl
import oracle


def threads() -> int:
    return cl.THREADS


def _buf(arr):
    return cl.Buffer(None, 0, hostbuf=np.ascontiguousarray(arr))


def _launch(kernel, n_items, wg):
    total = int(wg * int(np.ceil(n_items / wg))) if n_items > 0 else 0
    if total:
        cl.enqueue_nd_range_kernel(None, kernel, (total,), (wg,), global_work_offset=(0,))


def pursue_chunk(chunk, templates, tss, thr, W, S, do_overlap, wg):
    """One chunk through the reference kernels; returns (indices, labels, residual buffer)."""
    C, N = chunk.shape
    M = templates.shape[0]
    u32 = np.uint32
    V = _buf(chunk.reshape(-1))
    T = _buf(templates.reshape(-1))
    tssb = _buf(tss)
    thrb = _buf(thr)
    L = _buf(np.zeros(N * M, dtype=np.float32))
    nw = int(np.ceil(N / W))
    count = _buf(np.zeros(1, dtype=np.uint32))
    add_idx = _buf(np.zeros(nw, dtype=np.uint32))
    add_lab = _buf(np.zeros(nw, dtype=np.uint32))
    b_lik = _buf(np.zeros(nw, dtype=np.float32))
    b_lab = _buf(np.zeros(nw, dtype=np.uint32))
    b_idx = _buf(np.zeros(nw, dtype=np.uint32))
    wlist = _buf(np.arange(nw, dtype=np.uint32))
    nextc = _buf(np.zeros(nw, dtype=np.uint8))
    orech = _buf(np.zeros(nw, dtype=np.uint8))
    olist = _buf(np.arange(nw, dtype=np.uint32))
    o_idx = _buf(np.zeros(nw, dtype=np.uint32))
    o_lab = _buf(np.zeros(nw, dtype=np.uint32))
    k_res = cl.Kernel("compute_residual")
    k_lik = cl.Kernel("compute_full_likelihood")
    k_max = cl.Kernel("compute_template_maximum_likelihood")
    k_ov = cl.Kernel("overlap_recheck_indices")
    k_parse = cl.Kernel("parse_overlap_recheck_indices")
    k_chk = cl.Kernel("check_overlap_reassignments")
    k_bp = cl.Kernel("binary_pursuit")
    for i, a in enumerate([V, u32(N), u32(C), T, u32(M), u32(W)]):
        k_res.set_arg(i, a)
    for i, a in enumerate([V, u32(N), u32(C), T, u32(M), u32(W), tssb, wlist, u32(nw), L]):
        k_lik.set_arg(i, a)
    for i, a in enumerate([u32(N), u32(W), u32(0), wlist, u32(nw), b_idx, b_lab, b_lik, nextc, orech,
                           o_idx, o_lab, L, thrb]):
        k_max.set_arg(i, a)
    for i, a in enumerate([V, u32(N), u32(C), T, u32(M), u32(W), olist, u32(nw), b_idx, b_lab, L, u32(S),
                           cl.LocalMemory(4 * wg), cl.LocalMemory(4 * wg)]):
        k_ov.set_arg(i, a)
    k_ov.set_arg(16, thrb)
    for i, a in enumerate([u32(N), u32(M), olist, u32(nw), b_idx, b_lab, b_lik, o_idx, o_lab, L, u32(S), thrb]):
        k_parse.set_arg(i, a)
    k_parse.set_arg(14, orech)
    for i, a in enumerate([u32(N), u32(W), olist, u32(nw), b_idx, b_lab, nextc, o_idx, o_lab, orech]):
        k_chk.set_arg(i, a)
    for i, a in enumerate([u32(N), u32(C), u32(W), thrb, wlist, u32(nw), b_idx, b_lab, b_lik,
                           cl.LocalMemory(4 * wg), count, add_idx, add_lab, orech, nextc]):
        k_bp.set_arg(i, a)
    items = (2 * S + 1) * (2 * S + 1) * M
    n_local = (items - 1) // wg + 1
    leftover = (wg * n_local) % items
    nlist = nw
    found_idx, found_lab = [], []
    while True:
        _launch(k_lik, nlist * M, wg)
        for t in range(M):
            k_max.set_arg(2, u32(t))
            _launch(k_max, nlist, wg)
        flagged = np.nonzero(orech.view(np.uint8))[0].astype(np.uint32)
        if flagged.size and do_overlap:
            olist.view(np.uint32)[: flagged.size] = flagged
            k_ov.set_arg(7, u32(flagged.size))
            k_parse.set_arg(3, u32(flagged.size))
            k_chk.set_arg(3, u32(flagged.size))
            groups = flagged.size * n_local
            gl = _buf(np.zeros(groups, dtype=np.float32))
            gw = _buf(np.zeros(groups, dtype=np.uint32))
            k_ov.set_arg(14, gl)
            k_ov.set_arg(15, gw)
            k_parse.set_arg(12, gl)
            k_parse.set_arg(13, gw)
            _launch(k_ov, flagged.size * items + flagged.size * leftover, wg)
            _launch(k_parse, flagged.size, wg)
            _launch(k_chk, flagged.size, wg)
        _launch(k_bp, nlist, wg)
        n = int(count.view(np.uint32)[0])
        if n == 0:
            break
        orech.view(np.uint8)[:] = 0
        nxt = np.nonzero(nextc.view(np.uint8))[0].astype(np.uint32)
        wlist.view(np.uint32)[: nxt.size] = nxt
        nlist = nxt.size
        k_lik.set_arg(8, u32(nlist))
        k_max.set_arg(4, u32(nlist))
        k_bp.set_arg(5, u32(nlist))
        nextc.view(np.uint8)[:] = 0
        found_idx.append(add_idx.view(np.uint32)[:n].copy())
        found_lab.append(add_lab.view(np.uint32)[:n].copy())
        k_res.set_arg(6, add_idx)
        k_res.set_arg(7, add_lab)
        k_res.set_arg(8, u32(n))
        _launch(k_res, n, wg)
        count.view(np.uint32)[0] = 0
    if found_idx:
        return np.hstack(found_idx), np.hstack(found_lab), V
    return np.zeros(0, np.uint32), np.zeros(0, np.uint32), V


def binary_pursuit(voltage, sort_info, separability_metrics, n_max_shift_inds=None,
                   max_gpu_memory=None, global_mem_size=None, work_group_size=256):
    """Spike indices and labels of the whole recording (no clips)."""
    C, Ns = voltage.shape
    W = int(sort_info["n_samples_per_chan"])
    chan_win, _ = oracle.time_window_to_samples(sort_info["clip_width"], sort_info["sampling_rate"])
    templates = np.float32(separability_metrics["templates"]).reshape(-1, C * W)
    tss = np.float32(-0.5 * separability_metrics["template_SS"])
    thr = np.float32(separability_metrics["neuron_lower_thresholds"])
    S = W // 2 if n_max_shift_inds is None or n_max_shift_inds < 0 else int(n_max_shift_inds)
    onsets, chunk = oracle.plan_chunks(Ns, C, templates.shape[0], W, sort_info["sampling_rate"], S,
                                       global_mem_size or cl.GLOBAL_MEM_SIZE, max_gpu_memory,
                                       work_group_size)
    out_i, out_l = [], []
    for start in onsets:
        stop = min(Ns, start + chunk)
        si, sl, _ = pursue_chunk(np.float32(voltage[:, start:stop]), templates, tss, thr, W, S,
                                 bool(sort_info["do_overlap_recheck"]), work_group_size)
        out_i.append(si.astype(np.int64) + start)
        out_l.append(sl.astype(np.int64))
    if not out_i:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.hstack(out_i) + int(abs(chan_win[0])), np.hstack(out_l)


if __name__ == "__main__":
    print("threads", threads(), "lib", os.path.exists(os.path.join(os.path.dirname(__file__), "_ref", "libbp_ref.so")))
