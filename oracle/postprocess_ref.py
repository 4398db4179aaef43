"""CPU restatement of the reference's post-pursuit duplicate removal.

TEST INFRASTRUCTURE ONLY: the checker for csrc/postprocess.cu.

``remove_binary_pursuit_duplicates`` restates
spikesorting_fullpursuit/analyze_spike_timing.py:148-193 (the sequential walk
over one unit's spikes); ``remove_segment_duplicates`` restates the per-unit
loop of WorkItemSummary.remove_segment_binary_pursuit_duplicates
(spikesorting_fullpursuit/postprocessing.py:646-675) for one channel and
segment.  numpy does the float32 arithmetic, as in the reference.
"""
from __future__ import annotations

import numpy as np


def remove_binary_pursuit_duplicates(event_indices, clips, unit_template, binary_pursuit_bool, tol_inds):
    ev = np.asarray(event_indices)
    bp = np.asarray(binary_pursuit_bool, dtype=bool)
    keep = np.ones(ev.size, dtype=bool)
    cur, nxt = 0, 1
    while nxt < ev.size:
        if ev[nxt] - ev[cur] <= tol_inds:
            if bp[cur] and bp[nxt]:
                s_cur = np.sum((clips[cur, :] - unit_template) ** 2)
                s_nxt = np.sum((clips[nxt, :] - unit_template) ** 2)
                if s_cur <= s_nxt:
                    keep[nxt] = False
                    nxt += 1
                else:
                    keep[cur] = False
                    cur = nxt
                    nxt += 1
            elif bp[cur] and not bp[nxt]:
                nxt += 1
            else:
                cur = nxt
                nxt += 1
        else:
            cur = nxt
            nxt += 1
    return keep


def remove_segment_duplicates(event_indices, neuron_labels, clips, binary_pursuit_bool, tol_inds):
    labels = np.asarray(neuron_labels)
    keep = np.ones(labels.size, dtype=bool)
    for lab in np.unique(labels):
        sel = labels == lab
        keep[sel] = remove_binary_pursuit_duplicates(np.asarray(event_indices)[sel], clips[sel, :],
                                                     np.mean(clips[sel, :], axis=0),
                                                     np.asarray(binary_pursuit_bool)[sel], tol_inds)
    return keep
