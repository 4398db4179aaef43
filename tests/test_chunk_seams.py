"""Exact de-duplication of the spikes two chunks both find in their 3-window
overlap (binary_pursuit_parallel.py:498-507 overlaps the chunks; :1491 keeps
both copies).  The host rule on the CPU; the GPU test runs the drop-in on the
multi-chunk golden made by the reference with the option off and on."""
import copy

import numpy as np
import pytest

from conftest import load_golden
from spikesorting_fullpursuit_b200.overlap.binary_pursuit_parallel import seam_duplicates


def test_seam_duplicates_marks_same_index_and_label_in_the_overlap():
    prev_idx = np.array([10, 500, 900, 950, 990])
    prev_lab = np.array([0, 1, 2, 3, 1])
    idx = np.array([900, 950, 950, 991, 1200, 940])
    lab = np.array([2, 1, 3, 1, 0, 2])
    dup = seam_duplicates(prev_idx, prev_lab, idx, lab, seam_start=900)
    assert dup.tolist() == [True, False, True, False, False, False]
    # only spikes at or after the seam count; empty inputs
    assert not seam_duplicates(prev_idx, prev_lab, idx, lab, seam_start=1000).any()
    assert seam_duplicates([], [], idx, lab, 0).tolist() == [False] * idx.size
    assert seam_duplicates(prev_idx, prev_lab, [], [], 0).size == 0


def _split_by_chunk(arr, meta):
    counts = [sum(c["passes"]) for c in meta["chunks"]]
    return np.split(np.asarray(arr), np.cumsum(counts)[:-1])


@pytest.mark.gpu
def test_multichunk_golden_with_and_without_seam_dedupe():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spikesorting_fullpursuit_b200 import binary_pursuit
    V, si, sm, call, expect, meta = load_golden("multichunk_0p6s")
    assert len(meta["chunks"]) > 1
    off = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), verbose=False, **call)
    assert np.array_equal(off[0], expect["event_indices"])
    assert np.array_equal(off[1], expect["neuron_labels"])
    on = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), verbose=False, dedupe_chunk_seams=True, **call)
    # expected: each chunk's spikes minus those (index, label) the previous chunk kept
    ev_c = _split_by_chunk(expect["event_indices"], meta)
    lab_c = _split_by_chunk(expect["neuron_labels"], meta)
    clip_c = _split_by_chunk(expect["adjusted_clips"], meta)
    want_ev, want_lab, want_clips, prev = [], [], [], set()
    for e, l, c in zip(ev_c, lab_c, clip_c):
        keep = np.array([(int(a), int(b)) not in prev for a, b in zip(e, l)], dtype=bool)
        want_ev.append(e[keep]); want_lab.append(l[keep]); want_clips.append(c[keep])
        prev = set(zip(e[keep].tolist(), l[keep].tolist()))
    assert np.array_equal(on[0], np.concatenate(want_ev))
    assert np.array_equal(on[1], np.concatenate(want_lab))
    assert np.array_equal(on[3], np.concatenate(want_clips))
    assert on[2].all() and on[2].size == on[0].size
