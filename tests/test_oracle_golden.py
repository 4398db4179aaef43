"""The CPU oracle against the golden vectors made by the reference itself."""
import copy
import hashlib

import numpy as np

import pytest

import oracle
from conftest import golden_names, load_golden, skip_heavy


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _same(got, want):
    return np.array_equal(np.asarray(got), np.asarray(want))


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_outputs(name):
    skip_heavy(name, "end_to_end")
    V, si, sm, call, expect, meta = load_golden(name)
    out = oracle.binary_pursuit(V, np.float32, si, copy.deepcopy(sm),
                                global_mem_size=meta["global_mem_size"],
                                work_group_size=meta["work_group_size"], **call)
    ev, lab, bl, clips = out
    if expect["empty"]:
        assert isinstance(ev, list) and ev == [] and lab == [] and bl == [] and clips == []
        return
    assert _same(ev, expect["event_indices"]), name
    assert _same(lab, expect["neuron_labels"]), name
    assert _same(bl, expect["spike_bool"]), name
    if si["get_adjusted_clips"]:
        assert clips.dtype == np.float32
        assert _same(clips, expect["adjusted_clips"]), name
    else:
        assert np.asarray(clips).size == 0


@pytest.mark.parametrize("name", golden_names())
def test_oracle_chunk_internals(name):
    """First-pass likelihood buffer, final residual and per-pass spike counts."""
    skip_heavy(name, "internals")
    V, si, sm, call, expect, meta = load_golden(name)
    W = si["n_samples_per_chan"]
    S = call.get("n_max_shift_inds")
    if S is None:
        S = W // 2
    M = sm["templates"].shape[0]
    onsets, chunk = ([], 0)
    if V.shape[1] > W:
        onsets, chunk = oracle.plan_chunks(V.shape[1], V.shape[0], M, W, si["sampling_rate"], S,
                                           meta["global_mem_size"], call.get("max_gpu_memory"),
                                           meta["work_group_size"])
    assert len(onsets) == len(meta["chunks"])
    bias = np.float32(-0.5 * sm["template_SS"])
    theta = np.float32(sm["neuron_lower_thresholds"])
    for start, ch in zip(onsets, meta["chunks"]):
        stop = min(V.shape[1], start + chunk)
        cv = np.float32(V[:, start:stop])
        L = oracle.likelihood_all(cv, sm["templates"], bias, W)
        assert _sha(L) == ch["lik_sha256"], name
        si_, sl_, resid, st = oracle.pursue_chunk(cv, sm["templates"], bias, theta, W, S,
                                                  si["do_overlap_recheck"],
                                                  meta["work_group_size"])
        assert st.passes == len(ch["passes"])
        assert int(st.spikes) == sum(ch["passes"])
        if ch["resid_sha256"] is not None:
            assert _sha(resid) == ch["resid_sha256"], name


@pytest.mark.parametrize("name", golden_names())
def test_reference_kernels_with_restated_host_loop(name):
    """oracle/ref_host.py (the CPU baseline of bench.py) reproduces the goldens."""
    import os
    if not os.path.exists(os.path.join(os.path.dirname(oracle.__file__), "_ref", "libbp_ref.so")):
        pytest.skip("oracle/_ref not built")
    import ref_host
    skip_heavy(name, "reference_kernels")
    V, si, sm, call, expect, meta = load_golden(name)
    ev, lab = ref_host.binary_pursuit(V, si, copy.deepcopy(sm), global_mem_size=meta["global_mem_size"],
                                      work_group_size=meta["work_group_size"], **call)
    if expect["empty"]:
        assert ev.size == 0
        return
    assert _same(ev, expect["event_indices"]), name
    assert _same(lab, expect["neuron_labels"]), name
