"""The C oracle against the reference's own kernels on random small recordings.

The goldens pin the oracle on fixed cases made by the reference's unmodified
host code.  Here the reference's kernels (binary_pursuit.cl compiled for the
CPU into oracle/_ref, driven by the restated host loop oracle/ref_host.py) and
the oracle (oracle/bp_oracle.c) pursue the same seeded recordings over a
spread of shapes: 1 to 16 channels, 30 or 40 kHz, 1 to 10 units, overlapping
spikes, shift ranges from 0 to W-1, the overlap recheck on and off, work-group
sizes of 256 and 128 (the order in which the reference's groups resolve
races), and chunk budgets that split the recording into several chunks.
Spike indices and labels must agree exactly."""
import copy
import os

import numpy as np
import pytest

import oracle
from spikesorting_fullpursuit_b200 import synth

REF_SO = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libbp_ref.so")


def _budget_for_chunk(V, si, M, S, wg, samples):
    """A max_gpu_memory whose chunks hold about ``samples`` samples (>= 4 W)."""
    C, N = V.shape
    W = si["n_samples_per_chan"]
    b = 1 << 12
    while True:
        try:
            _, chunk = oracle.plan_chunks(N, C, M, W, si["sampling_rate"], S, 1 << 40, b, wg)
        except ValueError:   # chunk shorter than 4 W
            chunk = 0
        if chunk >= samples:
            return b
        b = int(b * 1.25) + 1


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    n_chans = int(rng.choice([1, 2, 4, 8, 16]))
    kw = dict(n_chans=n_chans, fs=int(rng.choice([30000, 40000])), duration_s=float(rng.uniform(0.1, 0.6)),
              n_units=int(rng.integers(1, 11)), overlap_frac=float(rng.choice([0.0, 0.2, 0.4])))
    if n_chans >= 8:
        kw.update(layout="linear", pitch_um=50.0, nbhd=(3, 5), sigma_um=60.0)
    V, si, sm, _ = synth.make_recording(seed, **kw)
    si["do_overlap_recheck"] = bool(rng.random() < 0.8)
    W = si["n_samples_per_chan"]
    S = [W - 1, None, int(rng.integers(0, W))][seed % 3]
    wg = 256 if seed % 4 else 128
    call = dict(n_max_shift_inds=S, global_mem_size=183 * 1024 ** 3, work_group_size=wg)
    if seed % 5 == 2:   # several chunks
        M = sm["templates"].shape[0]
        S_eff = W // 2 if S is None else S
        call["max_gpu_memory"] = _budget_for_chunk(V, si, M, S_eff, wg, max(5 * W, V.shape[1] // 3))
    return V, si, sm, call


@pytest.mark.parametrize("seed", range(32))
def test_oracle_equals_reference_kernels_on_random_recordings(seed):
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref not built")
    import ref_host

    V, si, sm, call = _case(seed)
    want_ev, want_lab = ref_host.binary_pursuit(V, si, copy.deepcopy(sm), **call)
    got = oracle.binary_pursuit(V, np.float32, si, copy.deepcopy(sm), **call)
    ev, lab = np.asarray(got[0], dtype=np.int64), np.asarray(got[1], dtype=np.int64)
    assert np.array_equal(ev, np.asarray(want_ev, dtype=np.int64)), seed
    assert np.array_equal(lab, np.asarray(want_lab, dtype=np.int64)), seed
