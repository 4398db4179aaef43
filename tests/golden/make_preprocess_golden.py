"""Golden vectors for the pursuit's pre-processing, from the reference.

For seeded recordings (spikesorting_fullpursuit_b200.synth) and each unit's
true spike onsets, runs the reference's own get_clips and
calculate_robust_template (spikesorting_fullpursuit/processing/clip_utils.py)
and get_channel_covariance_matrix (overlap/full_binary_pursuit.py, imported
with the stand-in modules of make_golden.py) as full_binary_pursuit.py:325-349
chains them, with numpy's global generator seeded before the covariance draws.
Keeps: SHA-256 of every unit's clips and valid mask, the robust templates, the
covariances.  Inputs are rebuilt by ``case_inputs``.

Usage: FBP_REFERENCE_ROOT=<checkout> python tests/golden/make_preprocess_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

from spikesorting_fullpursuit_b200 import synth  # noqa: E402

CASES = {
    # name: (recording kwargs, n_cov_samples, generator seed of the covariance draws)
    "tetrode_2s": (dict(seed=31, n_chans=4, duration_s=2.0, n_units=6), 100000, 5),
    "linear8_1s_subsampled": (dict(seed=32, n_chans=8, duration_s=1.0, n_units=10, layout="linear", pitch_um=50.0,
                                   nbhd=(3, 5), sigma_um=60.0, rate_model=("lognormal", 20.0, 80.0)), 150, 6),
}


def case_inputs(name):
    """voltage, probe dict, neighbours, per-unit ordered onsets, clip width, W, n_cov_samples, seed."""
    rec, n_cov, seed = CASES[name]
    rec = dict(rec)
    s = rec.pop("seed")
    V, si, sm, truth = synth.make_recording(s, **rec)
    probe = {"sampling_rate": si["sampling_rate"], "n_samples": V.shape[1], "v_dtype": np.float32}
    pre = 40   # clip window [-1.0, +1.5] ms at 40 kHz: the trough 40 samples in
    units = [np.sort(truth["times"][truth["labels"] == u]).astype(np.int64) for u in range(sm["templates"].shape[0])]
    # onsets around the trough times; a spike near each edge exercises the valid mask
    units[0] = np.concatenate([[3], units[0], [V.shape[1] - 5]])
    return V, probe, np.arange(V.shape[0]), units, si["clip_width"], si["n_samples_per_chan"], n_cov, seed


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    import make_golden
    make_golden._import_reference()
    from spikesorting_fullpursuit.overlap import full_binary_pursuit as fbp_ref
    from spikesorting_fullpursuit.processing import clip_utils as cu
    for name in CASES:
        V, probe, nbrs, units, cw, W, n_cov, seed = case_inputs(name)
        shas, templates, residuals = [], [], []
        for idx in units:
            clips, valid = cu.get_clips(probe, V, nbrs, idx, clip_width_s=cw)
            shas.append([sha(clips), sha(valid)])
            t = cu.calculate_robust_template(clips)
            templates.append(t)
            residuals.append(clips - t)
        np.random.seed(seed)
        covs = fbp_ref.get_channel_covariance_matrix(residuals, V.shape[0], W, n_cov, False)
        np.savez_compressed(os.path.join(HERE, "preprocess_%s.npz" % name), templates=np.vstack(templates),
                            covariances=np.stack(covs), clip_sha=np.array(shas))
        print(name, np.vstack(templates).shape, np.stack(covs).shape)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main()
