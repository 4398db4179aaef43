"""Golden vectors for the pursuit's noise model, from the reference.

Runs the reference's own compute_separability_metrics and set_bp_threshold
(spikesorting_fullpursuit/overlap/neuron_separability.py:113-195, 319-331,
imported from the reference checkout with the stand-in modules of
make_golden.py) on seeded templates and noise covariances of the benchmark
shapes.  Inputs are rebuilt by ``case_inputs``; the file keeps the outputs only:
tests/golden/separability_<case>.npz.  The reference's pairwise_separability
(neuron_separability.py:348-444) is run on the same metrics (the leading units only
where all pairs would take the reference minutes), with the shift its
optimal_align_templates picks for every pair: tests/golden/separability_pairs_<case>.npz.

Usage: FBP_REFERENCE_ROOT=<checkout> python tests/golden/make_separability_golden.py
"""
from __future__ import annotations

import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

from spikesorting_fullpursuit_b200 import synth  # noqa: E402

CASES = {
    # name: (config, seed, n_units, template dtype)
    "tetrode_f32": ("tetrode", 1, 6, np.float32),
    "linear16_f32": ("linear16", 1, 40, np.float32),
    "linear16_f64": ("linear16", 2, 40, np.float64),
    "dense64_f32": ("dense64", 1, 200, np.float32),
}
# pairwise cases: leading units used (None: all)
PAIR_UNITS = {"tetrode_f32": None, "linear16_f32": None, "linear16_f64": None, "dense64_f32": 24}
KEYS = ("template_SS", "neuron_variances", "neuron_lower_CI", "neuron_lower_thresholds", "contamination",
        "peak_channel", "channel_p_noise")


def case_inputs(name):
    """(templates list, covariances, sort_info) of a case."""
    cfg, seed, n_units, dt = CASES[name]
    kw = dict(synth.CONFIGS[cfg])
    rng = np.random.default_rng(seed)
    fs = kw["fs"]
    T, W, _ = synth.make_templates(rng, n_units, kw["n_chans"], fs, [-1.0e-3, 1.5e-3], kw["layout"],
                                   kw.get("pitch_um", 50.0), kw.get("nbhd"), kw.get("sigma_um", 60.0))
    noise = synth.band_noise(rng, kw["n_chans"], int(fs * 2), fs)
    covs = synth.noise_covariance(rng, noise, W, 4000)
    n_samples = int(fs * 60)
    sort_info = {"n_channels": kw["n_chans"], "n_samples_per_chan": W, "sigma": 4.0, "n_samples": n_samples,
                 "n_threshold_crossings": rng.integers(0, 5000, size=kw["n_chans"]),
                 "sigma_bp_noise": 3.719, "sigma_bp_CI": np.inf if seed == 1 else 12.0}
    return [t.astype(dt) for t in T], covs, sort_info


def pair_case_inputs(name):
    """Inputs of a pairwise case: the case's inputs, leading units only."""
    T, covs, si = case_inputs(name)
    units = PAIR_UNITS[name]
    return (T if units is None else T[:units]), covs, si


def main():
    import make_golden
    _, _, ns = make_golden._import_reference()
    for name in CASES:
        T, covs, si = case_inputs(name)
        with contextlib.redirect_stdout(io.StringIO()):
            sm = ns.compute_separability_metrics(T, covs, si)
            sm = ns.set_bp_threshold(sm)
        np.savez_compressed(os.path.join(HERE, "separability_%s.npz" % name), **{k: np.asarray(sm[k]) for k in KEYS})
        print(name, {k: np.asarray(sm[k]).dtype.str for k in KEYS})
    for name, units in PAIR_UNITS.items():
        T, covs, si = pair_case_inputs(name)
        with contextlib.redirect_stdout(io.StringIO()):
            sm = ns.set_bp_threshold(ns.compute_separability_metrics(T, covs, si))
            pair, contamination, misses = ns.pairwise_separability(sm, si)
        W = sm["bp_n_samples_per_chan"]
        M = sm["templates"].shape[0]
        shifts = np.zeros((M, M), dtype=np.int32)
        for n1 in range(M):
            for n2 in range(M):
                shifts[n1, n2] = ns.optimal_align_templates(sm["templates"][n1, :], sm["templates"][n2, :],
                                                            si["n_channels"], max_shift=(W // 4) - 1,
                                                            align_abs=True, zero_pad=True)[2]
        np.savez_compressed(os.path.join(HERE, "separability_pairs_%s.npz" % name), pair=np.asarray(pair),
                            noise_contamination=np.asarray(contamination), noise_misses=np.asarray(misses),
                            shifts=shifts)
        print(name, "pairs", M, "nonzero shifts", int(np.count_nonzero(shifts)))


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main()
