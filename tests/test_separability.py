"""The pursuit's noise model (compute_separability_metrics + set_bp_threshold,
neuron_separability.py:113-195, 319-331) against the reference's own outputs.
Template energies, peak channels and per-channel noise fractions are
bit-exact; variances and what derives from them agree to FP64 rounding
(rtol 1e-12; tail probabilities 1e-9), since the reference's matrix products
run in BLAS order."""
import copy
import importlib.util
import os

import numpy as np
import pytest

import separability_ref
from conftest import GOLDEN

_spec = importlib.util.spec_from_file_location("make_separability_golden",
                                               os.path.join(GOLDEN, "make_separability_golden.py"))
msg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(msg)

CASES = sorted(msg.CASES)
EXACT = ("template_SS", "peak_channel", "channel_p_noise")
RTOL = {"neuron_variances": 1e-12, "neuron_lower_CI": 1e-12, "neuron_lower_thresholds": 1e-12,
        "contamination": 1e-9}


def _check(got, want):
    for k in EXACT:
        assert np.asarray(got[k]).dtype == want[k].dtype, k
        assert np.array_equal(np.asarray(got[k]), want[k]), k
    for k, tol in RTOL.items():
        g, w = np.asarray(got[k], dtype=np.float64), want[k]
        finite = np.isfinite(w)
        # relative to the value, or to the largest finite threshold for values near 0
        floor = 1e-300 if k == "contamination" else np.abs(want["neuron_lower_thresholds"]).max()
        scale = np.maximum(np.abs(np.where(finite, w, 0.0)), floor)
        ok = (g == w) | (finite & (np.abs(g - np.where(finite, w, 0.0)) <= tol * scale))
        assert np.all(ok), (k, g[~ok], w[~ok])


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(name):
    T, covs, si = msg.case_inputs(name)
    want = np.load(os.path.join(GOLDEN, "separability_%s.npz" % name))
    _check(separability_ref.separability(T, covs, si), want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference(name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spikesorting_fullpursuit_b200.overlap import neuron_separability as ns
    T, covs, si = msg.case_inputs(name)
    want = np.load(os.path.join(GOLDEN, "separability_%s.npz" % name))
    sm = ns.set_bp_threshold(ns.compute_separability_metrics(T, covs, si))
    _check(sm, want)
    ss, thr = ns.bp_thresholds(T, covs, si["n_channels"], si["n_samples_per_chan"], si["sigma_bp_noise"],
                               si["sigma_bp_CI"])
    assert np.array_equal(ss, want["template_SS"])
    assert np.allclose(thr, want["neuron_lower_thresholds"], rtol=1e-12, atol=1e-12 * np.abs(thr).max())
