"""The pursuit's noise model (compute_separability_metrics + set_bp_threshold,
neuron_separability.py:113-195, 319-331) against the reference's own outputs.
Template energies, peak channels and per-channel noise fractions are
bit-exact; variances and what derives from them agree to FP64 rounding
(rtol 1e-12; tail probabilities 1e-9), since the reference's matrix products
run in BLAS order."""
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


# ---- pairwise_separability (neuron_separability.py:348-444) ----
#
# Shifts are exact.  Probabilities are compared relative to their value (most are
# far tails, down to 1e-310), with an absolute floor of 1e-300 for tails that
# underflow.  For float32 templates the reference forms the templates' dot
# product at shift 0 in float32 with BLAS in an unspecified order, and the
# device rounds its FP64 sum once: E_diff then differs by float32 ulps, and a
# tail probability by about z times that relative to its scale (measured up to
# 5.7e-5 relative on these cases, test_device_arithmetic_matches_reference),
# hence 5e-4.  Everything else differs by FP64 rounding (measured 2e-13).
PAIR_CASES = sorted(msg.PAIR_UNITS)
PAIR_FLOOR = 1e-300


def _pair_rtol(key, f32):
    return 5e-4 if (key == "pair" and f32) else 1e-10


def _pair_inputs(name):
    T, covs, si = msg.pair_case_inputs(name)
    sm = separability_ref.separability(T, covs, si)
    sm.update({"templates": np.vstack(T), "channel_covariance_mats": covs,
               "bp_n_samples_per_chan": si["n_samples_per_chan"]})
    return sm, si


def _check_pairs(got, want, f32):
    pair, contamination, misses, shifts = got
    assert np.array_equal(shifts, want["shifts"])
    for g, k in ((pair, "pair"), (contamination, "noise_contamination"), (misses, "noise_misses")):
        w = want[k]
        assert g.shape == w.shape, k
        same_nan = np.isnan(g) & np.isnan(w)
        with np.errstate(invalid="ignore"):
            ok = same_nan | (np.abs(g - w) <= PAIR_FLOOR + _pair_rtol(k, f32) * np.abs(w))
        assert np.all(ok), (k, g[~ok][:5], w[~ok][:5])


def _device_arithmetic(sm, si):
    """The pair kernel's arithmetic restated in numpy (csrc/separability.cu): FP64
    correlation sums, the first arg-max, FP64 quadratic forms, and the float32
    roundings the reference makes when the shift is 0."""
    from scipy.special import erfc
    T = sm["templates"]
    F = T.dtype.type
    C, W = si["n_channels"], sm["bp_n_samples_per_chan"]
    ms = (W // 4) - 1
    M, L = T.shape
    ss, covs = sm["template_SS"], sm["channel_covariance_mats"]
    pair = np.zeros((M, M))
    shifts = np.zeros((M, M), dtype=np.int32)
    for n1 in range(M):
        a = T[n1].astype(np.float64)
        for n2 in range(M):
            b = T[n2].astype(np.float64)
            cc = [abs(np.dot(a[max(0, k):L + min(0, k)], b[max(0, -k):L - max(0, k)])) for k in range(-ms, ms + 1)]
            sh = int(np.argmax(cc)) - ms
            lo, hi = max(sh, 0), W + min(sh, 0)
            var = 0.0
            ss12 = 0.0
            for c in range(C):
                t1 = T[n1, c * W + lo:c * W + hi]
                t2 = T[n2, c * W + lo - sh:c * W + hi - sh]
                d = np.zeros(W)
                d[lo:hi] = (t1 - t2).astype(np.float64) if sh == 0 else t1.astype(np.float64) - t2.astype(np.float64)
                var += d @ covs[c] @ d
                ss12 += np.dot(t1.astype(np.float64), t2.astype(np.float64))
            e1 = F(0.5) * ss[n1]
            if sh == 0:
                e_diff = float(F(e1 - (F(ss12) - F(0.5) * ss[n2])))
            else:
                e_diff = float(e1) - (ss12 - float(F(0.5) * ss[n2]))
            pair[n1, n2] = 0.5 * erfc(e_diff / np.sqrt(var) / np.sqrt(2.0)) if var > 0 else 0.0
            shifts[n1, n2] = sh
    sd = np.sqrt(sm["neuron_variances"])
    e = (F(0.5) * ss).astype(np.float64)
    thr = sm["neuron_lower_thresholds"]
    with np.errstate(divide="ignore", invalid="ignore"):
        misses = np.where(sd > 0, 0.5 * erfc((e - thr) / sd / np.sqrt(2.0)), np.nan)
        contamination = np.where(sd > 0, 0.5 * erfc((thr + e) / sd / np.sqrt(2.0)), np.nan)
    return pair, contamination, misses, shifts


@pytest.mark.parametrize("name", PAIR_CASES)
def test_pair_oracle_matches_reference(name):
    sm, si = _pair_inputs(name)
    want = np.load(os.path.join(GOLDEN, "separability_pairs_%s.npz" % name))
    pair, contamination, misses, shifts = separability_ref.pairwise(sm, si)
    assert np.array_equal(shifts, want["shifts"])
    for g, k in ((pair, "pair"), (contamination, "noise_contamination"), (misses, "noise_misses")):
        assert np.allclose(g, want[k], rtol=1e-12, atol=1e-300, equal_nan=True), k


@pytest.mark.parametrize("name", PAIR_CASES)
def test_device_arithmetic_matches_reference(name):
    sm, si = _pair_inputs(name)
    want = np.load(os.path.join(GOLDEN, "separability_pairs_%s.npz" % name))
    _check_pairs(_device_arithmetic(sm, si), want, sm["templates"].dtype == np.float32)


def test_pair_oracle_detects_a_wrong_shift():
    sm, si = _pair_inputs("tetrode_f32")
    want = np.load(os.path.join(GOLDEN, "separability_pairs_tetrode_f32.npz"))
    got = list(separability_ref.pairwise(sm, si))
    got[3] = got[3].copy()
    got[3][0, 1] += 1
    with pytest.raises(AssertionError):
        _check_pairs(got, want, True)
    got = list(separability_ref.pairwise(sm, si))
    got[0] = got[0] * (1 + 1e-3)   # a probability off by more than float32 rounding explains
    with pytest.raises(AssertionError):
        _check_pairs(got, want, True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", PAIR_CASES)
def test_gpu_pairs_match_reference(name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spikesorting_fullpursuit_b200.overlap import neuron_separability as ns
    T, covs, si = msg.pair_case_inputs(name)
    want = np.load(os.path.join(GOLDEN, "separability_pairs_%s.npz" % name))
    sm = ns.set_bp_threshold(ns.compute_separability_metrics(T, covs, si))
    got = ns._pair_metrics(sm, si)
    _check_pairs(got, want, sm["templates"].dtype == np.float32)
    pair, contamination, misses = ns.pairwise_separability(sm, si)
    assert np.array_equal(pair, got[0]) and np.array_equal(misses, got[2])
