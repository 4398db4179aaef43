"""The pursuit's inputs built from sorted spikes (full_binary_pursuit.py:325-349):
clips (get_clips) and robust templates (calculate_robust_template) must equal
the reference's bit for bit; per-channel noise covariances
(get_channel_covariance_matrix) agree to FP64 rounding (rtol 1e-12 of the
largest entry: the reference multiplies with BLAS)."""
import hashlib
import importlib.util
import os

import numpy as np
import pytest

import preprocess_ref
from conftest import GOLDEN

_spec = importlib.util.spec_from_file_location("make_preprocess_golden",
                                               os.path.join(GOLDEN, "make_preprocess_golden.py"))
mpg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(mpg)
CASES = sorted(mpg.CASES)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _close(got, want):
    got, want = np.asarray(got), np.asarray(want)
    return got.shape == want.shape and np.all(np.abs(got - want) <= 1e-12 * np.abs(want).max())


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(name):
    V, probe, nbrs, units, cw, W, n_cov, seed = mpg.case_inputs(name)
    g = np.load(os.path.join(GOLDEN, "preprocess_%s.npz" % name))
    templates, residuals = [], []
    for u, idx in enumerate(units):
        clips, valid = preprocess_ref.get_clips(probe, V, nbrs, idx, cw)
        assert [_sha(clips), _sha(valid)] == list(g["clip_sha"][u])
        t = preprocess_ref.robust_template(clips)
        templates.append(t)
        residuals.append(clips - t)
    assert np.array_equal(np.vstack(templates), g["templates"])
    np.random.seed(seed)
    assert _close(np.stack(preprocess_ref.channel_covariances(residuals, V.shape[0], W, n_cov)), g["covariances"])


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference(name):
    _gpu()
    from spikesorting_fullpursuit_b200.overlap import full_binary_pursuit as fbp
    from spikesorting_fullpursuit_b200.processing import clip_utils
    V, probe, nbrs, units, cw, W, n_cov, seed = mpg.case_inputs(name)
    g = np.load(os.path.join(GOLDEN, "preprocess_%s.npz" % name))
    templates, residuals = [], []
    for u, idx in enumerate(units):
        clips, valid = clip_utils.get_clips(probe, V, nbrs, idx, cw)
        assert [_sha(clips), _sha(valid)] == list(g["clip_sha"][u])
        t = clip_utils.calculate_robust_template(clips)
        templates.append(t)
        residuals.append(clips - t)
    assert np.array_equal(np.vstack(templates), g["templates"])
    np.random.seed(seed)
    covs = fbp.get_channel_covariance_matrix(residuals, V.shape[0], W, n_cov, False)
    assert _close(np.stack(covs), g["covariances"])
    # the whole chain with the clips left on the device
    np.random.seed(seed)
    T, covs2 = fbp.templates_and_covariances(probe, V, nbrs, units, cw, V.shape[0], W, n_cov)
    assert np.array_equal(T, g["templates"])
    assert _close(np.stack(covs2), g["covariances"])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(5))
def test_gpu_robust_template_random(seed):
    _gpu()
    from spikesorting_fullpursuit_b200.processing import clip_utils
    rng = np.random.default_rng(seed)
    n = int(rng.choice([2, 3, 64, 1001, 5000]))
    L = int(rng.integers(1, 300))
    c = (rng.standard_normal((n, L)) * rng.uniform(0.1, 40)).astype(np.float32)
    c[:, 0] = c[0, 0]                         # constant column: empty 1-MAD set
    c[rng.integers(0, n, size=n // 3), -1] = 2.5   # many ties
    assert np.array_equal(clip_utils.calculate_robust_template(c), preprocess_ref.robust_template(c))
