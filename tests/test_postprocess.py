"""Post-pursuit duplicate removal (remove_binary_pursuit_duplicates,
analyze_spike_timing.py:148-193, per unit as postprocessing.py:646-675 calls it).
Keep masks must equal the reference's bit for bit: the oracle restatement on the
CPU, the CUDA kernels on the GPU."""
import importlib.util
import os

import numpy as np
import pytest

import postprocess_ref
from conftest import GOLDEN

_spec = importlib.util.spec_from_file_location("make_postprocess_golden",
                                               os.path.join(GOLDEN, "make_postprocess_golden.py"))
mpg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(mpg)

CASES = sorted(mpg.CASES)


def _want(name):
    return np.load(os.path.join(GOLDEN, "postprocess_%s.npz" % name))["keep"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_keep_masks(name):
    ev, lab, clips, bp, tol = mpg.case_inputs(name)
    got = postprocess_ref.remove_segment_duplicates(ev, lab, clips, bp, tol)
    assert np.array_equal(got, _want(name))


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_keep_masks_equal_the_reference(name):
    torch = _gpu()
    from spikesorting_fullpursuit_b200 import postprocessing
    ev, lab, clips, bp, tol = mpg.case_inputs(name)
    want = _want(name)
    assert np.array_equal(postprocessing.remove_segment_duplicates(ev, lab, clips, bp, tol), want)
    # the same with the inputs already on the device
    got = postprocessing.remove_segment_duplicates(torch.as_tensor(ev).cuda(), torch.as_tensor(lab).cuda(),
                                                   torch.as_tensor(clips).cuda(), torch.as_tensor(bp).cuda(), tol)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(6))
def test_gpu_single_unit_walk_matches_oracle(seed):
    _gpu()
    from spikesorting_fullpursuit_b200 import postprocessing
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 4000))
    L = int(rng.choice([1, 7, 8, 9, 127, 128, 129, 300, 1616, 4864]))
    # sorted or not (the walk follows the given order), runs of close spikes
    ev = np.cumsum(rng.integers(0, 30, size=n)).astype(np.int64)
    if seed % 3 == 2:
        ev = rng.permutation(ev)
    clips = (rng.standard_normal((n, L)) * rng.uniform(0.5, 20)).astype(np.float32)
    clips[rng.choice(n, size=n // 10)] = clips[0]     # exact ties
    tmpl = np.mean(clips, axis=0)
    bp = rng.random(n) < 0.7
    tol = int(rng.integers(0, 60))
    want = postprocess_ref.remove_binary_pursuit_duplicates(ev, clips, tmpl, bp, tol)
    got = postprocessing.remove_binary_pursuit_duplicates(ev, clips, tmpl, bp, tol)
    assert np.array_equal(got, want)
    assert np.array_equal(postprocessing.mean_clip(clips).cpu().numpy(), tmpl)


def test_float64_clips_are_rejected():
    from spikesorting_fullpursuit_b200 import postprocessing
    with pytest.raises(TypeError):
        postprocessing.remove_binary_pursuit_duplicates(np.arange(3), np.zeros((3, 4)), np.zeros(4, np.float32),
                                                        np.ones(3, bool), 5)
