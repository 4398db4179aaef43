"""Launch shapes change speed only: every candidate the autotuner measures, and
the shapes it picks, give the same spikes as the library's own choice."""
import copy

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spikesorting_fullpursuit_b200 import autotune, binary_pursuit, synth  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("case", [dict(seed=71, n_chans=4, n_units=6),
                                  dict(seed=72, n_chans=16, n_units=40, layout="linear", pitch_um=50.0, nbhd=(4, 6),
                                       sigma_um=60.0, rate_model=("lognormal", 10.0, 80.0), overlap_frac=0.2)])
def test_every_tuning_candidate_gives_the_same_spikes(case, tmp_path, monkeypatch):
    monkeypatch.setenv("FBP_TUNE_CACHE", str(tmp_path / "tuning.json"))
    kw = dict(case)
    V, si, sm, _ = synth.make_recording(kw.pop("seed"), duration_s=1.0, **kw)
    W = si["n_samples_per_chan"]
    want = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1, verbose=False)
    M = sm["templates"].shape[0]
    cands = autotune.lik_candidates(M)[::3] + [{"pc_group": q} for q in (1, 2, 4, 8)]
    for cand in cands:
        got = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1, verbose=False, tuning=cand)
        for g, w in zip(got, want):
            assert np.array_equal(np.asarray(g), np.asarray(w)), cand
    got = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1, verbose=False, tuning="auto")
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g), np.asarray(w))
    assert (tmp_path / "tuning.json").exists()
