"""Several segments pursued at once on one GPU (worker threads, one CUDA stream
each) give the same results, in segment order, as one after another."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spikesorting_fullpursuit_b200 import _native, synth  # noqa: E402
from spikesorting_fullpursuit_b200.segments import pursue_segments  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _native.lib()


def test_concurrent_segments_match_sequential():
    # uneven lengths, channel counts and template counts, as in the batched workload
    segs = synth.batched_segments(seed=3, n_segments=5, min_s=0.5, max_s=2.0)
    args = [(V, np.float32, si, sm) for V, si, sm in segs]
    seq = pursue_segments(args, streams=1, verbose=False)
    conc = pursue_segments(args, streams=3, verbose=False)
    assert len(seq) == len(conc) == len(segs)
    n_total = 0
    for k, (a, b) in enumerate(zip(seq, conc)):
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x), np.asarray(y)), k
        n_total += len(a[0])
    assert n_total > 0
