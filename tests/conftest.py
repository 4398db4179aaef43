import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libfbp.so")


def golden_names():
    """Pursuit goldens (tests/golden/*.npz other than those of the pre- and post-processing steps)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and not f.startswith(("postprocess_", "separability_", "preprocess_")))


_VOLTAGE_CACHE = {}


def _golden_voltage(d, meta):
    """The stored voltage, or (for large recordings) the seeded regeneration of
    it, checked against the SHA-256 the golden recorded."""
    if "voltage" in d.files:
        return d["voltage"]
    key = meta["case"]
    if key not in _VOLTAGE_CACHE:
        import hashlib
        import importlib.util
        spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
        mg = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mg)
        V = mg.make_inputs(meta["recording"])[0]
        got = hashlib.sha256(np.ascontiguousarray(np.float32(V)).tobytes()).hexdigest()
        assert got == meta["voltage_sha256"], "regenerated voltage of %s differs from the golden's" % key
        _VOLTAGE_CACHE[key] = V
    return _VOLTAGE_CACHE[key]


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(d["meta"]))
    si = dict(meta["sort_info"])
    sm = {
        "templates": d["templates"],
        "template_SS": d["template_SS"],
        "template_SS_by_chan": d["template_SS_by_chan"],
        "neuron_lower_thresholds": d["neuron_lower_thresholds"],
    }
    call = dict(meta["call"])
    expect = {
        "event_indices": d["event_indices"],
        "neuron_labels": d["neuron_labels"],
        "spike_bool": d["spike_bool"],
        "adjusted_clips": d["adjusted_clips"],
        "empty": bool(d["empty_result"]),
    }
    return _golden_voltage(d, meta), si, sm, call, expect, meta


# Goldens whose CPU checks take minutes: in the default CPU run the oracle is
# checked end to end on two of them only; FBP_FULL_GOLDEN=1 runs every check on
# all of them (the chunk internals, the reference kernels' restated host loop,
# the 3 s slice of the 10-minute recording, which is regenerated, and the
# 200-template case, whose brute-force oracle takes minutes).
HEAVY_GOLDENS = {"linear16_bench_1s": "end_to_end", "tetrode_cfg0_30s": "end_to_end",
                 "linear16_bench_3s": "full_only", "dense64_m200_0p1s": "full_only"}


def full_golden_run():
    return os.environ.get("FBP_FULL_GOLDEN", "") not in ("", "0")


def skip_heavy(name, check):
    """Skip a CPU check of a heavy golden unless the full run is requested."""
    mode = HEAVY_GOLDENS.get(name)
    if mode is None or full_golden_run():
        return
    if mode == "full_only" or check != "end_to_end":
        pytest.skip("heavy golden: set FBP_FULL_GOLDEN=1 for this check")


@pytest.fixture(params=golden_names())
def golden(request):
    return (request.param,) + load_golden(request.param)
