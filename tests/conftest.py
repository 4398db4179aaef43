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
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


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
    return d["voltage"], si, sm, call, expect, meta


@pytest.fixture(params=golden_names())
def golden(request):
    return (request.param,) + load_golden(request.param)
