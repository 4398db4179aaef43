"""Golden vectors for the post-pursuit duplicate removal, from the reference.

Calls the reference's own remove_binary_pursuit_duplicates
(spikesorting_fullpursuit/analyze_spike_timing.py:148-193, a numpy-only module
imported from the reference checkout) per unit with the unit's mean clip as
template, as WorkItemSummary.remove_segment_binary_pursuit_duplicates
(postprocessing.py:646-675) does.  Inputs: the spikes and adjusted clips the
reference's binary_pursuit returned for golden cases of tests/golden, plus
seeded synthetic spike lists with planted near-duplicates.  Output:
tests/golden/postprocess_<case>.npz with the reference's keep mask only; the
inputs are rebuilt by ``case_inputs`` (from the pursuit golden, or seeded).

Usage: FBP_REFERENCE_ROOT=<checkout> python tests/golden/make_postprocess_golden.py
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("FBP_REFERENCE_ROOT", os.path.join(os.path.dirname(REPO), "reference"))


def _reference_module():
    path = os.path.join(REFERENCE, "spikesorting_fullpursuit", "analyze_spike_timing.py")
    spec = importlib.util.spec_from_file_location("ref_analyze_spike_timing", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _segment_keep(ref, ev, lab, clips, bp, tol):
    keep = np.ones(lab.size, dtype=bool)
    for u in np.unique(lab):
        sel = lab == u
        keep[sel] = ref.remove_binary_pursuit_duplicates(ev[sel], clips[sel, :], np.mean(clips[sel, :], axis=0),
                                                         bp[sel], tol)
    return keep


def _from_golden(name):
    d = np.load(os.path.join(HERE, name + ".npz"))
    ev = d["event_indices"].astype(np.int64)
    order = np.argsort(ev, kind="stable")
    return ev[order], d["neuron_labels"][order].astype(np.int64), d["adjusted_clips"][order], \
        np.ones(ev.size, dtype=bool)


def _synthetic(seed, n_units, n, clip_len):
    rng = np.random.default_rng(seed)
    base = np.sort(rng.integers(0, 200000, size=n)).astype(np.int64)
    # plant near-duplicates: copies 0-20 samples after a spike, same unit
    dup = rng.choice(n, size=n // 4, replace=False)
    ev = np.concatenate([base, base[dup] + rng.integers(0, 21, size=dup.size)])
    lab = np.concatenate([rng.integers(0, n_units, size=n), np.zeros(dup.size, dtype=np.int64)])
    lab[n:] = lab[dup]
    order = np.argsort(ev, kind="stable")
    ev, lab = ev[order], lab[order]
    tmpl = rng.standard_normal((n_units, clip_len)).astype(np.float32) * 5
    clips = (tmpl[lab] + rng.standard_normal((ev.size, clip_len)).astype(np.float32)).astype(np.float32)
    # some exact ties: identical clips
    tie = rng.choice(ev.size, size=ev.size // 20, replace=False)
    clips[tie[1:]] = clips[tie[0]]
    bp = rng.random(ev.size) < 0.8
    return ev, lab, clips, bp


CASES = {
    # the adjusted clips the reference's binary_pursuit returned; tol = 2 * half clip width at 40 kHz
    "linear16_bench_1s": dict(golden="linear16_bench_1s", tol=80),
    "linear16_0p5s": dict(golden="linear16_0p5s", tol=80),
    "synthetic_4units": dict(seed=1, n_units=4, n=3000, clip_len=404, tol=40),
    "synthetic_40units": dict(seed=2, n_units=40, n=8000, clip_len=1616, tol=80),
}


def case_inputs(name):
    """(event_indices, labels, clips, bp, tol) of a case, rebuilt from its recipe."""
    c = CASES[name]
    if "golden" in c:
        ev, lab, clips, bp = _from_golden(c["golden"])
    else:
        ev, lab, clips, bp = _synthetic(c["seed"], c["n_units"], c["n"], c["clip_len"])
    return ev, lab, clips, bp, c["tol"]


def main():
    ref = _reference_module()
    for name in CASES:
        ev, lab, clips, bp, tol = case_inputs(name)
        keep = _segment_keep(ref, ev, lab, clips, bp, tol)
        np.savez_compressed(os.path.join(HERE, "postprocess_%s.npz" % name), keep=keep,
                            n=np.int64(ev.size), tol=np.int64(tol))
        print(name, ev.size, "dropped", int((~keep).sum()))


if __name__ == "__main__":
    sys.exit(main())
