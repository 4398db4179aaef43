"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own, unmodified host function
``spikesorting_fullpursuit.overlap.binary_pursuit_parallel.binary_pursuit``
(imported from the read-only reference checkout) with its own OpenCL kernels
compiled for the CPU (oracle/build_ref.py) behind a stand-in pyopencl module
(oracle/fake_pyopencl.py).  Inputs are seeded synthetic recordings from
spikesorting_fullpursuit_b200.synth.  Each case is saved as one .npz with its
inputs, the call arguments, the four return values, and per chunk: the
SHA-256 of the first-pass likelihood buffer and of the final residual, and
the spike count of every pursuit pass.

Cases with ``config`` are recordings of the benchmark generator
(``synth.config_recording``): a leading slice of the recording the benchmark
pursues, or the configuration at a shorter duration.  Large voltages are not
stored: the file keeps the recipe and the SHA-256 of the voltage, and
tests/conftest.py regenerates it (seeded) and checks the hash.

Usage (needs the reference checkout; runs where the reference can be read):
    FBP_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import contextlib
import copy
import hashlib
import io
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("FBP_REFERENCE_ROOT", os.path.join(os.path.dirname(REPO), "reference"))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

from spikesorting_fullpursuit_b200 import synth  # noqa: E402

# name -> (recording kwargs, call kwargs, extra)
CASES = {
    "tetrode_1s": (dict(seed=10, n_chans=4, duration_s=1.0, n_units=6),
                   dict(n_max_shift_inds=100), dict(clips=True)),
    "linear16_0p5s": (dict(seed=11, n_chans=16, duration_s=0.5, n_units=10, layout="linear",
                           pitch_um=50.0, nbhd=(4, 6), sigma_um=60.0,
                           rate_model=("lognormal", 10.0, 80.0), overlap_frac=0.2),
                      dict(n_max_shift_inds=100), dict(clips=True)),
    "dense64_0p1s": (dict(seed=12, n_chans=64, fs=30000, duration_s=0.1, n_units=12,
                          layout="two_column", pitch_um=25.0, nbhd=8, sigma_um=40.0,
                          rate_model=("lognormal", 30.0, 100.0), overlap_frac=0.25),
                     dict(n_max_shift_inds=75), dict(clips=True)),
    "multichunk_0p6s": (dict(seed=13, n_chans=4, duration_s=0.6, n_units=4),
                        dict(n_max_shift_inds=100, max_gpu_memory=600000), dict(clips=True)),
    "shift3_m2": (dict(seed=14, n_chans=4, duration_s=0.25, n_units=2),
                  dict(n_max_shift_inds=3), dict(clips=False)),
    "no_overlap_recheck": (dict(seed=15, n_chans=4, duration_s=0.25, n_units=5),
                           dict(n_max_shift_inds=100), dict(clips=False, overlap=False)),
    "default_shift": (dict(seed=16, n_chans=4, duration_s=0.25, n_units=5),
                      dict(), dict(clips=False)),
    "noise_only": (dict(seed=17, n_chans=4, duration_s=0.25, n_units=4, add_spikes=False),
                   dict(n_max_shift_inds=100), dict(clips=True)),
    "noise_only_no_recheck": (dict(seed=17, n_chans=4, duration_s=0.25, n_units=4,
                                   add_spikes=False),
                              dict(n_max_shift_inds=100), dict(clips=True, overlap=False)),
    "shorter_than_window": (dict(seed=18, n_chans=4, duration_s=0.002, n_units=3),
                            dict(n_max_shift_inds=100), dict(clips=False)),
    "duplicate_template": (dict(seed=19, n_chans=4, duration_s=0.25, n_units=3),
                           dict(n_max_shift_inds=20), dict(clips=True, duplicate=True)),
    # the benchmark's own recording (16 ch, 40 templates, 10 min), its leading second
    "linear16_bench_1s": (dict(config="linear16", seed=1, slice_s=1.0),
                          dict(n_max_shift_inds=100), dict(clips=True, store_voltage=True)),
    # the same recording's leading 3 seconds (voltage regenerated, not stored)
    "linear16_bench_3s": (dict(config="linear16", seed=1, slice_s=3.0),
                          dict(n_max_shift_inds=100), dict(clips=False, store_voltage=False)),
    # the tetrode configuration in full: 4 ch, 30 s, 6 templates
    "tetrode_cfg0_30s": (dict(config="tetrode", seed=1),
                         dict(n_max_shift_inds=100), dict(clips=False, store_voltage=False)),
    # the dense 64-channel configuration's 200 templates (76 taps) on 0.1 s
    "dense64_m200_0p1s": (dict(config="dense64", seed=1, duration_s=0.1),
                          dict(n_max_shift_inds=75), dict(clips=True, store_voltage=True)),
}

HEAVY = ("linear16_bench_1s", "linear16_bench_3s", "tetrode_cfg0_30s", "dense64_m200_0p1s")


def make_inputs(rec_kw):
    """Voltage, sort_info, metrics of a case's recording kwargs (see CASES)."""
    rec_kw = dict(rec_kw)
    seed = rec_kw.pop("seed")
    if "config" not in rec_kw:
        voltage, sort_info, metrics, _ = synth.make_recording(seed, **rec_kw)
        return voltage, sort_info, metrics
    name = rec_kw.pop("config")
    slice_s = rec_kw.pop("slice_s", None)
    voltage, sort_info, metrics, _ = synth.config_recording(name, seed, **rec_kw)
    if slice_s is not None:
        n = int(round(slice_s * sort_info["sampling_rate"]))
        voltage = np.ascontiguousarray(voltage[:, :n])
        sort_info = dict(sort_info, n_samples=n)
    return voltage, sort_info, metrics


def _import_reference():
    import fake_pyopencl as fcl
    fcl.install()
    fcl.reference_import_stubs()
    sys.path.insert(0, REFERENCE)
    import spikesorting_fullpursuit.c_cython as cc
    cc.sort_cython = sys.modules["spikesorting_fullpursuit.c_cython.sort_cython"]
    from spikesorting_fullpursuit.overlap import binary_pursuit_parallel as bpp
    from spikesorting_fullpursuit.overlap import neuron_separability as ns
    return fcl, bpp, ns


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def build_case(name, fcl, bpp, ns):
    rec_kw, call_kw, extra = CASES[name]
    seed = rec_kw["seed"]
    voltage, sort_info, metrics = make_inputs(rec_kw)
    if extra.get("duplicate"):
        T = metrics["templates"].copy()
        T[2] = T[0]
        covs = synth.noise_covariance(np.random.default_rng(seed + 1000),
                                      voltage, sort_info["n_samples_per_chan"])
        metrics = synth.separability_metrics(T, covs, sort_info["n_channels"],
                                             sort_info["n_samples_per_chan"])
    sort_info["get_adjusted_clips"] = bool(extra.get("clips", False))
    sort_info["do_overlap_recheck"] = bool(extra.get("overlap", True))
    # Cross-check the synthetic bias/threshold model against the reference's own
    # separability code on the same covariance (neuron_separability.py:113-195, 319-331).
    covs = synth.noise_covariance(np.random.default_rng(seed + 2000), voltage,
                                  sort_info["n_samples_per_chan"], 2000)
    mine = synth.separability_metrics(metrics["templates"], covs, sort_info["n_channels"],
                                      sort_info["n_samples_per_chan"])
    si_ref = dict(sort_info, sigma=4.0, sigma_bp_CI=np.inf,
                  n_threshold_crossings=np.zeros(sort_info["n_channels"]))
    with contextlib.redirect_stdout(io.StringIO()):
        ref_m = ns.compute_separability_metrics(list(metrics["templates"]), covs, si_ref)
        ref_m = ns.set_bp_threshold(ref_m)
    np.testing.assert_allclose(ref_m["neuron_lower_thresholds"], mine["neuron_lower_thresholds"],
                               rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(ref_m["template_SS"], mine["template_SS"], rtol=1e-12)

    chunks = []
    state = {}

    def hook(kname, kernel):
        if kname == "compute_full_likelihood":
            vbuf, lbuf = kernel.args[0], kernel.args[9]
            if id(vbuf) != state.get("vbuf"):
                state["vbuf"] = id(vbuf)
                chunks.append({"lik_sha256": _sha(lbuf.view(np.float32)), "passes": [],
                               "vbuf": vbuf, "n_samples": int(kernel.args[1])})
        elif kname == "binary_pursuit":
            chunks[-1]["passes"].append(int(kernel.args[10].view(np.uint32)[0]))
        elif kname in ("get_adjusted_clips",):
            pass

    fcl.launch_hooks[:] = [hook]
    # the residual is read when the voltage buffer is released at the end of a chunk
    orig_release = fcl.Buffer.release

    def release(self):
        for ch in chunks:
            if ch.get("vbuf") is self and "resid_sha256" not in ch:
                ch["resid_sha256"] = _sha(self.view(np.float32))
        orig_release(self)

    fcl.Buffer.release = release
    sm = copy.deepcopy(metrics)
    out_log = io.StringIO()
    error = None
    try:
        with contextlib.redirect_stdout(out_log):
            res = bpp.binary_pursuit(voltage, np.float32, sort_info, sm, kernels_path=None,
                                     **call_kw)
    except Exception as exc:  # the reference's own failure is part of the record
        error = "%s: %s" % (type(exc).__name__, exc)
        res = ([], [], [], [])
        sm["n_spikes"] = np.zeros(len(metrics["templates"]))
    finally:
        fcl.Buffer.release = orig_release
        fcl.launch_hooks[:] = []
    ev, lab, bl, clips = res
    meta = {
        "case": name,
        "recording": dict(CASES[name][0]),
        "call": call_kw,
        "work_group_size": fcl.WORK_GROUP_SIZE,
        "global_mem_size": fcl.GLOBAL_MEM_SIZE,
        "sort_info": {k: (list(v) if isinstance(v, (list, tuple)) else v)
                      for k, v in sort_info.items()},
        "chunks": [{k: v for k, v in ch.items() if k != "vbuf"} for ch in chunks],
        "n_spikes": int(len(ev)),
        "reference_error": error,
        "n_spikes_per_unit": [int(x) for x in sm["n_spikes"]],
    }
    for ch in meta["chunks"]:
        ch.setdefault("resid_sha256", None)
    meta["voltage_sha256"] = _sha(np.float32(voltage))
    stored = {"voltage": voltage} if extra.get("store_voltage", True) else {}
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        **stored,
        templates=np.asarray(metrics["templates"]),
        template_SS=np.asarray(metrics["template_SS"]),
        template_SS_by_chan=np.asarray(metrics["template_SS_by_chan"]),
        neuron_lower_thresholds=np.asarray(metrics["neuron_lower_thresholds"]),
        event_indices=np.asarray(ev, dtype=np.int64),
        neuron_labels=np.asarray(lab, dtype=np.int64),
        spike_bool=np.asarray(bl, dtype=bool),
        adjusted_clips=np.asarray(clips, dtype=np.float32),
        empty_result=np.array(isinstance(ev, list)),
        meta=np.array(json.dumps(meta)),
    )
    return meta


def main(argv):
    fcl, bpp, ns = _import_reference()
    names = argv or list(CASES)
    manifest_path = os.path.join(HERE, "MANIFEST.json")
    manifest = json.load(open(manifest_path)) if os.path.exists(manifest_path) else {}
    for name in names:
        meta = build_case(name, fcl, bpp, ns)
        manifest[name] = {"n_spikes": meta["n_spikes"], "chunks": len(meta["chunks"]),
                          "passes": [len(c["passes"]) for c in meta["chunks"]]}
        print(name, manifest[name])
    with open(manifest_path, "w") as fp:
        json.dump(manifest, fp, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
