"""Host-side checks that need no GPU: the C ABI loads and exports what
include/fbp.h declares, argument validation, and the host logic shared with
the oracle (chunk planner, clip window)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from spikesorting_fullpursuit_b200 import _native, build
from spikesorting_fullpursuit_b200.overlap import binary_pursuit_parallel as bpp
from spikesorting_fullpursuit_b200.processing.conversions import time_window_to_samples

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()   # no-op unless a source is newer than the library
    return _native.lib()


def declared_functions():
    src = open(os.path.join(REPO, "include", "fbp.h")).read()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(fbp_\w+)\s*\(", src, re.M)))


def test_header_declares_exports():
    assert declared_functions() == sorted(_native.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.fbp_abi_version() == _native.ABI_VERSION == 4


def test_workspace_bytes(lib):
    d = _native.dims(16, 400000, 40, 101, 100)
    b = _native.workspace_bytes(d, _native.FBP_PLAIN_FP32)
    assert b >= 40 * 400000 * 4
    assert _native.workspace_bytes(d, 0) > b  # tensor-core buffers on top
    bad = [_native.dims(0, 1000, 4, 101, 100), _native.dims(4, 100, 4, 101, 100),
           _native.dims(4, 100000, 4, 101, 100, 100), _native.dims(4, 100000, 0, 101, 100),
           _native.dims(4, 100000, 4, 2000, 100)]
    for d in bad:
        assert _native.workspace_bytes(d, 0) == 0


def test_invalid_arguments_fail_before_any_device_call(lib):
    d = _native.dims(4, 50, 4, 101, 100)
    n = ctypes.c_uint32(0)
    rc = lib.fbp_pursue_chunk(ctypes.byref(d), 0, None, None, None, None, None, 0, None, None, 0,
                              ctypes.byref(n), None, 0, None)
    assert rc == _native.FBP_E_ARG
    assert b"invalid" in lib.fbp_last_error()
    d = _native.dims(4, 5000, 4, 101, 100)
    rc = lib.fbp_pursue_chunk(ctypes.byref(d), 0, None, None, None, None, None, 0, None, None, 0,
                              ctypes.byref(n), None, 0, None)
    assert rc == _native.FBP_E_ARG
    buf = ctypes.c_void_p(1 << 40)
    rc = lib.fbp_pursue_chunk(ctypes.byref(d), 0, buf, buf, buf, buf, buf, 16, buf, buf, 10,
                              ctypes.byref(n), None, 0, None)
    assert rc == _native.FBP_E_WORKSPACE


def test_staged_pursuit_validates_ready_ranges_before_any_device_call(lib):
    d = _native.dims(4, 5000, 4, 101, 100)
    n = ctypes.c_uint32(0)
    buf = ctypes.c_void_p(1 << 40)

    def call(events, upto, k):
        ev = (ctypes.c_void_p * max(1, len(events)))(*events)
        up = np.array(upto or [0], dtype=np.uint32)
        fl = np.ones(max(1, len(upto)), dtype=np.uint32)
        return lib.fbp_pursue_chunk_staged(ctypes.byref(d), 0, buf, buf, buf, buf, buf, 1 << 40, buf, buf, 10,
                                           ctypes.byref(n), None, 0, ev, up.ctypes.data_as(ctypes.c_void_p),
                                           fl.ctypes.data_as(ctypes.c_void_p), k, None)

    assert call([], [], 0) == _native.FBP_E_ARG                       # no ranges
    assert call([None], [5000], 1) == _native.FBP_E_ARG               # null event
    assert call([1, 1], [3000, 2000], 2) == _native.FBP_E_ARG         # not increasing
    assert call([1, 1], [2000, 4000], 2) == _native.FBP_E_ARG         # does not reach n_samples
    assert b"n_samples" in lib.fbp_last_error()

@pytest.mark.parametrize("seed", range(40))
def test_chunk_planner_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    C = int(rng.integers(1, 70))
    M = int(rng.integers(1, 250))
    fs = int(rng.choice([20000, 30000, 40000]))
    W = int(rng.integers(20, 130))
    S = int(rng.integers(0, W + 5))
    n = int(rng.integers(W + 1, 10 ** 8))
    mem = int(rng.choice([8 * 1024 ** 3, 183 * 1024 ** 3, 48 * 1024 ** 3]))
    mgm = None if rng.random() < 0.5 else int(rng.integers(10 ** 6, 10 ** 10))
    try:
        want = oracle.plan_chunks(n, C, M, W, fs, S, mem, mgm, 256)
    except ValueError:
        with pytest.raises(ValueError):
            bpp.plan_chunks(n, C, M, W, fs, S, mem, mgm, 256)
        return
    assert bpp.plan_chunks(n, C, M, W, fs, S, mem, mgm, 256) == want


@pytest.mark.parametrize("win", [[-1.0e-3, 1.5e-3], [1.0e-3, 1.5e-3], (-2.0e-4, 3.3e-4), [0.0, 0.0]])
@pytest.mark.parametrize("fs", [30000, 40000, 24414.0625])
def test_clip_window(win, fs):
    assert time_window_to_samples(win, fs)[0] == oracle.time_window_to_samples(win, fs)[0]


def test_product_does_not_import_oracle():
    pkg = os.path.join(REPO, "spikesorting_fullpursuit_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                src = open(os.path.join(root, f)).read()
                assert "oracle" not in re.findall(r"^\s*(?:import|from)\s+(\w+)", src, re.M), f


def test_adjoint_arguments_fail_before_any_device_call(lib):
    P = ctypes.c_void_p
    fake = P(16)   # never dereferenced: validation rejects the call first
    d = _native.dims(4, 1000, 3, 21, 0)
    loss = ctypes.c_void_p(32)
    # null dims, zero sizes, null inputs, null spike arrays with spikes, null outputs
    assert lib.fbp_adjoint_loss(None, fake, fake, fake, fake, fake, fake, 1, loss, None) == _native.FBP_E_ARG
    for bad in (_native.dims(0, 1000, 3, 21, 0), _native.dims(4, 0, 3, 21, 0), _native.dims(4, 1000, 0, 21, 0),
                _native.dims(4, 1000, 3, 0, 0)):
        assert lib.fbp_adjoint_loss(ctypes.byref(bad), fake, fake, fake, fake, fake, fake, 1, loss,
                                    None) == _native.FBP_E_ARG
    assert lib.fbp_adjoint_loss(ctypes.byref(d), None, fake, fake, fake, fake, fake, 1, loss, None) == _native.FBP_E_ARG
    assert lib.fbp_adjoint_loss(ctypes.byref(d), fake, fake, None, fake, fake, fake, 1, loss, None) == _native.FBP_E_ARG
    assert lib.fbp_adjoint_loss(ctypes.byref(d), fake, fake, fake, fake, fake, fake, 1, None, None) == _native.FBP_E_ARG
    assert lib.fbp_adjoint_grad(ctypes.byref(d), fake, fake, fake, fake, fake, fake, 1, ctypes.c_double(1.0),
                                None, fake, fake, fake, None) == _native.FBP_E_ARG
    assert lib.fbp_adjoint_grad(ctypes.byref(d), fake, fake, fake, fake, fake, fake, 1, ctypes.c_double(1.0),
                                fake, fake, None, fake, None) == _native.FBP_E_ARG
    # one spike's FP64 residual tile (C x (W + 2) doubles) must fit in shared memory
    big = _native.dims(256, 100000, 3, 101, 0)
    assert lib.fbp_adjoint_loss(ctypes.byref(big), fake, fake, fake, fake, fake, fake, 1, loss,
                                None) == _native.FBP_E_ARG
    assert b"tile" in lib.fbp_last_error()


def test_tuning_validation(lib):
    t = _native.FbpTuning(5, 0, 0, 0)   # more than four tiles per CTA
    assert lib.fbp_set_tuning(ctypes.byref(t)) == _native.FBP_E_ARG
    t = _native.FbpTuning(0, 0, 9, 0)   # ring deeper than 8
    assert lib.fbp_set_tuning(ctypes.byref(t)) == _native.FBP_E_ARG
    t = _native.FbpTuning(0, 0, 0, 3)   # group size not a power of two
    assert lib.fbp_set_tuning(ctypes.byref(t)) == _native.FBP_E_ARG
    t = _native.FbpTuning(0, 0, 0, 0, 5)   # more than four epilogue warpgroups
    assert lib.fbp_set_tuning(ctypes.byref(t)) == _native.FBP_E_ARG
    t = _native.FbpTuning(1, 2, 4, 4, 3)
    assert lib.fbp_set_tuning(ctypes.byref(t)) == _native.FBP_OK
    assert lib.fbp_set_tuning(None) == _native.FBP_OK


def test_pair_separability_arguments_fail_before_any_device_call(lib):
    fake = ctypes.c_void_p(16)   # never dereferenced: validation rejects the call first

    def call(M=4, C=4, W=40, max_shift=9, ptrs=(fake,) * 9):
        t, ss, cov, var, thr, pair, cont, miss, sh = ptrs
        return lib.fbp_pair_separability(t, 0, ss, cov, var, thr, M, C, W, max_shift, pair, cont, miss, sh, None)

    # no templates: nothing to do
    assert call(M=0) == _native.FBP_OK
    for kw, msg in (({"C": 0}, b"invalid sizes"), ({"W": 0}, b"invalid sizes"),
                    ({"max_shift": -1}, b"max_shift"), ({"max_shift": 40}, b"max_shift"),
                    ({"M": 65536}, b"65535")):
        assert call(**kw) == _native.FBP_E_ARG, kw
        assert msg in lib.fbp_last_error(), kw
    # every input and the three result arrays are required; the shift matrix is optional
    for k in range(8):
        ptrs = [fake] * 9
        ptrs[k] = None
        assert call(ptrs=tuple(ptrs)) == _native.FBP_E_ARG, k
        assert b"null" in lib.fbp_last_error(), k


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the behaviour without a GPU")
def test_public_functions_fail_loudly_without_a_gpu():
    """No CPU fallback: every GPU-backed drop-in raises the reference's own error
    (binary_pursuit_parallel.py:292-293) when no CUDA device is present."""
    from spikesorting_fullpursuit_b200 import binary_pursuit, postprocessing, synth
    from spikesorting_fullpursuit_b200.overlap import full_binary_pursuit, neuron_separability
    from spikesorting_fullpursuit_b200.processing import clip_utils

    V, si, sm, _ = synth.make_recording(3, n_chans=2, duration_s=0.05, n_units=2, n_cov_clips=100)
    W = si["n_samples_per_chan"]
    covs = [np.eye(W) for _ in range(2)]
    sm_cov = dict(sm, channel_covariance_mats=covs)
    calls = [
        lambda: binary_pursuit(V, np.float32, si, sm),
        lambda: neuron_separability.compute_separability_metrics(list(sm["templates"]), covs, si),
        lambda: neuron_separability.pairwise_separability(sm_cov, si),
        lambda: clip_utils.get_clips({"sampling_rate": si["sampling_rate"]}, V, [0], np.array([100]), si["clip_width"]),
        lambda: clip_utils.calculate_robust_template(np.zeros((3, W), dtype=np.float32)),
        lambda: postprocessing.remove_binary_pursuit_duplicates(np.array([5, 7]), np.zeros((2, W), np.float32),
                                                                np.zeros(W, np.float32), np.ones(2, bool), 3),
        lambda: full_binary_pursuit.get_channel_covariance_matrix(np.zeros((4, 2 * W), np.float32), 2, W, 4, False),
    ]
    for call in calls:
        with pytest.raises(RuntimeError, match="No GPU available"):
            call()


C_CONSUMER = r"""
#include <stdio.h>
#include <string.h>
#include "fbp.h"

int main(void)
{
    fbp_dims d = {16, 400000, 40, 101, 100, 256};
    fbp_dims bad = {0, 1000, 4, 101, 100, 256};
    uint32_t n = 0;
    int rc;
    if (fbp_abi_version() != FBP_ABI_VERSION) return 1;
    if (fbp_workspace_bytes(&d, FBP_OVERLAP_RECHECK) <= fbp_workspace_bytes(&d, FBP_PLAIN_FP32)) return 2;
    if (fbp_workspace_bytes(&bad, 0) != 0) return 3;
    rc = fbp_pursue_chunk(&bad, 0, NULL, NULL, NULL, NULL, NULL, 0, NULL, NULL, 0, &n, NULL, 2048, NULL);
    if (rc != FBP_E_ARG || strlen(fbp_last_error()) == 0) return 4;
    printf("ok %d\n", fbp_abi_version());
    return 0;
}
"""


def test_header_compiles_as_c_and_links_the_library(lib, tmp_path):
    """A C99 program that includes include/fbp.h and links libfbp.so runs the host-side
    paths of the ABI (version, workspace sizes, argument rejection) without a GPU."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "consumer.c"
    src.write_text(C_CONSUMER)
    exe = tmp_path / "consumer"
    libdir = os.path.dirname(build.LIB)
    subprocess.check_call([gcc, "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(REPO, "include"),
                           str(src), "-o", str(exe), "-L", libdir, "-l:libfbp.so", "-Wl,-rpath," + libdir])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, (out.returncode, out.stderr)
    assert out.stdout.strip() == "ok %d" % _native.ABI_VERSION
