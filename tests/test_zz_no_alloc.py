"""The allocation-free residual entry point against the regular one, on the GPU.

fbp_residual_noalloc serves callers that cannot call cudaMalloc (a plug-in in a
host that owns all device memory and forbids allocation while streaming): its
scratch is a static device array instead of a caller workspace.  Its results must
equal fbp_residual's on the same inputs -- bit for bit, the tolerance every
parity test here uses -- on consecutive calls (the array keeps the previous
call's contents).  This file is collected last so that a failure here leaves
every other test already run.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spikesorting_fullpursuit_b200 import _native  # noqa: E402


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _inputs(seed, C=8, N=100000, M=6, W=61, n=300):
    rng = np.random.default_rng(seed)
    V = rng.standard_normal((C, N)).astype(np.float32)
    T = rng.standard_normal((M, C * W)).astype(np.float32)
    # onsets in window order, with some ranges overlapping their predecessor
    idx = np.sort(rng.integers(0, N - 1, size=n)).astype(np.uint32)
    lab = rng.integers(0, M, size=n).astype(np.uint32)
    return V, T, idx, lab, W


def _run_both(V, T, idx, lab, W):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _native.lib()
    C, N = V.shape
    M = T.shape[0]
    n = idx.size
    d = _native.dims(C, N, M, W, 10)
    Td = torch.from_numpy(T).cuda()
    idd = torch.from_numpy(idx.view(np.int32)).cuda()
    ld = torch.from_numpy(lab.view(np.int32)).cuda()
    ws = torch.empty(_native.workspace_bytes(d, _native.FBP_PLAIN_FP32), dtype=torch.uint8, device="cuda")
    Va = torch.from_numpy(V).cuda()
    _native.check(L.fbp_residual(ctypes.byref(d), _ptr(Va), _ptr(Td), _ptr(idd), _ptr(ld), n, _ptr(ws),
                                 ws.numel(), None))
    Vb = torch.from_numpy(V).cuda()
    _native.check(L.fbp_residual_noalloc(ctypes.byref(d), _ptr(Vb), _ptr(Td), _ptr(idd), _ptr(ld), n, None))
    torch.cuda.synchronize()
    return Va.cpu().numpy(), Vb.cpu().numpy()


def test_noalloc_residual_equals_regular_on_consecutive_calls():
    for seed in (1, 2):
        V, T, idx, lab, W = _inputs(seed, n=300 if seed == 1 else 1200)
        want, got = _run_both(V, T, idx, lab, W)
        assert not np.array_equal(want, V)
        assert np.array_equal(got, want), "call %d" % seed


def test_noalloc_rejects_more_spikes_than_its_array():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _native.lib()
    V = torch.zeros((4, 1000), device="cuda")
    T = torch.zeros((2, 4 * 21), device="cuda")
    idx = torch.zeros(8, dtype=torch.int32, device="cuda")
    d = _native.dims(4, 1000, 2, 21, 5)
    rc = L.fbp_residual_noalloc(ctypes.byref(d), _ptr(V), _ptr(T), _ptr(idx), _ptr(idx),
                                _native.NOALLOC_MAX_SPIKES + 1, None)
    assert rc == _native.FBP_E_ARG
    assert b"FBP_NOALLOC_MAX_SPIKES" in L.fbp_last_error()


def test_noalloc_clears_the_previous_error():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _native.lib()
    V, T, idx, lab, W = _inputs(3, N=20000, n=50)
    d = _native.dims(V.shape[0], V.shape[1], T.shape[0], W, 10)
    Vd, Td = torch.from_numpy(V).cuda(), torch.from_numpy(T).cuda()
    idd = torch.from_numpy(idx.view(np.int32)).cuda()
    ld = torch.from_numpy(lab.view(np.int32)).cuda()
    # more spikes than the chunk has windows: rejected like fbp_residual rejects it
    nw = (V.shape[1] + W - 1) // W
    many = torch.zeros(nw + 1, dtype=torch.int32, device="cuda")
    assert L.fbp_residual_noalloc(ctypes.byref(d), _ptr(Vd), _ptr(Td), _ptr(many), _ptr(many), nw + 1,
                                  None) == _native.FBP_E_ARG
    assert L.fbp_last_error() != b""
    _native.check(L.fbp_residual_noalloc(ctypes.byref(d), _ptr(Vd), _ptr(Td), _ptr(idd), _ptr(ld), idx.size, None))
    torch.cuda.synchronize()
    assert L.fbp_last_error() == b""
