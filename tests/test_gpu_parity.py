"""GPU parity: the CUDA path through the C ABI against the golden vectors made
by the reference and against the CPU oracle.  Integer outputs (spike indices,
labels, order) must be bit-exact; so must every float the plain path produces,
and every float the fast path produces that the pursuit can read as positive."""
import copy
import ctypes
import hashlib

import numpy as np
import pytest

import oracle
from conftest import golden_names, load_golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spikesorting_fullpursuit_b200 import _native, binary_pursuit, synth  # noqa: E402

MODES = ["plain", "fast"]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _native.lib()


def _assert_same_result(got, want, name):
    ev, lab, bl, clips = got
    if want["empty"]:
        assert isinstance(ev, list) and ev == [] and lab == [] and bl == [] and clips == []
        return
    assert np.array_equal(ev, want["event_indices"]), name
    assert np.array_equal(lab, want["neuron_labels"]), name
    assert np.array_equal(bl, want["spike_bool"]), name
    if np.asarray(want["adjusted_clips"]).size:
        assert clips.dtype == np.float32
        assert np.array_equal(clips, want["adjusted_clips"]), name


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", golden_names())
def test_golden_end_to_end(name, mode):
    V, si, sm, call, expect, meta = load_golden(name)
    sm2 = copy.deepcopy(sm)
    got = binary_pursuit(V, np.float32, si, sm2, mode=mode, verbose=False, **call)
    _assert_same_result(got, expect, name)
    assert list(sm2["n_spikes"]) == meta["n_spikes_per_unit"]


def _chunks(V, si, sm, call, meta):
    W = si["n_samples_per_chan"]
    S = call.get("n_max_shift_inds")
    S = W // 2 if S is None else S
    M = sm["templates"].shape[0]
    if V.shape[1] <= W:
        return [], W, S
    onsets, chunk = oracle.plan_chunks(V.shape[1], V.shape[0], M, W, si["sampling_rate"], S,
                                       meta["global_mem_size"], call.get("max_gpu_memory"),
                                       meta["work_group_size"])
    return [np.ascontiguousarray(np.float32(V[:, s:min(V.shape[1], s + chunk)])) for s in onsets], W, S


def _likelihood(chunk, templates, bias, W, S, mode):
    C, N = chunk.shape
    M = templates.shape[0]
    d = _native.dims(C, N, M, W, S)
    flags = _native.FBP_PLAIN_FP32 if mode == 0 else 0
    ws = torch.empty(_native.workspace_bytes(d, flags), dtype=torch.uint8, device="cuda")
    Vd = torch.from_numpy(chunk).cuda()
    Td = torch.from_numpy(np.ascontiguousarray(templates, dtype=np.float32)).cuda()
    bd = torch.from_numpy(bias).cuda()
    Ld = torch.full((M, N), float("nan"), device="cuda")
    _native.check(_native.lib().fbp_likelihood(ctypes.byref(d), mode, _ptr(Vd), _ptr(Td), _ptr(bd), None, 0,
                                               _ptr(Ld), _ptr(ws), ws.numel(), None))
    torch.cuda.synchronize()
    return Ld.cpu().numpy()


@pytest.mark.parametrize("name", [n for n in golden_names() if n != "shorter_than_window"])
def test_golden_first_pass_likelihood(name):
    V, si, sm, call, expect, meta = load_golden(name)
    chunks, W, S = _chunks(V, si, sm, call, meta)
    bias = np.float32(-0.5 * sm["template_SS"])
    for ch, info in zip(chunks, meta["chunks"]):
        L0 = _likelihood(ch, sm["templates"], bias, W, S, 0)
        assert _sha(L0) == info["lik_sha256"], name
        L1 = _likelihood(ch, sm["templates"], bias, W, S, 1)
        pos = L0 > 0
        assert np.array_equal(L1[pos], L0[pos])
        assert np.all(L1[~pos] <= 0)


def _pursue_chunk(chunk, templates, bias, theta, W, S, flags):
    C, N = chunk.shape
    M = templates.shape[0]
    d = _native.dims(C, N, M, W, S)
    ws = torch.empty(_native.workspace_bytes(d, flags), dtype=torch.uint8, device="cuda")
    Vd = torch.from_numpy(chunk.copy()).cuda()
    Td = torch.from_numpy(np.ascontiguousarray(templates, dtype=np.float32)).cuda()
    bd = torch.from_numpy(bias).cuda()
    td = torch.from_numpy(theta).cuda()
    cap = 8 * (N // W + 1) + 1024
    idx = torch.zeros(cap, dtype=torch.int32, device="cuda")
    lab = torch.zeros(cap, dtype=torch.int32, device="cuda")
    n = ctypes.c_uint32(0)
    st = _native.FbpChunkStats()
    _native.check(_native.lib().fbp_pursue_chunk(ctypes.byref(d), flags, _ptr(Vd), _ptr(Td), _ptr(bd), _ptr(td),
                                                 _ptr(ws), ws.numel(), _ptr(idx), _ptr(lab), cap, ctypes.byref(n),
                                                 ctypes.byref(st), 0, None))
    k = n.value
    return (idx[:k].cpu().numpy().view(np.uint32), lab[:k].cpu().numpy().view(np.uint32),
            Vd.cpu().numpy(), st)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", [n for n in golden_names() if n != "shorter_than_window"])
def test_golden_chunk_residual_and_passes(name, mode):
    V, si, sm, call, expect, meta = load_golden(name)
    chunks, W, S = _chunks(V, si, sm, call, meta)
    bias = np.float32(-0.5 * sm["template_SS"])
    theta = np.float32(sm["neuron_lower_thresholds"])
    flags = (_native.FBP_OVERLAP_RECHECK if si["do_overlap_recheck"] else 0)
    if mode == "plain":
        flags |= _native.FBP_PLAIN_FP32
    for ch, info in zip(chunks, meta["chunks"]):
        si_, sl_, resid, st = _pursue_chunk(ch, sm["templates"], bias, theta, W, S, flags)
        assert st.passes == len(info["passes"])
        assert si_.size == sum(info["passes"])
        if info["resid_sha256"] is not None:
            assert _sha(resid) == info["resid_sha256"]


CASES = {
    "tetrode_3s": dict(seed=101, n_chans=4, duration_s=3.0, n_units=6),
    "linear16_2s": dict(seed=102, n_chans=16, duration_s=2.0, n_units=24, layout="linear", pitch_um=50.0,
                        nbhd=(4, 6), sigma_um=60.0, rate_model=("lognormal", 10.0, 80.0), overlap_frac=0.2),
    "dense64_0p5s": dict(seed=103, n_chans=64, fs=30000, duration_s=0.5, n_units=30, layout="two_column",
                         pitch_um=25.0, nbhd=8, sigma_um=40.0, rate_model=("lognormal", 8.0, 100.0),
                         overlap_frac=0.25),
}


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", sorted(CASES))
def test_random_recordings_match_oracle(case, mode):
    kw = dict(CASES[case])
    seed = kw.pop("seed")
    V, si, sm, truth = synth.make_recording(seed, **kw)
    si["get_adjusted_clips"] = True
    W = si["n_samples_per_chan"]
    want = oracle.binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1,
                                 global_mem_size=183 * 1024 ** 3)
    got = binary_pursuit(V, np.float32, si, copy.deepcopy(sm), n_max_shift_inds=W - 1, mode=mode,
                         verbose=False)
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g), np.asarray(w)), case


@pytest.mark.parametrize("mode", MODES)
def test_capacity_retry_gives_the_same_result(mode, monkeypatch):
    """A chunk whose spikes outgrow the first attempt's output buffers is
    pursued again with a larger capacity; the result must not change."""
    from spikesorting_fullpursuit_b200.overlap import binary_pursuit_parallel as bpp

    name = "linear16_0p5s"
    V, si, sm, call, expect, meta = load_golden(name)
    monkeypatch.setattr(bpp, "CAPACITY_PER_WINDOW", 0)
    monkeypatch.setattr(bpp, "CAPACITY_EXTRA", 8)
    assert len(expect["event_indices"]) > 8
    sm2 = copy.deepcopy(sm)
    got = binary_pursuit(V, np.float32, si, sm2, mode=mode, verbose=False, **call)
    _assert_same_result(got, expect, name)
    assert list(sm2["n_spikes"]) == meta["n_spikes_per_unit"]


def test_residual_kernel_matches_oracle_order():
    rng = np.random.default_rng(5)
    C, N, M, W = 8, 20000, 5, 61
    V = rng.standard_normal((C, N)).astype(np.float32)
    T = rng.standard_normal((M, C * W)).astype(np.float32)
    # window-ordered spikes, some overlapping their predecessor, one label out of range
    idx = np.sort(rng.integers(0, N - 1, size=150)).astype(np.uint32)
    lab = rng.integers(0, M, size=150).astype(np.uint32)
    lab[7] = M + 3
    want = V.copy()
    for s, l in zip(idx, lab):
        if l >= M:
            continue
        for c in range(C):
            for j in range(W):
                if s + j >= N:
                    break
                want[c, s + j] = np.float32(want[c, s + j] - T[l, c * W + j])
    d = _native.dims(C, N, M, W, 10)
    ws = torch.empty(_native.workspace_bytes(d, _native.FBP_PLAIN_FP32), dtype=torch.uint8, device="cuda")
    Vd = torch.from_numpy(V).cuda()
    Td = torch.from_numpy(T).cuda()
    idd = torch.from_numpy(idx.view(np.int32)).cuda()
    ld = torch.from_numpy(lab.view(np.int32)).cuda()
    _native.check(_native.lib().fbp_residual(ctypes.byref(d), _ptr(Vd), _ptr(Td), _ptr(idd), _ptr(ld), 150,
                                             _ptr(ws), ws.numel(), None))
    assert np.array_equal(Vd.cpu().numpy(), want)
