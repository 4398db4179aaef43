"""GPU: the CUDA residual energy and its hand-written adjoint (through the C ABI,
behind torch.autograd.Function) against the float64 torch restatement
(oracle/adjoint_ref.py, itself pinned by central finite differences)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import adjoint_ref  # noqa: E402
from spikesorting_fullpursuit_b200 import _native, synth  # noqa: E402
from spikesorting_fullpursuit_b200.adjoint import residual_energy  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _native.lib()


def _check(V, T, idx, lab, amp, tau, rtol=1e-6):
    """V [C,N] f32, T [M,C,W] f32, idx/lab int, amp/tau f32 (numpy)."""
    Vd = torch.from_numpy(V).cuda()
    Td = torch.from_numpy(T).cuda().requires_grad_(True)
    ad = torch.from_numpy(amp).cuda().requires_grad_(True)
    sd = torch.from_numpy(tau).cuda().requires_grad_(True)
    e = residual_energy(Vd, Td, torch.from_numpy(idx).cuda(), torch.from_numpy(lab).cuda(), ad, sd)
    (2.5 * e).backward()
    V64 = torch.from_numpy(V.astype(np.float64))
    T64 = torch.from_numpy(T.astype(np.float64)).requires_grad_(True)
    a64 = torch.from_numpy(amp.astype(np.float64)).requires_grad_(True)
    s64 = torch.from_numpy(tau.astype(np.float64)).requires_grad_(True)
    e64 = adjoint_ref.residual_energy(V64, T64, idx, lab, a64, s64)
    (2.5 * e64).backward()
    assert abs(float(e) - float(e64)) <= 1e-10 * abs(float(e64))
    for got, want in ((Td.grad, T64.grad), (ad.grad, a64.grad), (sd.grad, s64.grad)):
        g = got.detach().cpu().double().numpy().ravel()
        w = want.numpy().ravel()
        scale = np.abs(w).max()
        np.testing.assert_allclose(g, w, rtol=rtol, atol=rtol * scale)


def test_adjoint_small_edges_and_overlaps():
    rng = np.random.default_rng(11)
    C, N, M, W = 5, 700, 4, 21
    V = rng.standard_normal((C, N)).astype(np.float32)
    T = rng.standard_normal((M, C, W)).astype(np.float32)
    idx = np.array([0, 3, 50, 50, 60, 61, 300, N - W - 1, N - W, N - 2, 400], dtype=np.int64)
    lab = np.array([0, 1, 2, 3, 0, 1, 2, 3, 0, 1, M + 2], dtype=np.int64)   # last one: invalid label
    amp = rng.normal(1.0, 0.1, size=len(idx)).astype(np.float32)
    tau = rng.uniform(-0.5, 0.5, size=len(idx)).astype(np.float32)
    tau[np.abs(tau) < 0.01] = 0.2
    perm = rng.permutation(len(idx))   # unsorted onsets: gradients must come back in input order
    _check(V, T, idx[perm], lab[perm], amp[perm], tau[perm])


def test_adjoint_recording_with_pursuit_sized_templates():
    V, si, sm, truth = synth.make_recording(21, n_chans=16, duration_s=0.5, n_units=8, layout="linear",
                                            pitch_um=50.0, nbhd=(4, 6), sigma_um=60.0,
                                            rate_model=("lognormal", 10.0, 80.0), overlap_frac=0.2)
    W = si["n_samples_per_chan"]
    M = sm["templates"].shape[0]
    T = np.ascontiguousarray(sm["templates"].reshape(M, 16, W), dtype=np.float32)
    pre = 40   # trough sample of the clip window: onsets = spike time - 40
    idx = truth["times"] - pre
    ok = (idx >= 0) & (idx < V.shape[1])
    idx, lab = idx[ok].astype(np.int64), truth["labels"][ok].astype(np.int64)
    rng = np.random.default_rng(5)
    amp = rng.normal(1.0, 0.1, size=len(idx)).astype(np.float32)
    tau = rng.uniform(-0.5, 0.5, size=len(idx)).astype(np.float32)
    tau[np.abs(tau) < 0.01] = -0.3
    _check(V, T, idx, lab, amp, tau)


def test_adjoint_no_spikes_is_voltage_energy():
    rng = np.random.default_rng(2)
    V = rng.standard_normal((3, 500)).astype(np.float32)
    T = rng.standard_normal((2, 3, 11)).astype(np.float32)
    Vd, Td = torch.from_numpy(V).cuda(), torch.from_numpy(T).cuda()
    e = residual_energy(Vd, Td, torch.zeros(0, dtype=torch.int64, device="cuda"),
                        torch.zeros(0, dtype=torch.int64, device="cuda"),
                        torch.zeros(0, device="cuda"), torch.zeros(0, device="cuda"))
    assert abs(float(e) - float((V.astype(np.float64) ** 2).sum())) <= 1e-10 * float(e)
