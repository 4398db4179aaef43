"""The float64 residual-energy restatement (oracle/adjoint_ref.py) against central
finite differences (h = 1e-3) and an independent numpy evaluation of the energy.
CPU only: this pins the checker the CUDA adjoint is compared with."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import adjoint_ref  # noqa: E402


def _case(seed=0, C=3, N=300, M=3, W=11, n=9):
    rng = np.random.default_rng(seed)
    V = torch.tensor(rng.standard_normal((C, N)), dtype=torch.float64)
    T = torch.tensor(rng.standard_normal((M, C, W)), dtype=torch.float64, requires_grad=True)
    # overlapping spikes, one at each edge, one duplicate onset
    idx = np.array([0, 40, 45, 45, 120, 125, 200, N - W - 1, N - 3])[:n]
    lab = rng.integers(0, M, size=n)
    a = torch.tensor(rng.normal(1.0, 0.1, size=n), dtype=torch.float64, requires_grad=True)
    tau = rng.uniform(-0.5, 0.5, size=n)
    tau = np.where(np.abs(tau) < 0.05, 0.25 * np.sign(tau + 1e-9), tau)   # away from the kink at 0
    s = torch.tensor(tau, dtype=torch.float64, requires_grad=True)
    return V, T, idx, lab, a, s


def _energy_numpy(V, T, idx, lab, a, s):
    V, T, a, s = V.numpy(), T.detach().numpy(), a.detach().numpy(), s.detach().numpy()
    C, N = V.shape
    M, _, W = T.shape
    r = V.copy()
    for k in range(len(idx)):
        u, d = abs(s[k]), (-1 if s[k] >= 0 else 1)
        for c in range(C):
            for j in range(-1, W + 1):
                x = idx[k] + j
                if not (0 <= x < N):
                    continue
                t0 = T[lab[k], c, j] if 0 <= j < W else 0.0
                t1 = T[lab[k], c, j + d] if 0 <= j + d < W else 0.0
                r[c, x] -= a[k] * ((1 - u) * t0 + u * t1)
    return float((r * r).sum())


def test_energy_matches_numpy_loop():
    V, T, idx, lab, a, s = _case()
    e = adjoint_ref.residual_energy(V, T, idx, lab, a, s)
    ev = float(e.detach())
    assert abs(ev - _energy_numpy(V, T, idx, lab, a, s)) <= 1e-10 * abs(ev)


def test_gradients_match_central_differences():
    V, T, idx, lab, a, s = _case(seed=3)
    e = adjoint_ref.residual_energy(V, T, idx, lab, a, s)
    gT, ga, gs = torch.autograd.grad(e, (T, a, s))
    h = 1e-3

    def fd(tensor, pos):
        with torch.no_grad():
            old = tensor[pos].item()
            tensor[pos] = old + h
            ep = float(adjoint_ref.residual_energy(V, T, idx, lab, a, s))
            tensor[pos] = old - h
            em = float(adjoint_ref.residual_energy(V, T, idx, lab, a, s))
            tensor[pos] = old
        return (ep - em) / (2 * h)

    rng = np.random.default_rng(7)
    scale = max(float(gT.abs().max()), float(ga.abs().max()), float(gs.abs().max()))
    for _ in range(12):
        pos = tuple(int(rng.integers(0, n)) for n in T.shape)
        assert abs(fd(T, pos) - float(gT[pos])) <= 1e-6 * scale
    for k in range(len(idx)):
        assert abs(fd(a, k) - float(ga[k])) <= 1e-6 * scale
        assert abs(fd(s, k) - float(gs[k])) <= 1e-6 * scale
