"""Test infrastructure (CPU): float64 restatement of the residual energy of a fixed
spike assignment, differentiated by torch autograd.  It is the checker of
spikesorting_fullpursuit_b200.adjoint (the reference has no such component, so
this restatement is pinned by central finite differences in the tests).

    E = sum_{c,x} (v[c, x] - sum_k a_k * T~_k[c, x - s_k])^2
    T~(c, j) = (1 - |tau|) T[c, j] + |tau| T[c, j + dir],  dir = -1 (tau >= 0) / +1 (tau < 0),
    j in [-1, W], T = 0 outside [0, W); samples outside [0, N) are not modelled.
"""
from __future__ import annotations

import torch


def shifted(T: torch.Tensor, tau: torch.Tensor) -> torch.Tensor:
    """T [C, W] -> T~ [C, W + 2] (columns j = -1 .. W)."""
    C, W = T.shape
    Tp = torch.zeros(C, W + 4, dtype=T.dtype)
    Tp[:, 2:W + 2] = T                    # Tp[:, j + 2] = T[:, j]
    j = torch.arange(-1, W + 1)
    u = tau.abs()
    dir_ = -1 if float(tau.detach()) >= 0.0 else 1
    return (1 - u) * Tp[:, j + 2] + u * Tp[:, j + dir_ + 2]


def residual_energy(voltage, templates, spike_idx, spike_lab, amplitude, shift):
    """float64 autograd reference; templates [M, C, W]."""
    C, N = voltage.shape
    M, _, W = templates.shape
    model = torch.zeros(C, N + W + 4, dtype=torch.float64)
    for k in range(len(spike_idx)):
        s, l = int(spike_idx[k]), int(spike_lab[k])
        if l >= M:
            continue
        ts = shifted(templates[l], shift[k])          # columns x = s-1 .. s+W
        model = model.index_add(1, torch.arange(s - 1, s + W + 1) + 1, amplitude[k] * ts)
    r = voltage - model[:, 1:N + 1]
    return (r * r).sum()
