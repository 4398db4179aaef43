"""The screened overlap recheck's rigorous bound, checked on the CPU.

For items (a, t, b) of flagged-style windows, the reference's own float32 pair value
(oracle bpo_pair_value: the order of binary_pursuit.cl:578-632) must lie inside the
interval the screen computes from its estimate:
    LB = (Al[a] + Bl[t][b]) - X,   UB = (Au[a] + Bu[t][b]) - X
    Au/Al = G_f(a) +- alpha(a),  Bu/Bl = G_t(b) +- beta_t(b),
    alpha + beta = K (sqrt E_f |v|_f + sqrt E_t |v|_t + E_f + E_t),
    |v|_x = the window's norm over template x's non-zero channels,
    K = 1.01 * 1.05 * 2 (C W + C + W + 24) 2^-24
with the partial correlations G summed in float32 in an order unlike the reference's
(numpy's pairwise reduction), the truncated energies rounded up and the cross terms X
rounded from float64 -- the arithmetic of csrc/overlap_fast.cu."""
import numpy as np

import oracle
from spikesorting_fullpursuit_b200 import synth

f32 = np.float32


def _trunc(T, C, W, S, t, x):
    """Template t placed at shift x (x - S samples from the window start), cut to the window."""
    Z = np.zeros((C, W), dtype=np.float32)
    sh = x - S
    lo, hi = max(0, sh), min(W, W + sh)
    if hi > lo:
        Z[:, lo:hi] = T[t][:, lo - sh:hi - sh]
    return Z


def _up(x):
    """float64 -> float32 rounded up (like __double2float_ru)."""
    y = f32(x)
    return y if float(y) >= x else np.nextafter(y, f32(np.inf))


def test_reference_pair_values_lie_inside_the_screen_interval():
    V, si, sm, truth = synth.make_recording(31, n_chans=16, duration_s=0.4, n_units=12, layout="linear",
                                            pitch_um=50.0, nbhd=(4, 6), sigma_um=60.0,
                                            rate_model=("lognormal", 20.0, 80.0), overlap_frac=0.3)
    C, N = V.shape
    W = si["n_samples_per_chan"]
    S = W - 1
    S2 = 2 * S + 1
    M = sm["templates"].shape[0]
    T = np.ascontiguousarray(sm["templates"], dtype=np.float32).reshape(M, C, W)
    K = f32(1.01 * 1.05 * 2.0 * (C * W + C + W + 24) / 2.0 ** 24)
    rng = np.random.default_rng(4)
    onsets = truth["times"] - 40
    keep = (onsets >= S) & (onsets + S + W < N)
    onsets, labels = onsets[keep], truth["labels"][keep]
    checked = 0
    chans = [np.flatnonzero(np.any(T[t] != 0, axis=1)) for t in range(M)]
    tighter = []
    for p, f in zip(onsets[:4], labels[:4]):
        v = V[:, p:p + W]
        vc2 = (v.astype(np.float64) ** 2).sum(axis=1)
        nv_all = f32(np.sqrt(vc2.sum()) * 1.001)
        nv = [f32(np.sqrt(vc2[chans[t]].sum()) * 1.001) for t in range(M)]
        tighter += [float(nv[t] / nv_all) for t in range(M)]
        shifts = np.unique(np.concatenate([np.arange(S - 3, S + 4), rng.integers(0, S2, 20)]))
        G, Es = {}, {}
        for t in range(M):
            for x in shifts:
                Z = _trunc(T, C, W, S, t, int(x))
                e64 = float((Z.astype(np.float64) ** 2).sum())
                E, sE = _up(e64 * (1 + 1e-12)), _up(np.sqrt(e64) * (1 + 1e-12))
                G[(t, x)] = f32(np.add.reduce((Z * v).ravel(), dtype=np.float32) - f32(0.5) * E)
                Es[(t, x)] = (E, sE)
        for _ in range(400):
            t = int(rng.integers(0, M))
            a, b = (int(s) for s in rng.choice(shifts, 2))
            if abs(a - b) > W:
                continue
            Fa, Tb = _trunc(T, C, W, S, int(f), a), _trunc(T, C, W, S, t, b)
            X = f32((Fa.astype(np.float64) * Tb.astype(np.float64)).sum())
            (Ef, sEf), (Et, sEt) = Es[(int(f), a)], Es[(t, b)]
            al, be = K * (nv[int(f)] * sEf + Ef), K * (nv[t] * sEt + Et)
            Au, Al = G[(int(f), a)] + al, G[(int(f), a)] - al
            Bu, Bl = G[(t, b)] + be, G[(t, b)] - be
            ub, lb = f32(f32(Au + Bu) - X), f32(f32(Al + Bl) - X)
            ref = oracle.pair_value(V, sm["templates"], W, S, int(f), t, int(p), a, b)
            assert lb <= ref <= ub, (int(p), int(f), t, a, b, float(lb), ref, float(ub))
            checked += 1
    assert checked > 1000
    # templates on 4-6 of 16 channels: the per-template norms are well below the window's
    assert np.mean(tighter) < 0.8
