"""Seeded synthetic recordings for the binary-pursuit workloads.

No public dataset is involved: these recordings stand in for real ones, with
the shapes and value distributions of the benchmark configurations.

* Noise: white N(0, 1), 4th-order Butterworth band-pass 300-8000 Hz applied
  forward and backward (``sosfiltfilt``) in float64, rescaled to unit standard
  deviation per channel, stored as float32.
* Templates: biphasic differences of Gaussians over the clip window
  [-1.0, +1.5] ms, trough between -6 and -12 noise sigma at the alignment
  sample, scaled per channel by a Gaussian fall-off (over channel index, or
  over probe distance inside a channel neighbourhood; channels outside the
  neighbourhood are exactly zero).
* Spike trains: Poisson per unit with a 1.5 ms refractory period; rates uniform
  or lognormal (median, cap); a fraction of spikes can be moved to within
  +-1 ms of another unit's spike; each spike's amplitude is scaled by N(1, 0.1).
* Bias and thresholds follow the noise model of the reference's
  neuron_separability.compute_separability_metrics + set_bp_threshold
  (spikesorting_fullpursuit/overlap/neuron_separability.py:113-195, 319-331):
  theta_t = max(0, -0.5 |T_t|^2 + sigma_bp_noise sqrt(sum_c T_tc' Cov_c T_tc),
  lower_CI), with the per-channel noise covariance estimated from random clips
  of the noise-only trace (empirical, zero-mean).
"""
from __future__ import annotations

import numpy as np

from .processing.conversions import time_window_to_samples


def band_noise(rng, n_chans, n_samples, fs, lo=300.0, hi=8000.0):
    from scipy import signal
    hi = min(hi, 0.45 * fs)
    sos = signal.butter(4, [lo, hi], btype="band", fs=fs, output="sos")
    out = np.empty((n_chans, n_samples), dtype=np.float32)
    for c in range(n_chans):
        x = rng.standard_normal(n_samples)
        y = signal.sosfiltfilt(sos, x)
        y /= np.std(y)
        out[c] = y.astype(np.float32)
    return out


def channel_positions(layout, n_chans, pitch_um):
    if layout == "linear":
        return np.stack([np.zeros(n_chans), np.arange(n_chans) * pitch_um], axis=1)
    if layout == "two_column":
        rows = (n_chans + 1) // 2
        pos = [(col * pitch_um, row * pitch_um) for row in range(rows) for col in range(2)]
        return np.asarray(pos[:n_chans], dtype=np.float64)
    return np.stack([np.zeros(n_chans), np.arange(n_chans, dtype=np.float64)], axis=1)


def make_templates(rng, n_units, n_chans, fs, clip_width, layout="index", pitch_um=50.0,
                   nbhd=None, sigma_um=60.0, amp=(6.0, 12.0)):
    """Templates as an (M, C*W) float32 array, channel-major per template."""
    win, _ = time_window_to_samples(clip_width, fs)
    W = win[1] - win[0]
    t = (np.arange(W) + win[0]) / fs * 1e3  # ms, trough at t = 0
    pos = channel_positions(layout, n_chans, pitch_um)
    out = np.zeros((n_units, n_chans, W), dtype=np.float64)
    for m in range(n_units):
        s1 = rng.uniform(0.08, 0.16)
        d = rng.uniform(0.3, 0.5)
        s2 = rng.uniform(0.2, 0.4)
        r = rng.uniform(0.2, 0.45)
        w = -np.exp(-t ** 2 / (2 * s1 ** 2)) + r * np.exp(-(t - d) ** 2 / (2 * s2 ** 2))
        w = w / -w.min()
        A = rng.uniform(*amp)
        if layout == "index":
            peak = rng.integers(0, n_chans)
            sig = rng.uniform(0.7, 1.5)
            g = np.exp(-(np.arange(n_chans) - peak) ** 2 / (2 * sig ** 2))
        else:
            lo, hi = pos.min(axis=0), pos.max(axis=0)
            centre = rng.uniform(lo, hi)
            dist = np.linalg.norm(pos - centre, axis=1)
            k = nbhd if np.isscalar(nbhd) else int(rng.integers(nbhd[0], nbhd[1] + 1))
            keep = np.argsort(dist, kind="stable")[:k]
            g = np.zeros(n_chans)
            g[keep] = np.exp(-dist[keep] ** 2 / (2 * sigma_um ** 2))
            g[keep] /= g[keep].max()
        out[m] = A * g[:, None] * w[None, :]
    return out.reshape(n_units, n_chans * W).astype(np.float32), W, -win[0]


def spike_trains(rng, n_units, duration_s, fs, rates, refractory_ms=1.5, overlap_frac=0.0,
                 overlap_ms=1.0):
    """Spike sample times and unit labels, sorted by time."""
    refr = refractory_ms * 1e-3
    times, labels = [], []
    for m in range(n_units):
        rate = rates[m]
        tt = []
        cur = 0.0
        mean_isi = max(1.0 / rate - refr, 1e-4)
        while True:
            cur += refr + rng.exponential(mean_isi)
            if cur >= duration_s:
                break
            tt.append(cur)
        times.append(np.asarray(tt))
        labels.append(np.full(len(tt), m))
    t_all = np.concatenate(times) if times else np.zeros(0)
    l_all = np.concatenate(labels) if labels else np.zeros(0, dtype=int)
    if overlap_frac > 0 and t_all.size > 1 and n_units > 1:
        n_move = int(round(overlap_frac * t_all.size))
        movers = rng.choice(t_all.size, size=n_move, replace=False)
        # each unit's spikes are one contiguous block [lo, hi) of the concatenation, so
        # the r-th spike of another unit is r below the block and r + (hi - lo) above it
        counts = np.array([t.size for t in times], dtype=np.int64)
        ends = np.cumsum(counts)
        starts = ends - counts
        n_all = t_all.size
        for i in movers:
            m = l_all[i]
            lo, hi = int(starts[m]), int(ends[m])
            n_other = n_all - (hi - lo)
            if n_other == 0:
                continue
            r = int(rng.integers(0, n_other))
            j = r if r < lo else r + (hi - lo)
            t_all[i] = t_all[j] + rng.uniform(-overlap_ms, overlap_ms) * 1e-3
        # restore each unit's refractory period after the moves
        keep = np.ones(t_all.size, dtype=bool)
        for m in range(n_units):
            idx = np.flatnonzero(l_all == m)
            order = idx[np.argsort(t_all[idx], kind="stable")]
            last = -np.inf
            for k in order:
                if t_all[k] - last < refr:
                    keep[k] = False
                else:
                    last = t_all[k]
        t_all, l_all = t_all[keep], l_all[keep]
    samples = np.round(t_all * fs).astype(np.int64)
    order = np.argsort(samples, kind="stable")
    return samples[order], l_all[order].astype(np.int64)


def noise_covariance(rng, noise, W, n_clips=10000):
    C, N = noise.shape
    if N <= W + 1:  # too short to sample a clip: unit-variance white noise
        return [np.eye(W) for _ in range(C)]
    n_clips = int(min(n_clips, max(1, N - W - 1)))
    starts = rng.integers(0, N - W, size=n_clips)
    idx = starts[:, None] + np.arange(W)[None, :]
    covs = []
    for c in range(C):
        X = noise[c][idx].astype(np.float64)
        covs.append(X.T @ X / n_clips)
    return covs


def separability_metrics(templates, covs, n_chans, W, sigma_bp_noise=3.719, sigma_bp_CI=None):
    """Bias/threshold inputs of binary_pursuit (neuron_separability.py:113-195, 319-331)."""
    T = np.asarray(templates)
    M = T.shape[0]
    ci = np.inf if sigma_bp_CI is None else sigma_bp_CI
    # summed in the templates' own dtype, as neuron_separability.py:132-134 does
    ss = np.sum(T ** 2, axis=1).astype(np.float64)
    var = np.zeros(M)
    for n in range(M):
        for c in range(n_chans):
            tc = T[n, c * W:(c + 1) * W]
            var[n] += tc @ covs[c] @ tc
    lower_ci = 0.5 * ss - ci * np.sqrt(var)
    thr = -0.5 * ss + sigma_bp_noise * np.sqrt(var)
    thr = np.maximum(np.maximum(thr, 0.0), lower_ci)
    return {
        "bp_n_samples_per_chan": W,
        "templates": np.asarray(templates),
        "template_SS": ss,
        "template_SS_by_chan": np.zeros((M, n_chans)),
        "neuron_variances": var,
        "neuron_lower_thresholds": thr,
        "neuron_lower_CI": lower_ci,
    }


def make_recording(seed, n_chans=4, fs=40000, duration_s=1.0, n_units=6, layout="index",
                   pitch_um=50.0, nbhd=None, sigma_um=60.0, rate_model=("uniform", 5.0, 30.0),
                   overlap_frac=0.0, clip_width=(-1.0e-3, 1.5e-3), amp=(6.0, 12.0),
                   add_spikes=True, n_cov_clips=10000):
    """A full binary_pursuit input set: voltage, sort_info, separability_metrics."""
    rng = np.random.default_rng(seed)
    n_samples = int(round(duration_s * fs))
    clip_width = list(clip_width)
    templates, W, pre = make_templates(rng, n_units, n_chans, fs, clip_width, layout, pitch_um,
                                       nbhd, sigma_um, amp)
    if rate_model[0] == "uniform":
        rates = rng.uniform(rate_model[1], rate_model[2], size=n_units)
    else:
        rates = np.minimum(np.exp(rng.normal(np.log(rate_model[1]), 0.6, size=n_units)),
                           rate_model[2])
    noise = band_noise(rng, n_chans, n_samples, fs)
    covs = noise_covariance(rng, noise, W, n_cov_clips)
    voltage = noise.copy()
    times, labels = spike_trains(rng, n_units, duration_s, fs, rates, overlap_frac=overlap_frac)
    scales = rng.normal(1.0, 0.1, size=times.size)
    if add_spikes and times.size:
        onset = times - pre
        ok = (onset >= 0) & (onset + W <= n_samples)
        onset, lab, sc = onset[ok], labels[ok], scales[ok]
        T3 = templates.reshape(n_units, n_chans, W).astype(np.float64)
        taps = np.arange(W)
        for c in range(n_chans):
            on_chan = np.flatnonzero(np.any(T3[:, c, :] != 0, axis=1))
            sel = np.isin(lab, on_chan)
            if not np.any(sel):
                continue
            cols = (onset[sel][:, None] + taps[None, :]).ravel()
            vals = (sc[sel][:, None] * T3[lab[sel], c, :]).ravel()
            add = np.bincount(cols, weights=vals, minlength=n_samples)
            voltage[c] = (voltage[c] + add).astype(np.float32)
    sort_info = {
        "sampling_rate": fs,
        "clip_width": clip_width,
        "n_samples_per_chan": W,
        "n_channels": n_chans,
        "n_samples": n_samples,
        "do_overlap_recheck": True,
        "get_adjusted_clips": False,
        "sigma_bp_noise": 3.719,
        "sigma_bp_CI": None,
    }
    metrics = separability_metrics(templates, covs, n_chans, W)
    truth = {"times": times, "labels": labels, "scales": scales}
    return voltage, sort_info, metrics, truth


# Shapes of the benchmark configurations (durations in seconds).
CONFIGS = {
    "tetrode": dict(n_chans=4, fs=40000, duration_s=30.0, n_units=6, layout="index",
                    rate_model=("uniform", 5.0, 30.0)),
    "linear16": dict(n_chans=16, fs=40000, duration_s=600.0, n_units=40, layout="linear",
                     pitch_um=50.0, nbhd=(4, 6), sigma_um=60.0,
                     rate_model=("lognormal", 10.0, 80.0), overlap_frac=0.2),
    "dense64": dict(n_chans=64, fs=30000, duration_s=1800.0, n_units=200, layout="two_column",
                    pitch_um=25.0, nbhd=8, sigma_um=40.0,
                    rate_model=("lognormal", 8.0, 100.0), overlap_frac=0.25),
}


def make_recording_gpu(seed, device, n_chans, fs, duration_s, n_units, layout="index", pitch_um=50.0, nbhd=None,
                       sigma_um=60.0, rate_model=("uniform", 5.0, 30.0), overlap_frac=0.0,
                       clip_width=(-1.0e-3, 1.5e-3), amp=(6.0, 12.0), n_cov_clips=10000):
    """make_recording for recordings too long to filter on the host: the same
    templates, spike trains and threshold model (numpy, seeded), with the noise
    drawn and band-passed on the GPU: white N(0, 1) per channel (torch
    generator seeded from ``seed``), the zero-phase magnitude |H(f)|^2 of the
    same 4th-order Butterworth band-pass applied in the frequency domain
    (what forward-backward filtering does away from the edges), rescaled to
    unit standard deviation; spikes added with index_add on the device.
    Returns the voltage as a tensor [C, N] float32 on ``device``, sort_info,
    metrics."""
    import torch
    from scipy import signal

    rng = np.random.default_rng(seed)
    n_samples = int(round(duration_s * fs))
    clip_width = list(clip_width)
    templates, W, pre = make_templates(rng, n_units, n_chans, fs, clip_width, layout, pitch_um, nbhd, sigma_um, amp)
    if rate_model[0] == "uniform":
        rates = rng.uniform(rate_model[1], rate_model[2], size=n_units)
    else:
        rates = np.minimum(np.exp(rng.normal(np.log(rate_model[1]), 0.6, size=n_units)), rate_model[2])
    hi = min(8000.0, 0.45 * fs)
    sos = signal.butter(4, [300.0, hi], btype="band", fs=fs, output="sos")
    freqs = np.fft.rfftfreq(n_samples, d=1.0 / fs)
    _, h = signal.sosfreqz(sos, worN=freqs, fs=fs)
    gain = torch.from_numpy((np.abs(h) ** 2).astype(np.float32)).to(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    V = torch.empty((n_chans, n_samples), dtype=torch.float32, device=device)
    for c in range(n_chans):
        x = torch.randn(n_samples, generator=gen, device=device, dtype=torch.float32)
        y = torch.fft.irfft(torch.fft.rfft(x) * gain, n=n_samples)
        V[c] = y / y.std()
        del x, y
    noise_head = V[:, :min(n_samples, int(fs * 10))].cpu().numpy()
    covs = noise_covariance(rng, noise_head, W, n_cov_clips)
    times, labels = spike_trains(rng, n_units, duration_s, fs, rates, overlap_frac=overlap_frac)
    scales = rng.normal(1.0, 0.1, size=times.size)
    onset = times - pre
    ok = (onset >= 0) & (onset + W <= n_samples)
    onset, lab, sc = onset[ok], labels[ok], scales[ok]
    T3 = torch.from_numpy(templates.reshape(n_units, n_chans, W)).to(device)
    taps = torch.arange(W, device=device)
    on = torch.from_numpy(onset).to(device)
    lb = torch.from_numpy(lab).to(device)
    scd = torch.from_numpy(sc.astype(np.float32)).to(device)
    for c in range(n_chans):
        units_on = torch.nonzero(torch.any(T3[:, c, :] != 0, dim=1)).flatten()
        sel = torch.isin(lb, units_on)
        if not bool(sel.any()):
            continue
        cols = (on[sel][:, None] + taps[None, :]).reshape(-1)
        vals = (scd[sel][:, None] * T3[lb[sel], c, :]).reshape(-1)
        V[c].index_add_(0, cols, vals)
    sort_info = {
        "sampling_rate": fs, "clip_width": clip_width, "n_samples_per_chan": W, "n_channels": n_chans,
        "n_samples": n_samples, "do_overlap_recheck": True, "get_adjusted_clips": False,
        "sigma_bp_noise": 3.719, "sigma_bp_CI": None,
    }
    return V, sort_info, separability_metrics(templates, covs, n_chans, W)


def batched_segments(seed, n_segments=64, min_s=5.0, max_s=60.0, chans=(4, 12), units=(5, 30), fs=40000,
                     scale=1.0):
    """Independent segments of uneven length (uniform in [min_s, max_s] seconds,
    times ``scale``), each with its own channel count and templates, generated as
    the tetrode configuration with lognormal rates: a list of
    (voltage, sort_info, separability_metrics)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_segments):
        dur = float(rng.uniform(min_s, max_s)) * scale
        C = int(rng.integers(chans[0], chans[1] + 1))
        M = int(rng.integers(units[0], units[1] + 1))
        V, si, sm, _ = make_recording(int(rng.integers(1 << 31)), n_chans=C, fs=fs, duration_s=dur, n_units=M,
                                      layout="index", rate_model=("lognormal", 10.0, 80.0))
        out.append((V, si, sm))
    return out


def config_recording(name, seed, duration_s=None, **overrides):
    kw = dict(CONFIGS[name])
    if duration_s is not None:
        kw["duration_s"] = duration_s
    kw.update(overrides)
    return make_recording(seed, **kw)


def config_recording_gpu(name, seed, device, duration_s=None, **overrides):
    """config_recording with the noise generated on the GPU (make_recording_gpu)."""
    kw = dict(CONFIGS[name])
    if duration_s is not None:
        kw["duration_s"] = duration_s
    kw.update(overrides)
    return make_recording_gpu(seed, device, **kw)
