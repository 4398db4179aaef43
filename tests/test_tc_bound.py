"""The tensor-core likelihood's rigorous bound, checked on the CPU.

The reference's float32 likelihood (oracle: compute_full_likelihood's sequential order)
must lie within the bound the lik_tc epilogue attaches to its estimate:
    est  = bias_t + sum_{c,j} tf32(T[t][c][j]) * tf32(V[c][s+j])   (float32 accumulation)
    bnd  = k_a * 1.0001 * sum_c |T_tc| |V_c strip| + k_b |bias_t|
    k_a  = 1.1 (2^-9 + (2n+8) 2^-22 + (n+2) 2^-24),  k_b = 1.1 (n+8) 2^-22,  n = C W
with tf32() dropping the 13 low mantissa bits (the tensor core reads float32 operands
that way), |V_c strip| the norm of the tile's voltage strip (128 + W - 1 samples) and
the accumulation done by BLAS (an order unlike the reference's).  Consequence checked too:
wherever est + bnd <= 0 the reference's value is <= 0 (the samples the kernel keeps).
On this recording the largest error reaches about a fifth of the bound, so a bound ten
times too small fails here."""
import numpy as np
from numpy.lib.stride_tricks import sliding_window_view

import oracle
from spikesorting_fullpursuit_b200 import synth


def _tf32(x):
    return (np.ascontiguousarray(x, dtype=np.float32).view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


def test_reference_likelihood_within_the_tensor_core_bound():
    V, si, sm, _ = synth.make_recording(41, n_chans=16, duration_s=0.2, n_units=12, layout="linear",
                                        pitch_um=50.0, nbhd=(4, 6), sigma_um=60.0,
                                        rate_model=("lognormal", 20.0, 80.0), overlap_frac=0.2)
    C, N = V.shape
    W = si["n_samples_per_chan"]
    M = sm["templates"].shape[0]
    T = np.ascontiguousarray(sm["templates"], dtype=np.float32).reshape(M, C, W)
    bias = np.float32(-0.5 * sm["template_SS"])
    L = oracle.likelihood_all(V, sm["templates"], bias, W)
    n = C * W
    u = 2.0 ** -24
    k_a = np.float32(1.1 * (1.0 / 512.0 + (2.0 * n + 8.0) * 4.0 * u + (n + 2.0) * u))
    k_b = np.float32(1.1 * (n + 8.0) * 4.0 * u)
    tnorm = (np.sqrt((T.astype(np.float64) ** 2).sum(axis=2)) * (1 + 1e-6)).astype(np.float32)   # [M][C]
    Tq = _tf32(T).reshape(M, C * W)                       # [M][(c, j)]
    Vq = _tf32(V)
    kept = positive = 0
    for s0 in range(0, N - W, 128):
        rows = min(128, N - W - s0)
        strip = V[:, s0:s0 + rows + W - 1].astype(np.float32)
        snorm = np.float32(np.sqrt(np.einsum("cr,cr->c", strip, strip, dtype=np.float32)) * 1.0001)
        bnd = k_a * np.float32(1.0001) * (tnorm @ snorm) + k_b * np.abs(bias)            # [M]
        A = np.concatenate([sliding_window_view(Vq[c, s0:s0 + rows + W - 1], W) for c in range(C)], axis=1)
        est = (A @ Tq.T).T + bias[:, None]                                               # [M][rows] float32
        ref = L[:, s0:s0 + rows]
        assert np.all(np.abs(ref.astype(np.float64) - est) <= bnd[:, None]), s0
        keep = est + bnd[:, None] <= 0
        assert np.all(ref[keep] <= 0)
        kept += int(keep.sum())
        positive += int((ref > 0).sum())
    assert kept > 0 and positive > 0
