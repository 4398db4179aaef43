"""Clip-window conversion used by binary_pursuit.

Same contract as spikesorting_fullpursuit/processing/conversions.py:4-39: the
window start is made non-positive and rounded to samples (at most 0); the end
is rounded (at least 1) and has 1 added, so the window is inclusively
sliceable.  Returns the sample window and the (sign-corrected) time window.
"""


def time_window_to_samples(time_window_s, sampling_rate):
    window = list(time_window_s)  # a copy: the caller's window is left as given
    if window[0] > 0:
        window[0] = -window[0]
    pre = min(int(round(window[0] * sampling_rate)), 0)
    post = max(int(round(window[1] * sampling_rate)), 1) + 1
    return [pre, post], window
