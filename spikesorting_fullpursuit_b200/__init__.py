"""B200-native (sm_100a) Full Binary Pursuit template matching.

``binary_pursuit`` is a drop-in for
spikesorting_fullpursuit.overlap.binary_pursuit_parallel.binary_pursuit.
"""
from .overlap.binary_pursuit_parallel import binary_pursuit, plan_chunks  # noqa: F401

__version__ = "0.1.0"
