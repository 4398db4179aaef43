"""ctypes binding of libfbp.so (the C ABI declared in include/fbp.h).

The library is built in-tree by spikesorting_fullpursuit_b200/build.py.  There
is no fallback: if it is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfbp.so")

FBP_OK = 0
FBP_E_ARG = -1
FBP_E_WORKSPACE = -2
FBP_E_CAPACITY = -3
FBP_E_PASSES = -4
FBP_E_CUDA = -5
FBP_E_DEVICE = -6

FBP_OVERLAP_RECHECK = 0x1
FBP_PLAIN_FP32 = 0x2
FBP_TIMING = 0x4

# every function include/fbp.h declares
EXPORTS = ("fbp_abi_version", "fbp_last_error", "fbp_workspace_bytes", "fbp_pursue_chunk", "fbp_pursue_chunk_staged",
           "fbp_adjusted_clips", "fbp_likelihood", "fbp_residual", "fbp_residual_noalloc",
           "fbp_adjoint_loss", "fbp_adjoint_grad", "fbp_mean_clip", "fbp_bp_duplicates_workspace",
           "fbp_bp_duplicates", "fbp_separability", "fbp_pair_separability", "fbp_gather_clips",
           "fbp_robust_template",
           "fbp_residual_covariance", "fbp_set_tuning")
NOALLOC_MAX_SPIKES = 65536
MAX_PASSES = 2048   # default pass limit of one chunk (the reference's loop has none)
PASS_RING = 64
ABI_VERSION = 4


class FbpDims(ctypes.Structure):
    _fields_ = [("n_chans", ctypes.c_uint32), ("n_samples", ctypes.c_uint32),
                ("n_templates", ctypes.c_uint32), ("template_len", ctypes.c_uint32),
                ("n_max_shift", ctypes.c_uint32), ("work_group", ctypes.c_uint32)]


class FbpChunkStats(ctypes.Structure):
    _fields_ = [("passes", ctypes.c_int32), ("n_spikes", ctypes.c_uint32),
                ("listed", ctypes.c_uint64), ("flagged", ctypes.c_uint64),
                ("fixups", ctypes.c_uint64), ("pair_exact", ctypes.c_uint64),
                ("ms_likelihood", ctypes.c_float), ("ms_argmax", ctypes.c_float),
                ("ms_overlap", ctypes.c_float), ("ms_accept", ctypes.c_float),
                ("ms_residual", ctypes.c_float), ("ms_total", ctypes.c_float),
                ("ms_lik_tc", ctypes.c_float), ("ms_fixup", ctypes.c_float),
                ("ms_lik_exact", ctypes.c_float), ("ms_partial_corr", ctypes.c_float),
                ("ms_screen", ctypes.c_float), ("ms_score", ctypes.c_float),
                ("ms_overlap_plain", ctypes.c_float), ("fixup_runs_queued", ctypes.c_uint32),
                ("launches", ctypes.c_uint64), ("pc_macs", ctypes.c_uint64),
                ("pass_spikes", ctypes.c_uint32 * PASS_RING)]

    def as_dict(self):
        out = {k: getattr(self, k) for k, _ in self._fields_}
        # spikes per pass, oldest first (the ring keeps the last PASS_RING passes)
        p = int(self.passes)
        ring = list(self.pass_spikes)
        first = max(1, p - PASS_RING + 1)
        out["pass_spikes"] = [ring[(q - 1) % PASS_RING] for q in range(first, p + 1)]
        return out


class FbpTuning(ctypes.Structure):
    _fields_ = [("lik_tiles", ctypes.c_uint32), ("lik_group", ctypes.c_uint32), ("lik_stages", ctypes.c_uint32),
                ("pc_group", ctypes.c_uint32), ("lik_epi", ctypes.c_uint32)]


class FbpError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("libfbp status %d: %s" % (status, msg))
        self.status = status


_lib = None


def lib():
    """Load libfbp.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libfbp.so is not built; run spikesorting_fullpursuit_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    L.fbp_abi_version.restype = ctypes.c_int
    if L.fbp_abi_version() != ABI_VERSION:
        raise OSError("libfbp.so has ABI %d, this binding needs %d: rebuild it" % (L.fbp_abi_version(), ABI_VERSION))
    P, vp, u32, sz = ctypes.POINTER, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_size_t
    L.fbp_abi_version.restype = ctypes.c_int
    L.fbp_last_error.restype = ctypes.c_char_p
    L.fbp_workspace_bytes.argtypes = [P(FbpDims), u32]
    L.fbp_workspace_bytes.restype = sz
    L.fbp_pursue_chunk.argtypes = [P(FbpDims), u32, vp, vp, vp, vp, vp, sz, vp, vp, u32,
                                   P(u32), P(FbpChunkStats), ctypes.c_int32, vp]
    L.fbp_pursue_chunk.restype = ctypes.c_int
    L.fbp_pursue_chunk_staged.argtypes = [P(FbpDims), u32, vp, vp, vp, vp, vp, sz, vp, vp, u32,
                                          P(u32), P(FbpChunkStats), ctypes.c_int32, vp, vp, vp, u32, vp]
    L.fbp_pursue_chunk_staged.restype = ctypes.c_int
    L.fbp_adjusted_clips.argtypes = [P(FbpDims), vp, vp, vp, vp, u32, vp, vp]
    L.fbp_adjusted_clips.restype = ctypes.c_int
    L.fbp_likelihood.argtypes = [P(FbpDims), ctypes.c_int, vp, vp, vp, vp, u32, vp, vp, sz, vp]
    L.fbp_likelihood.restype = ctypes.c_int
    L.fbp_residual.argtypes = [P(FbpDims), vp, vp, vp, vp, u32, vp, sz, vp]
    L.fbp_residual.restype = ctypes.c_int
    L.fbp_residual_noalloc.argtypes = [P(FbpDims), vp, vp, vp, vp, u32, vp]
    L.fbp_residual_noalloc.restype = ctypes.c_int
    L.fbp_adjoint_loss.argtypes = [P(FbpDims), vp, vp, vp, vp, vp, vp, u32, vp, vp]
    L.fbp_adjoint_loss.restype = ctypes.c_int
    L.fbp_adjoint_grad.argtypes = [P(FbpDims), vp, vp, vp, vp, vp, vp, u32, ctypes.c_double, vp, vp, vp, vp, vp]
    L.fbp_adjoint_grad.restype = ctypes.c_int
    L.fbp_mean_clip.argtypes = [vp, u32, u32, vp, vp]
    L.fbp_mean_clip.restype = ctypes.c_int
    L.fbp_bp_duplicates_workspace.argtypes = [u32]
    L.fbp_bp_duplicates_workspace.restype = sz
    L.fbp_bp_duplicates.argtypes = [vp, vp, vp, vp, u32, u32, ctypes.c_int64, vp, vp, sz, vp]
    L.fbp_bp_duplicates.restype = ctypes.c_int
    dbl, i32 = ctypes.c_double, ctypes.c_int
    L.fbp_separability.argtypes = [vp, i32, vp, u32, u32, u32, dbl, dbl, i32, vp, vp, vp, vp, vp, vp, vp]
    L.fbp_separability.restype = ctypes.c_int
    L.fbp_pair_separability.argtypes = [vp, i32, vp, vp, vp, vp, u32, u32, u32, ctypes.c_int32, vp, vp, vp, vp, vp]
    L.fbp_pair_separability.restype = ctypes.c_int
    L.fbp_gather_clips.argtypes = [vp, u32, ctypes.c_uint64, vp, u32, vp, u32, ctypes.c_int32, u32, vp, vp]
    L.fbp_gather_clips.restype = ctypes.c_int
    L.fbp_robust_template.argtypes = [vp, u32, u32, vp, vp]
    L.fbp_robust_template.restype = ctypes.c_int
    L.fbp_residual_covariance.argtypes = [vp, vp, vp, vp, u32, u32, u32, u32, vp, vp]
    L.fbp_residual_covariance.restype = ctypes.c_int
    L.fbp_set_tuning.argtypes = [P(FbpTuning)]
    L.fbp_set_tuning.restype = ctypes.c_int
    _lib = L
    return L


def check(status):
    if status != FBP_OK:
        raise FbpError(status, lib().fbp_last_error().decode(errors="replace"))
    return status


def dims(n_chans, n_samples, n_templates, template_len, n_max_shift, work_group=256):
    return FbpDims(int(n_chans), int(n_samples), int(n_templates), int(template_len),
                   int(n_max_shift), int(work_group))


def workspace_bytes(d: FbpDims, flags: int) -> int:
    return int(lib().fbp_workspace_bytes(ctypes.byref(d), int(flags)))
