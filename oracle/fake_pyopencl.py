"""A stand-in for the ``pyopencl`` module over oracle/_ref/libbp_ref.so.

TEST INFRASTRUCTURE ONLY.  It implements the part of the pyopencl API that the
reference's host function binary_pursuit()
(spikesorting_fullpursuit/overlap/binary_pursuit_parallel.py:175-1532) calls, so
that function runs unmodified with its kernels executed on the CPU by the
shim.  Install it with ``install()`` before importing the reference module.

One device is exposed, typed GPU so the reference's device search accepts it
(binary_pursuit_parallel.py:283-293).  Every kernel reports the same
work-group size (``WORK_GROUP_SIZE``, default 256).  Buffers carry 64 zero
bytes of slack past their end: the reference's binary_pursuit kernel reads
overlap_recheck[N/W + 1] for padding work-items (binary_pursuit.cl:939-944,
982), one or two bytes past the buffer, and the slack makes that read 0.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

WORK_GROUP_SIZE = 256
GLOBAL_MEM_SIZE = 8 * 1024 ** 3
MAX_COMPUTE_UNITS = 8
THREADS = os.cpu_count() or 1
# callables invoked as hook(kernel_name, kernel) after every launch
launch_hooks: list = []


class _Arg(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("size", ctypes.c_uint64), ("ptr", ctypes.c_void_p)]


_lib = None


def _shim():
    global _lib
    if _lib is None:
        sys.path.insert(0, HERE)
        import build_ref  # noqa: E402
        path = build_ref.build()
        if path is None:
            raise RuntimeError("oracle/_ref/libbp_ref.so is missing and the reference is absent")
        _lib = ctypes.CDLL(path)
        _lib.clshim_launch.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_Arg),
                                       ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_int]
        _lib.clshim_launch.restype = ctypes.c_int
        _lib.clshim_nargs.argtypes = [ctypes.c_char_p]
        _lib.clshim_nargs.restype = ctypes.c_int
    return _lib


class device_type:
    GPU = 4
    CPU = 2
    ALL = 0xFFFFFFFF


class device_info:
    GLOBAL_MEM_SIZE = "GLOBAL_MEM_SIZE"
    ADDRESS_BITS = "ADDRESS_BITS"
    MAX_WORK_GROUP_SIZE = "MAX_WORK_GROUP_SIZE"


class kernel_work_group_info:
    WORK_GROUP_SIZE = "WORK_GROUP_SIZE"


class mem_flags:
    READ_WRITE = 1
    WRITE_ONLY = 2
    READ_ONLY = 4
    COPY_HOST_PTR = 32


class Device:
    max_compute_units = MAX_COMPUTE_UNITS

    def get_info(self, key):
        if key == device_info.GLOBAL_MEM_SIZE:
            return GLOBAL_MEM_SIZE
        if key == device_info.ADDRESS_BITS:
            return 64
        if key == device_info.MAX_WORK_GROUP_SIZE:
            return WORK_GROUP_SIZE
        raise KeyError(key)


class Platform:
    def get_devices(self, dtype=device_type.ALL):
        return [Device()] if dtype in (device_type.GPU, device_type.ALL) else []


def get_platforms():
    return [Platform()]


class Context:
    def __init__(self, devices):
        self.devices = devices


class Event:
    def wait(self):
        return None


class CommandQueue:
    def __init__(self, ctx):
        self.ctx = ctx

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def finish(self):
        return None


class Buffer:
    def __init__(self, ctx, flags, size=None, hostbuf=None):
        if hostbuf is not None:
            src = np.ascontiguousarray(hostbuf).view(np.uint8).reshape(-1)
            self.nbytes = src.size
            self.mem = np.zeros(self.nbytes + 64, dtype=np.uint8)
            self.mem[: self.nbytes] = src
        else:
            self.nbytes = int(size)
            self.mem = np.zeros(self.nbytes + 64, dtype=np.uint8)

    @property
    def ptr(self):
        return self.mem.ctypes.data

    def view(self, dtype):
        return self.mem[: self.nbytes].view(dtype)

    def release(self):
        self.mem = np.zeros(64, dtype=np.uint8)
        self.nbytes = 0


class LocalMemory:
    def __init__(self, size):
        self.size = int(size)


class Kernel:
    def __init__(self, name):
        self.name = name
        self.nargs = _shim().clshim_nargs(name.encode())
        if self.nargs < 0:
            raise AttributeError(name)
        self.args = [None] * self.nargs

    def set_arg(self, i, value):
        self.args[i] = value

    def get_work_group_info(self, param, device):
        return WORK_GROUP_SIZE


class Program:
    def __init__(self, ctx, source):
        self.ctx = ctx
        stamp = os.path.join(HERE, "_ref", "SOURCE_SHA256")
        if os.path.exists(stamp):
            want = open(stamp).read().strip()
            got = hashlib.sha256(source.encode()).hexdigest()
            if want != got:
                raise RuntimeError("kernel source differs from the one compiled into libbp_ref.so")

    def build(self, *args, **kwargs):
        return self

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return Kernel(name)


def enqueue_nd_range_kernel(queue, kernel, global_size, local_size, global_work_offset=None,
                            wait_for=None):
    gsize = int(global_size[0])
    lsize = int(local_size[0])
    goff = int(global_work_offset[0]) if global_work_offset is not None else 0
    keep = []
    arr = (_Arg * kernel.nargs)()
    for i, v in enumerate(kernel.args):
        if isinstance(v, Buffer):
            arr[i] = _Arg(0, v.nbytes, v.ptr)
        elif isinstance(v, LocalMemory):
            arr[i] = _Arg(2, v.size, None)
        elif v is None:
            raise RuntimeError("kernel %s argument %d not set" % (kernel.name, i))
        else:
            cell = np.array([int(v)], dtype=np.uint32)
            keep.append(cell)
            arr[i] = _Arg(1, 4, cell.ctypes.data)
    if gsize > 0:
        rc = _shim().clshim_launch(kernel.name.encode(), kernel.nargs, arr, goff, gsize, lsize,
                                   THREADS)
        if rc != 0:
            raise RuntimeError("shim launch of %s failed" % kernel.name)
    for hook in launch_hooks:
        hook(kernel.name, kernel)
    return Event()


def enqueue_copy(queue, dest, src, wait_for=None, **kwargs):
    if isinstance(dest, Buffer) and isinstance(src, np.ndarray):
        b = np.ascontiguousarray(src).view(np.uint8).reshape(-1)
        dest.mem[: b.size] = b
    elif isinstance(dest, np.ndarray) and isinstance(src, Buffer):
        n = dest.nbytes
        flat = dest.reshape(-1).view(np.uint8)
        flat[:] = src.mem[:n]
    else:
        raise TypeError("unsupported enqueue_copy")
    return Event()


def install():
    """Register this module as ``pyopencl`` in sys.modules."""
    mod = sys.modules[__name__]
    sys.modules["pyopencl"] = mod
    return mod


def reference_import_stubs():
    """Stub modules the reference package imports but this path never uses:
    isosplit6 (consolidate.py:3, dim_reduce/pca.py:3), mkl
    (spikesorting_parallel.py:25, utils/parallel_funs.py) and the uncompiled
    Cython helper sort_cython."""
    for name in ["isosplit6", "mkl", "spikesorting_fullpursuit.c_cython.sort_cython"]:
        if name in sys.modules:
            continue
        m = types.ModuleType(name)
        if name == "isosplit6":
            m.isosplit6 = lambda *a, **k: None
        if name == "mkl":
            m.set_num_threads = lambda n: None
        sys.modules[name] = m
