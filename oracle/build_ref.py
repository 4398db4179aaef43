"""Recipe: compile the reference's OpenCL kernels for the CPU into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Reads spikesorting_fullpursuit/kernels/binary_pursuit.cl
where it lies in the reference checkout (nothing of it is committed), applies
one scripted line rewrite, and compiles it with oracle/ref_shim.cpp into
oracle/_ref/libbp_ref.so.  Outputs go only to oracle/_ref/ (git-ignored).

The rewrite: the kernel-scope ``__local unsigned int global_offset;`` of the
binary_pursuit kernel (binary_pursuit.cl:968) becomes a reference to one
per-work-group slot, because a C++ local would be private to each work-item.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference checkout beside the repository, unless FBP_REFERENCE_CL names the kernel file
REF_CL = os.environ.get(
    "FBP_REFERENCE_CL",
    os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "spikesorting_fullpursuit", "kernels",
                 "binary_pursuit.cl"))
LIB = os.path.join(OUT, "libbp_ref.so")


def reference_present() -> bool:
    return os.path.exists(REF_CL)


def build(force: bool = False) -> str | None:
    """Build oracle/_ref/libbp_ref.so; returns its path, or None when the
    reference checkout is absent and no prebuilt library exists."""
    if not reference_present():
        return LIB if os.path.exists(LIB) else None
    os.makedirs(OUT, exist_ok=True)
    with open(REF_CL, "r") as fp:
        src = fp.read()
    digest = hashlib.sha256(src.encode()).hexdigest()
    pat = re.compile(r"^(\s*)__local unsigned int global_offset;\s*$", re.M)
    if len(pat.findall(src)) != 1:
        raise RuntimeError("unexpected reference kernel source: global_offset line not found once")
    src = pat.sub(r"\1__local unsigned int &global_offset = *clshim_group_u32();", src)
    inc = os.path.join(OUT, "binary_pursuit_ref.inc")
    shim = os.path.join(HERE, "ref_shim.cpp")
    stamp = os.path.join(OUT, "SOURCE_SHA256")
    if (not force and os.path.exists(LIB) and os.path.exists(stamp)
            and open(stamp).read().strip() == digest
            and os.path.getmtime(LIB) >= os.path.getmtime(shim)):
        return LIB
    with open(inc, "w") as fp:
        fp.write(src)
    tmp = LIB + ".tmp%d" % os.getpid()
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math",
                           "-fwrapv", "-fno-strict-aliasing", "-fopenmp", "-fPIC", "-shared",
                           "-w", "-I", OUT, "-o", tmp, shim])
    os.replace(tmp, LIB)
    with open(stamp, "w") as fp:
        fp.write(digest + "\n")
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv)
    print(path if path else "reference checkout absent; nothing built")
