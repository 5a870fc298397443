"""Build the in-tree shared library libwds_b200.so for sm_100a with nvcc.

    python -m wdsgpu_b200.build          # or __graft_entry__.build()

The library is a plain C-ABI shared object (no torch types in its
signatures); Python reaches it through ctypes.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = ["csrc/wds_plan.cu", "csrc/wds_kernels.cu"]
LIB = os.path.join(HERE, "libwds_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(verbose=False, extra=()):
    srcs = [os.path.join(HERE, s) for s in SRC]
    deps = srcs + [os.path.join(HERE, "csrc", "wds_internal.h"),
                   os.path.join(REPO, "include", "wds_b200.h")]
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps) \
            and not extra:
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(REPO, "include"), "-I", os.path.join(HERE, "csrc"),
           *extra, "-o", LIB, *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
