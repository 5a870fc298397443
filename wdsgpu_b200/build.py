"""Build the in-tree shared library libwds_b200.so for sm_100a with nvcc.

    python -m wdsgpu_b200.build          # or __graft_entry__.build()

The library is a plain C-ABI shared object (no torch types in its
signatures); Python reaches it through ctypes.  Every translation unit is
compiled separately and in parallel (the kernel-instance sources once per
factor precision), into wdsgpu_b200/_build/, then linked; an object is
rebuilt when its source or any header is newer.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwds_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# (source, object name, extra defines); the k_* sources are compiled once per
# factor precision
UNITS = [("wds_plan.cu", "wds_plan", ()), ("wds_launch.cu", "wds_launch", ())]
for _k in ("forward", "adjoint", "unrolled", "multi"):
    UNITS += [("wds_k_%s.cu" % _k, "wds_k_%s_f64" % _k, ("-DWDS_FP32=0",)),
              ("wds_k_%s.cu" % _k, "wds_k_%s_f32" % _k, ("-DWDS_FP32=1",))]
HEADERS = [os.path.join(CSRC, "wds_internal.h"), os.path.join(CSRC, "wds_device.cuh"),
           os.path.join(REPO, "include", "wds_b200.h")]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra=(), jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    base = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
            "-I", os.path.join(REPO, "include"), "-I", CSRC, *extra]
    cmds, objs = [], []
    for src, name, defs in UNITS:
        o = os.path.join(OBJ, name + ".o")
        objs.append(o)
        s = os.path.join(CSRC, src)
        if extra or _stale(o, [s] + HEADERS):
            cmds.append([*base, *defs, "-c", "-o", o, s])
    if cmds:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            futs = []
            for c in cmds:
                if verbose:
                    print(" ".join(c), flush=True)
                futs.append(ex.submit(subprocess.run, c, capture_output=True, text=True))
            fails = []
            for c, f in zip(cmds, futs):
                r = f.result()
                if verbose and (r.stdout or r.stderr):
                    print(r.stdout + r.stderr, flush=True)
                if r.returncode != 0:
                    fails.append((c[-1], r.stderr))
            if fails:
                raise RuntimeError("nvcc failed:\n" + "\n".join("%s:\n%s" % f for f in fails))
    if cmds or _stale(LIB, objs):
        link = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs]
        if verbose:
            print(" ".join(link), flush=True)
        subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
