"""Build ``ggems_b200/libggems.so``: the CUDA transport layer (sm_100a) and the
C++ host API, linked into one shared library that the ctypes module loads.

Usage: python -m ggems_b200.build   (or python ggems_b200/build.py)
"""

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libggems.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


NVCC = ["nvcc", "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
        "-I" + CSRC] + ARCH
# Host code: no fused multiply-add so host-side table building rounds like the reference's host build.
CXX = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fvisibility=hidden",
       "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
# The transport kernels keep the reference's operation order: no contraction into FMA.
FMAD = {"gg_transport.cu": ["-fmad=false"], "gg_volume.cu": ["-fmad=false"]}


def _newer(src, obj, deps=()):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in (src,) + tuple(deps))


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) + \
        glob.glob(os.path.join(CSRC, "**", "*.hh"), recursive=True) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _newer(src, obj, headers):
            cmd = NVCC + FMAD.get(os.path.basename(src), []) + ["-Xptxas", "-v", "-c", src, "-o", obj]
            out = subprocess.run(cmd, capture_output=True, text=True)
            if out.returncode != 0:
                raise RuntimeError("nvcc failed for %s:\n%s" % (src, out.stderr))
            if verbose:
                print(out.stderr)
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "host", "*.cc"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _newer(src, obj, headers):
            subprocess.check_call(CXX + ["-c", src, "-o", obj])
        objs.append(obj)
    cmd = ["nvcc", "-shared"] + ARCH + objs + ["-o", LIB, "-Xcompiler", "-pthread"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
