"""Build libop2b200.so (the C-ABI library of the B200 backend) in-tree.

Compiles every ``*.cu`` file of this directory for sm_100a with nvcc and
links them, with NVRTC and the CUDA runtime, into ``pyop2_b200/_lib``.
Run ``python -m pyop2_b200.csrc.build`` or call :func:`build`.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "_lib")
LIBNAME = "libop2b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
              "-I" + INCLUDE, "-I" + HERE]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the B200 backend library cannot be built")


def sources():
    return sorted(os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith(".cu"))


def lib_path():
    return os.path.join(LIBDIR, LIBNAME)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it; return its path."""
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    srcs = sources()
    headers = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "op2b200.h"))
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    target = lib_path()
    if force or _stale(target, objs):
        cudalib = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "lib64")
        cmd = [nvcc] + ARCH + ["-shared", "-o", target] + objs + [
            "-L" + cudalib, "-lnvrtc", "-lcudart", "-Xlinker", "-rpath=" + cudalib]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return target


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
