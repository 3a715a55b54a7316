"""Build the native library ``wavemoth_b200/libwavemoth_b200.so`` in-tree.

Every CUDA source is compiled for sm_100a only; host C++ sources go through
nvcc as well so that one shared object carries the kernels, the host plan
code and the C-ABI (include/wavemoth.h, include/wavemoth_b200.h).

Usage: ``python -m wavemoth_b200.build`` (or ``build()`` from Python).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libwavemoth_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; cannot build the wavemoth_b200 CUDA library")
    return cand


def sources():
    srcs = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith(".cu") or name.endswith(".cpp"):
            srcs.append(os.path.join(CSRC, name))
    return srcs


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(verbose=False, ptxas_verbose=False):
    nvcc = _nvcc()
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, n) for n in os.listdir(CSRC)
               if n.endswith((".h", ".cuh", ".hpp"))]
    headers += [os.path.join(ROOT, "include", n) for n in os.listdir(os.path.join(ROOT, "include"))]
    objs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if not _stale(obj, src, headers):
            continue
        cmd = [nvcc] + ARCH + COMMON + ["-c", src, "-o", obj]
        if ptxas_verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    need_link = not os.path.exists(OUT) or any(
        os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs)
    if need_link:
        cmd = [nvcc] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv))
