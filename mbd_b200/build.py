"""Build libmbd_b200.so in-tree with nvcc for sm_100a.

    python -m mbd_b200.build          # incremental
    python -m mbd_b200.build --force  # rebuild everything

Objects go to mbd_b200/_build/, the library to mbd_b200/libmbd_b200.so.
The CUDA runtime is linked statically (nvcc's default), so the library does
not depend on which libcudart the host process loaded.  The pmbd.x front end
(host/pmbd_b200.cpp) is linked against the library into mbd_b200/pmbd_b200,
which finds libmbd_b200.so beside itself (rpath $ORIGIN).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmbd_b200.so")
HOST = os.path.join(HERE, "host")
EXE = os.path.join(HERE, "pmbd_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libmbd_b200.so")


def _deps() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(d) for d in _deps()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [nvcc()] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd += ["-Xptxas", "-warn-spills"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    build_host(force)
    if verbose:
        print(f"built {LIB} and {EXE}")
    return LIB


def build_host(force: bool = False) -> str:
    """Link the pmbd_b200 executable (plain C++, no device code) against
    libmbd_b200.so."""
    src = os.path.join(HOST, "pmbd_b200.cpp")
    deps = [src, LIB, os.path.join(HOST, "pmbd_io.h"), os.path.join(ROOT, "include", "mbd_b200.h")]
    if not force and os.path.exists(EXE) and os.path.getmtime(EXE) >= max(os.path.getmtime(d) for d in deps):
        return EXE
    cxx = shutil.which("g++") or "c++"
    # --allow-shlib-undefined: the library's own references into the CUDA
    # driver resolve when it is loaded on a GPU machine; a build machine
    # without a driver cannot resolve them at link time
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), "-I", HOST, src,
           "-o", EXE, "-L", HERE, "-lmbd_b200", "-Wl,-rpath,$ORIGIN", "-Wl,--allow-shlib-undefined"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"host link failed:\n{res.stdout}\n{res.stderr}")
    return EXE


if __name__ == "__main__":
    build(force="--force" in sys.argv)
