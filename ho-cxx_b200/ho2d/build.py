"""Build the in-tree CUDA library ``ho2d/_lib/libho2d.so`` (sm_100a) with nvcc.

Sources are ``ho-cxx_b200/csrc/*.cu`` and ``*.cpp``; objects go to ``ho-cxx_b200/_build``.
A source is recompiled when it or any header under ``csrc/`` or ``include/`` is newer
than its object. ``python -m ho2d.build`` (from ``ho-cxx_b200/``) builds; ``--cli`` also
links the ``ho2d_main`` command-line driver.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)  # ho-cxx_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIB_DIR, "libho2d.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


NO_FMAD = {"setup_device.cu", "output_device.cu"}


def _flags(src: str) -> list[str]:
    common = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC,-fopenmp", "-I", CSRC,
              "-I", os.path.join(REPO, "include")]
    if src.endswith(".cu"):
        # the device setup reproduces the host assembly bit for bit: no contraction to FMA
        extra = ["-fmad=false"] if os.path.basename(src) in NO_FMAD else []
        return common + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"] + extra
    return common + ["-x", "c++"]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, hmt: float, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hmt):
        return obj
    cmd = [nvcc(), "-c", src, "-o", obj] + _flags(src)
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, cli: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    srcs = [s for s in srcs if not s.endswith("ho2d_main.cpp")]
    hmt = _headers_mtime()
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile(s, hmt, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fopenmp", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if cli:
        main_src = os.path.join(CSRC, "ho2d_main.cpp")
        exe = os.path.join(LIB_DIR, "ho2d_main")
        cmd = [nvcc(), main_src, "-o", exe, "-std=c++17", "-O2", "-I", CSRC, "-I", os.path.join(REPO, "include"),
               "-L", LIB_DIR, "-lho2d", "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, cli="--cli" in sys.argv))
