"""Build ``libmeeuuw_b200.so`` (sm_100a) in-tree with nvcc.

    python -m meeuuw_b200.build [-v]

Every ``csrc/*.cu`` is compiled with ``-gencode arch=compute_100a,code=sm_100a`` and linked
into one shared library with a static CUDA runtime, so the library needs nothing at run time
but the driver.  Files listed in ``NO_FMA`` are built with ``-fmad=false``: their arithmetic
reproduces the reference's unfused double-precision rounding.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmeeuuw_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", os.path.join(ROOT, "include")]
NO_FMA = {"pic.cu"}
# extra nvcc flags for measurements (e.g. MW_NVCC_FLAGS="-DMW_APPLY_MINB=6"); empty by default
EXTRA = os.environ.get("MW_NVCC_FLAGS", "").split()


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src, verbose):
    obj = os.path.join(BUILD, src[:-3] + ".o")
    dep = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    dep.append(os.path.join(ROOT, "include", "meeuuw_b200.h"))
    if not EXTRA and os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in dep):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + EXTRA + (["-fmad=false"] if src in NO_FMA else []) + \
        ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 or verbose:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}")
    return obj


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), sources()))
    if not EXTRA and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
