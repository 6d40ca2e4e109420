"""Build the in-tree CUDA library ``neural3dstrokes_b200/lib/libn3ds.so`` for sm_100a.

Plain nvcc, no torch dependency in the library: every translation unit under
``csrc/`` is compiled with ``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``
and linked into one shared object with a C ABI (``include/n3ds.h``). Objects are
cached next to the library and rebuilt when a source or header is newer.

Usage: python -m neural3dstrokes_b200.build [--force] [--verbose] [--ptxas]
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.environ.get("N3DS_BUILD_DIR") or os.path.join(PKG, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libn3ds.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Approximate (MUFU-based) sqrt and division and flush-to-zero of denormals: the
# stroke kernels are FP32 issue-bound and their IEEE-rounded sqrt/div sequences cost
# several instructions each; the 1-2 ulp difference is far inside the 1e-5 tolerance.
FAST_MATH = ["-prec-sqrt=false", "-prec-div=false", "-ftz=true"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC] + \
    ([] if os.environ.get("N3DS_IEEE_MATH") else FAST_MATH)


def nvcc_path():
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found (set NVCC or put CUDA's bin on PATH)")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas=False, jobs=None):
    """Compile (if stale) and return the path of libn3ds.so."""
    nvcc = nvcc_path()
    os.makedirs(OBJDIR, exist_ok=True)
    headers = _headers()
    srcs = _sources()
    extra = ["-Xptxas", "-v"] if ptxas else []

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.basename(src).replace(".cu", ".o"))
        if not force and not ptxas and not _stale(obj, [src] + headers):
            return obj, ""
        cmd = [nvcc] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stdout + r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, srcs))
    objs = [o for o, _ in results]
    if ptxas or verbose:
        for _, log in results:
            if log:
                print(log, flush=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas))
    sys.exit(0)
