"""Build the reference strokelib and gridencoder CUDA extensions, unmodified, into
oracle/_ref/.

TEST INFRASTRUCTURE ONLY. The product never imports or links anything under
``oracle/``; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg may use it, and only as a checker.

Recipe: the four reference source files (source/strokelib/src/strokes_forward.cu,
strokes_backward.cu, compositing.cu, bindings.cpp) are compiled where they lie in
the read-only reference checkout with the reference's own flags
(source/strokelib/backend.py:6-12: -O3 -std=c++17 and the three -U__CUDA_NO_HALF*
switches) plus the sm_100a target, through torch's ``cpp_extension.load`` exactly
as backend.py:34-44 does. Objects and the resulting ``_strokelib*.so`` go to
``oracle/_ref/`` only. The .so is git-ignored but travels to the GPU box, where the
GPU parity tests load it as the reference op.

The grid encoder (source/gridencoder/src/gridencoder.cu, bindings.cpp) is built
the same way, as backend.py:33-39 of that package does, into ``oracle/_ref/grid/``
as ``_gridencoder*.so``; its flags ask for C++14, which torch's headers no longer
accept, so it is compiled as C++17 like the strokelib.

The checkout is found through ``reference_root()``: the ``N3DS_REFERENCE``
environment variable, else the default location below (this recipe's only machine
path).

Usage: python oracle/build_ref.py [--ref PATH] [--jobs 3] [--only strokes|grid]
"""
import argparse
import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SOURCES = ["strokes_forward.cu", "strokes_backward.cu", "compositing.cu", "bindings.cpp"]


DEFAULT_REFERENCE = "/root/reference"


def reference_root():
    """The read-only reference checkout: $N3DS_REFERENCE, else DEFAULT_REFERENCE."""
    return os.environ.get("N3DS_REFERENCE") or DEFAULT_REFERENCE


GRID_OUT = os.path.join(OUT, "grid")
GRID_SOURCES = ["gridencoder.cu", "bindings.cpp"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-U__CUDA_NO_HALF_OPERATORS__",
              "-U__CUDA_NO_HALF_CONVERSIONS__", "-U__CUDA_NO_HALF2_OPERATORS__"]


def built_path():
    """Return the path of the built reference strokelib extension, or None."""
    hits = sorted(glob.glob(os.path.join(OUT, "_strokelib*.so")))
    return hits[0] if hits else None


def grid_built_path():
    """Return the path of the built reference gridencoder extension, or None."""
    hits = sorted(glob.glob(os.path.join(GRID_OUT, "_gridencoder*.so")))
    return hits[0] if hits else None


def build_grid(ref_root=None, jobs=3, verbose=True):
    ref_root = ref_root or reference_root()
    src_dir = os.path.join(ref_root, "source", "gridencoder", "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference gridencoder sources not found at {src_dir}")
    os.makedirs(GRID_OUT, exist_ok=True)
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0a"
    os.environ.setdefault("MAX_JOBS", str(jobs))
    from torch.utils.cpp_extension import load

    load(name="_gridencoder",
         sources=[os.path.join(src_dir, f) for f in GRID_SOURCES],
         extra_cflags=["-O3", "-std=c++17"],
         extra_cuda_cflags=NVCC_FLAGS,
         build_directory=GRID_OUT,
         verbose=verbose)
    return grid_built_path()


def build(ref_root=None, jobs=3, verbose=True):
    ref_root = ref_root or reference_root()
    src_dir = os.path.join(ref_root, "source", "strokelib", "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference strokelib sources not found at {src_dir}")
    os.makedirs(OUT, exist_ok=True)
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0a"
    os.environ.setdefault("MAX_JOBS", str(jobs))
    from torch.utils.cpp_extension import load

    load(name="_strokelib",
         sources=[os.path.join(src_dir, f) for f in SOURCES],
         extra_cflags=["-O3", "-std=c++17"],
         extra_cuda_cflags=NVCC_FLAGS,
         extra_include_paths=[src_dir],
         build_directory=OUT,
         verbose=verbose)
    return built_path()


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (default: reference_root())")
    ap.add_argument("--jobs", type=int, default=3)
    ap.add_argument("--only", choices=["strokes", "grid"], default=None)
    a = ap.parse_args()
    ok = True
    if a.only in (None, "strokes"):
        p = build(a.ref, a.jobs)
        print("built:", p)
        ok = ok and p is not None
    if a.only in (None, "grid"):
        p = build_grid(a.ref, a.jobs)
        print("built:", p)
        ok = ok and p is not None
    sys.exit(0 if ok else 1)
