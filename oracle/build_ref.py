"""Build the reference strokelib CUDA extension, unmodified, into oracle/_ref/.

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

Usage: python oracle/build_ref.py [--ref /root/reference] [--jobs 3]
"""
import argparse
import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SOURCES = ["strokes_forward.cu", "strokes_backward.cu", "compositing.cu", "bindings.cpp"]


def built_path():
    """Return the path of the built reference extension, or None."""
    hits = sorted(glob.glob(os.path.join(OUT, "_strokelib*.so")))
    return hits[0] if hits else None


def build(ref_root="/root/reference", jobs=3, verbose=True):
    src_dir = os.path.join(ref_root, "source", "strokelib", "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference strokelib sources not found at {src_dir}")
    os.makedirs(OUT, exist_ok=True)
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0a"
    os.environ.setdefault("MAX_JOBS", str(jobs))
    from torch.utils.cpp_extension import load

    nvcc_flags = ["-O3", "-std=c++17", "-U__CUDA_NO_HALF_OPERATORS__",
                  "-U__CUDA_NO_HALF_CONVERSIONS__", "-U__CUDA_NO_HALF2_OPERATORS__"]
    load(name="_strokelib",
         sources=[os.path.join(src_dir, f) for f in SOURCES],
         extra_cflags=["-O3", "-std=c++17"],
         extra_cuda_cflags=nvcc_flags,
         extra_include_paths=[src_dir],
         build_directory=OUT,
         verbose=verbose)
    return built_path()


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--jobs", type=int, default=3)
    a = ap.parse_args()
    p = build(a.ref, a.jobs)
    print("built:", p)
    sys.exit(0 if p else 1)
