"""CPU oracle for the stroke-field path.

TEST INFRASTRUCTURE ONLY. Nothing in the product package imports, calls or links
anything under ``oracle/``. Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference legs may use it, and only as the checker or
as the labelled CPU port that is timed beside the CUDA path.

Contents
- ``strokefield``: line-by-line torch restatement of the reference strokelib kernels
  (source/strokelib/src/strokes_forward.cu, strokes_backward.cu, compositing.cu,
  strokes_sdf.h, common.h). It is dtype-generic: in float64 with torch.autograd it is
  the exact-gradient oracle; in float32 it is the CPU port of the reference op.
- ``render``: restatement of source/utils/render.py (cast_rays,
  compute_alpha_weights, volumetric_rendering).
- ``scenes``: seeded synthetic scene/ray generators with the shapes and value
  distributions of the benchmark configurations.
- ``build_ref.py``: compiles the unmodified reference strokelib extension into
  ``oracle/_ref/`` (GPU-box comparator).

Parity pinning: the restatement is checked against golden vectors under
``tests/golden/`` produced by the reference itself (render.py imported in FP64 on
CPU; the reference strokelib layouts from strokes.py; the reference CUDA op run on a
B200 through ``oracle/_ref``) by the scripts that sit beside those fixtures.
"""
