"""B200-native (sm_100a) stroke field of Neural 3D Strokes.

- ``neural3dstrokes_b200.strokelib``: drop-in for the reference native module
  ``_strokelib`` (stroke_forward, stroke_backward, compose_forward, compose_backward);
  ``neural3dstrokes_b200/shim`` on sys.path makes ``import _strokelib`` resolve to it.
- ``neural3dstrokes_b200.strokes``: the reference Python API (get_stroke,
  compose_strokes) over that backend.
- ``neural3dstrokes_b200.field``: the fused stroke field (evaluation, soft step,
  overlay compositing, volume rendering, exact adjoint) for one scene or a batch.
- ``neural3dstrokes_b200.train``: batched graph-captured training step with Adam.

All compute runs in the in-tree CUDA library ``lib/libn3ds.so`` (C ABI,
include/n3ds.h); there is no CPU fallback.
"""
__version__ = "0.1.0"
