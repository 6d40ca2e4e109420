"""Module named like the reference's native extension: with this directory on
sys.path, the reference's ``import _strokelib`` (source/strokelib/strokes.py:7-10)
binds the four B200 operators instead of JIT-building its own."""
from neural3dstrokes_b200.strokelib import (compose_backward, compose_forward, stroke_backward,  # noqa: F401
                                            stroke_forward)
