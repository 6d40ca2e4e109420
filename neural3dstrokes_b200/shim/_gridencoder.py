"""Module named like the reference's native grid-encoder extension: with this
directory on sys.path, the reference's ``import _gridencoder``
(source/gridencoder/grid.py:9-12) binds the B200 kernels instead of JIT-building
its own."""
from neural3dstrokes_b200.gridencoder import (grad_total_variation, grid_encode_backward,  # noqa: F401
                                              grid_encode_forward)
