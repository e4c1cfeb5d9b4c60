"""vfs_b200 — B200-native variational fisheye stereo (TGV-L1) solver.

The solver (``StereoTgv``) mirrors the interface of the reference class
(stereotgv/stereotgv.h) over a C ABI (include/vfs_b200.h) whose kernels are hand-written
CUDA for sm_100a.
"""
from ._native import VfsError  # noqa: F401

__version__ = "1.0"


def __getattr__(name):
    # the solver loads the CUDA library on first use
    if name == "StereoTgv":
        from .stereotgv import StereoTgv
        return StereoTgv
    raise AttributeError(name)
