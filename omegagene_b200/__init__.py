"""omegagene_b200 -- B200 (sm_100a) engine for omegagene's per-step MD hot path.

Host mirror of the C ABI in include/omegagene_b200.h; the compute path is the in-tree CUDA
library libomegagene_b200.so (see omegagene_b200/build.py).
"""
from . import cls_io, systems  # noqa: F401

__all__ = ["cls_io", "systems", "engine"]
