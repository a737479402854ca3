"""afid_b200: B200-native FP64 implementation of AFiD's RK3 time-step hot path.

The compute path is libafid_gpu.so (hand-written CUDA for sm_100a behind the
C-ABI in include/afid_gpu.h); this package is its host-side mirror.
"""
from .config import BouIn, read_bou_in, write_bou_in, largest_factor  # noqa: F401
from .solver import Box, Context, make_grid, device_bytes  # noqa: F401
from .ic import seeded_noise, initial_fields  # noqa: F401

__all__ = ["BouIn", "read_bou_in", "write_bou_in", "Box", "Context", "make_grid",
           "device_bytes", "seeded_noise", "initial_fields", "largest_factor"]
