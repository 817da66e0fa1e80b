"""Host-side mirror of the FESOM-C time-step interface for the B200 library.

The compute path is the in-tree CUDA library libfesomc_gpu.so (C-ABI in
include/fesomc_gpu.h); this package only binds it with ctypes, builds test
cases and drives the reference-style main loop.
"""
from . import abi  # noqa: F401
