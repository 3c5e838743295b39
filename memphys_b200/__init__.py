"""memphys_b200 -- B200-native (sm_100a) hot path of the MeMPhyS meshless solver.

The CUDA kernels and the C-ABI live in ``csrc/`` and build into
``libmemphys_cuda.so`` (see ``build.py``); ``capi`` binds that library and
``meshless`` mirrors the reference's PARAMETERS / POINTS / CLOUD / SOLVER /
FRACTIONAL_STEP_1 interface on top of it.  ``clouds`` generates the seeded
synthetic point clouds.  Importing this package does not load the CUDA
library; the first call that needs it does, and raises if it is missing.
"""
__all__ = ["clouds", "capi", "meshless"]
