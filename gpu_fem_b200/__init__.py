"""B200-native shell-analysis hot path of smdogroup/gpu_fem.

MITC4 shell residual/Jacobian assembly with a coloured 6x6 BSR scatter,
BSR SpMV, level-ordered block ILU(k) and GMRES, as sm_100a CUDA kernels
behind the C ABI in include/gpufem.h (libgpufem.so).
"""
from . import mesh  # noqa: F401  (host-only, no GPU needed)

__all__ = ["mesh"]
