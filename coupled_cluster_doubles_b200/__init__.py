"""B200-native drop-in for the CCD T2 iteration of justinlietz/coupled_cluster_doubles.

System      host-side problem (basis, channels, V blocks, remap tables): libccdhost.so
CCDSolver   the CUDA iteration behind the C ABI of include/ccdgpu.h: libccdgpu.so
"""
from .system import System  # noqa: F401
from .solver import CCDSolver, CCDGPUError, Result, solve_batch  # noqa: F401
