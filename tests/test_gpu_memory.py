"""Process-wide reuse of device memory across handles.

A destroyed handle's device blocks stay in the library's cache and serve the next create on
the same device; ccdgpu_release_cached_memory gives them back.  Device free memory is read
with cudaMemGetInfo (through torch, same primary context).
"""
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, _native
from helpers import golden, system_for

pytestmark = pytest.mark.gpu

MiB = 1 << 20


def test_device_memory_is_cached_reused_and_released():
    import torch
    lib = _native.gpu_lib()
    torch.cuda.init()
    lib.ccdgpu_release_cached_memory()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    g = golden("eg14_s19")
    with system_for(g) as s:
        with CCDSolver(s) as sol:
            e1 = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5).e_corr
        free1 = torch.cuda.mem_get_info()[0]
        assert free0 - free1 > 8 * MiB  # kept by the cache after destroy
        with CCDSolver(s) as sol:
            e2 = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5).e_corr
        free2 = torch.cuda.mem_get_info()[0]
        assert free1 - free2 < 64 * MiB  # the second handle ran on the cached blocks
        assert e1 == e2
    lib.ccdgpu_release_cached_memory()
    free3 = torch.cuda.mem_get_info()[0]
    assert free3 > free1 + 8 * MiB
    assert abs(free3 - free0) < 8 * MiB
