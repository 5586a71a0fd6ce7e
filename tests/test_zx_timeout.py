"""Failure detection on the GPU without a fault: a bounded device wait that runs out.

Every mbarrier wait of the pipelined kernels gives up after 1 s of %globaltimer, sets an error
bit and lets the kernel end; the host reads the bit and returns CCDGPU_ERR_TIMEOUT.  The test
hook ccdgpu_inject_wait_timeout makes the first CTA of each FP64 pp-ladder class withhold its
first shared-memory stage in the next iteration (a stage that nothing fills), so its consumers'
waits and then its producer's wait run out.  The test checks the status, the time it took, and
that the handle then solves to the reference's answer.
"""
import time

import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDGPUError, CCDSolver
from helpers import golden, system_for, t2_sample

pytestmark = pytest.mark.gpu

STATUS_TIMEOUT = -9


@pytest.mark.parametrize("path", ["fused", "tables"])
def test_expired_wait_returns_timeout_and_handle_recovers(path):
    g = golden("pnm14_s4")
    with system_for(g) as s, CCDSolver(s, path=path) as sol:
        for _ in range(2):
            sol.step(0.5)
        sol.inject_wait_timeout()
        t0 = time.perf_counter()
        with pytest.raises(CCDGPUError) as exc:
            sol.step(0.5)
        waited = time.perf_counter() - t0
        assert exc.value.status == STATUS_TIMEOUT
        assert 0.9 <= waited < 30.0
        # Reported once; the next iterations run normally from a fresh start.
        sol.reset()
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        assert abs(res.iterations - len(g["energies"])) <= 1
        e_ref = float(g["energies"][-1])
        assert abs(res.e_corr - e_ref) <= 1e-10 * abs(e_ref)
        assert np.max(np.abs(t2_sample(g, sol.t2()) - g["t2"])) < 1e-9
        # The hook applies to one step only.
        sol.reset()
        sol.step(0.5)
