"""Failure detection without a GPU fault: a NaN planted in the amplitudes (host data, through
ccdgpu_set_t2) makes the next iteration's energy non-finite; the energy reduction sets the
device error bit and the call returns CCDGPU_ERR_NONFINITE.  No trap, no bad address: the
handle is then destroyed normally."""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDGPUError, CCDSolver
from helpers import golden, system_for

pytestmark = pytest.mark.gpu


def test_nonfinite_amplitudes_are_reported():
    g = golden("eg14_s19")
    with system_for(g) as s, CCDSolver(s) as sol:
        t2 = np.zeros(sol.n_t2)
        t2[sol.n_t2 // 2] = np.nan
        sol.set_t2(t2)
        with pytest.raises(CCDGPUError) as ei:
            sol.step(0.5)
        assert ei.value.status == -5
