"""Channel construction on the device (ccdgpu_build_channels, SPBasis.cpp:80-441 with the
one-rank ffdBalance order): the builder run with CCDHOST_DEVICE_CHANNELS must produce the
reference's channel dimensions, channel maps, three-body dimensions and remap tables bit for
bit (FNV-1a hashes of the reference's own dumps), and the same solve."""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, System
from helpers import MAPS, SMALL, STRUCT, VKINDS, golden, system_for
from oracle.oracle import fnv1a

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", SMALL + ["eg54_s19"])
def test_device_channels_match_reference(name):
    g = golden(name)
    with getattr(System, g["kind"])(**g["params"], device_channels=True) as s:
        assert s.reference_energy == float(g["scalars"][0])
        assert s.mbpt2 == float(g["scalars"][1])
        for k, n in enumerate(STRUCT):
            assert fnv1a(s.array(n)) == int(g["struct_hashes"][k]), n
        for k, n in enumerate(MAPS):
            assert fnv1a(s.array(n)) == int(g["map_hashes"][k]), n
        for k, n in enumerate(VKINDS):
            assert fnv1a(s.array(n)) == int(g["v_hashes"][k]), n


def test_device_channels_structure_only_solve():
    """Structure from the device, no tables and no V from the host: the same solve."""
    g = golden("eg14_s19")
    with system_for(g) as s1, System.electron_gas(**g["params"], device_channels=True,
                                                  tables=False, v_blocks=False,
                                                  load_v_pppp=False) as s2, \
            CCDSolver(s1) as a, CCDSolver(s2, v_mode="on_the_fly") as b:
        ra = a.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        rb = b.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        assert ra.iterations == rb.iterations
        np.testing.assert_array_equal(a.t2(), b.t2())
