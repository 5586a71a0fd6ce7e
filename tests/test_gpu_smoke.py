"""The round-end smoke check (__graft_entry__.smoke) runs as a GPU test too: the known answer
E_CCD/A = 10.155078 for pure neutron matter at rho = 0.08 fm^-3, N = 14, through the C ABI and
against the oracle."""
import os
import sys

import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def test_smoke_entry():
    import __graft_entry__
    __graft_entry__.smoke()
