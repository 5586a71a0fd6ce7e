"""The CPU oracle is pinned to the reference: per-iteration energies, iteration counts and the
converged T2 of the reference's own runs (tests/golden, made by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from helpers import EXTRA, SMALL, golden, system_for
from oracle.oracle import Oracle


@pytest.mark.parametrize("name", SMALL + EXTRA)
def test_oracle_matches_reference(name):
    g = golden(name)
    with system_for(g) as s:
        o = Oracle(s)
        e, n, en = o.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        ref = g["energies"]
        assert n == len(ref)
        np.testing.assert_allclose(en, ref, rtol=1e-12, atol=1e-15)
        assert abs(e - ref[-1]) <= 1e-12 * abs(ref[-1])
        t2 = o.t2()
        t2 = t2 if int(g["t2_full"][0]) else t2[::97]
        assert np.max(np.abs(t2 - g["t2"])) < 1e-12
        o.close()


def test_oracle_readme_known_answer():
    """src/README.md:8-10: E_CCD/A = 10.155078 for PNM rho=0.08, 14 neutrons, tol 1e-8."""
    g = golden("pnm14_s4")
    with system_for(g) as s:
        o = Oracle(s)
        e, n, _ = o.solve(tol=1e-8)
        assert round((s.reference_energy + e) / s.n_particles, 6) == 10.155078
        o.close()


def test_oracle_iteration_cap():
    """g=+1.0 pairing does not converge: the loop stops after 101 iterations (main.cpp:509-519)."""
    g = golden("pairing_gp1.0")
    with system_for(g) as s:
        o = Oracle(s)
        _, n, _ = o.solve(tol=1e-12, max_iters=100)
        assert n == 101
        o.reset()
        _, n, _ = o.solve(tol=1e-12, max_iters=5)
        assert n == 6
        o.close()


def test_oracle_detects_planted_mistake():
    """A planted error in the oracle's input (one V_hhpp element) must move the energy: the
    checker is sensitive to the data it checks."""
    g = golden("pnm14_s4")
    with system_for(g) as s:
        p = s.problem.contents
        # first amplitude-carrying channel
        d = s.chan_dims()
        c = int(np.nonzero((d[:, 0] > 0) & (d[:, 1] > 0))[0][0])
        blk = p.v_hhpp[c]
        old = blk[0]
        blk[0] = old + 0.1
        o = Oracle(s)
        e, _, _ = o.solve(tol=g["tol"])
        blk[0] = old
        assert abs(e - float(g["scalars"][2])) > 1e-6
        o.close()
