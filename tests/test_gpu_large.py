"""GPU parity at the large workloads (1850 spin-orbitals, |n|^2 <= 36) against the reference.

The goldens are reference runs (oracle/_ref/ref_harness over the unmodified reference sources,
tests/golden/make_golden.py) at tol 1e-12:
  eg54c36_r2    electron gas, N=54, r_s=2.0   (pp-ladder blocks up to 1796 x 54)
  eg54c36_r05   electron gas, N=54, r_s=0.5
  pnm66_s32     neutron matter, N=66, rho=0.08 fm^-3 (blocks up to 1784 x 66: the FP64 wide
                ladder class at hh 56..72 and the widest ring channels)

Tolerances: FP64 (both paths, stored and generated V): every per-iteration energy within 1e-10
relative of the reference, the converged T2 within 1e-9 max-abs (every 97th element, as
stored in the golden).  Mixed precision (split-bf16 tensor-core ladder, FP64 polish):
|dE/N| <= 1e-7 relative and T2 within 1e-7 max-abs of the reference.
"""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver
from helpers import golden, system_for, t2_sample

pytestmark = pytest.mark.gpu

LARGE = ["eg54c36_r2", "eg54c36_r05", "pnm66_s32"]
E_RTOL = 1e-10
T2_ATOL = 1e-9


def _check_fp64(g, sol, res):
    ref = g["energies"]
    hist = sol.energy_history()
    assert abs(res.iterations - len(ref)) <= 1
    m = min(len(hist), len(ref))
    np.testing.assert_allclose(hist[:m], ref[:m], rtol=E_RTOL, atol=1e-14)
    assert abs(res.e_corr - ref[-1]) <= E_RTOL * abs(ref[-1])
    t2 = sol.t2()
    assert np.max(np.abs(t2_sample(g, t2) - g["t2"])) < T2_ATOL
    np.testing.assert_allclose(float(np.dot(t2, t2)), float(g["t2_sumsq"][0]), rtol=1e-8)


@pytest.mark.parametrize("path", ["fused", "tables"])
@pytest.mark.parametrize("name", LARGE)
def test_large_fp64_matches_reference(name, path):
    g = golden(name)
    with system_for(g) as s, CCDSolver(s, path=path) as sol:
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        _check_fp64(g, sol, res)


@pytest.mark.parametrize("name", LARGE)
def test_large_on_the_fly_fp64_matches_reference(name):
    g = golden(name)
    with system_for(g, load_v_pppp=False) as s, CCDSolver(s, v_mode="on_the_fly") as sol:
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        _check_fp64(g, sol, res)


@pytest.mark.parametrize("v_mode", ["stored", "on_the_fly", "in_ladder"])
@pytest.mark.parametrize("name", LARGE)
def test_large_mixed_matches_reference(name, v_mode):
    g = golden(name)
    e_ref = float(g["energies"][-1])
    with system_for(g, load_v_pppp=v_mode == "stored") as s, \
            CCDSolver(s, precision="mixed_bf16", v_mode=v_mode) as sol:
        n = s.n_particles
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        t2 = sol.t2()
    de_n = abs(res.e_corr - e_ref) / n
    t2_err = float(np.max(np.abs(t2_sample(g, t2) - g["t2"])))
    print(f"{name} {v_mode}: |dE/N| = {de_n:.3e}, T2 max-abs = {t2_err:.3e}, "
          f"iterations {res.iterations} (polish {res.polish_iterations}) vs {len(g['energies'])}")
    assert res.converged and res.polish_iterations >= 1
    assert de_n <= 1e-7 * abs(e_ref / n)
    assert t2_err <= 1e-7


@pytest.mark.parametrize("name", ["eg54c36_r2", "pnm66_s32"])
def test_large_headline_stop_rule_within_1e7_per_particle(name):
    """The bench's stop rule |dE| <= 1e-8 N lands within 1e-7 per particle of the reference's
    converged energy, for both precisions, with V_pppp generated on the device."""
    g = golden(name)
    e_ref = float(g["energies"][-1])
    with system_for(g, load_v_pppp=False) as s:
        n = s.n_particles
        for prec in ["mixed_bf16", "fp64"]:
            with CCDSolver(s, precision=prec, v_mode="on_the_fly") as sol:
                res = sol.solve(tol=1e-8 * n, max_iters=100, mixing=0.5)
                t2 = sol.t2()
            assert res.converged
            assert abs(res.e_corr - e_ref) / n <= 1e-7
            assert float(np.max(np.abs(t2_sample(g, t2) - g["t2"]))) <= 1e-5
