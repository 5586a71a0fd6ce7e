"""Mixed precision: the split-bf16 tensor-core pp ladder (tcgen05) and the FP64 polish.

Tolerances.  One ladder evaluation with 2-term bf16 operands (about 17 significant bits each,
FP32 accumulation) agrees with the FP64 ladder to 2e-4 of the largest |D| of the chain; with
3-term operands to 2e-6.  A mixed solve ends with FP64 iterations, so its converged energy
per particle agrees with the reference's to 1e-7 relative (the accuracy bound of the mixed
mode) and its T2 with the reference's to 1e-7 max-abs; both are usually far closer.
"""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, solver as solver_mod
from helpers import golden, system_for, t2_sample

pytestmark = pytest.mark.gpu

LADDER_RTOL = {"mixed_bf16": 2e-4, "mixed_bf16x3": 2e-6}
# Channels with long K (EG N=54: up to ~360 packed pairs c < d per row): the FP32 accumulator,
# not the operand split, sets the 3-term error, about sqrt(K) * 2^-24 of max|D|.
LADDER_RTOL_LONG_K = {"mixed_bf16": 2e-4, "mixed_bf16x3": 1e-5}
E_PER_N_RTOL = 1e-7
T2_ATOL = 1e-7


def _ladder_after_one_step(s, precision, t2):
    with CCDSolver(s, precision=precision) as sol:
        sol.set_t2(t2)
        sol.step(0.5)
        return sol.chain(solver_mod.CHAIN_DIFF_PPHH)


@pytest.mark.parametrize("precision", ["mixed_bf16", "mixed_bf16x3"])
@pytest.mark.parametrize("name", ["eg14_s19", "pnm14_s4", "pairing_gm0.5"])
def test_tensor_core_ladder_matches_fp64(name, precision):
    g = golden(name)
    with system_for(g) as s:
        # A converged-like amplitude set: a few FP64 iterations from zero.
        with CCDSolver(s) as ref:
            for _ in range(3):
                ref.step(0.5)
            t2 = ref.t2()
        d64 = _ladder_after_one_step(s, "fp64", t2)
        dmx = _ladder_after_one_step(s, precision, t2)
    scale = float(np.max(np.abs(d64)))
    err = float(np.max(np.abs(dmx - d64)))
    print(f"{name} {precision}: max|dD| = {err:.3e}, max|D| = {scale:.3e}, rel {err / scale:.3e}")
    assert scale > 0
    assert err <= LADDER_RTOL[precision] * scale


@pytest.mark.parametrize("precision", ["mixed_bf16", "mixed_bf16x3"])
@pytest.mark.parametrize("name", ["eg14_s19", "eg54_s19"])
def test_generated_v_ladder_matches_fp64(name, precision):
    """Electron gas with V regenerated inside the ladder (v_mode "in_ladder"): the tensor-core
    ladder builds its V operand planes itself (momentum/spin codes and a q^2 table, exact to the
    precision of the split) instead of reading bf16 images; checked against the FP64 ladder."""
    g = golden(name)
    with system_for(g) as s, system_for(g, load_v_pppp=False) as s_gen:
        with CCDSolver(s) as ref:
            for _ in range(3):
                ref.step(0.5)
            t2 = ref.t2()
        d64 = _ladder_after_one_step(s, "fp64", t2)
        with CCDSolver(s_gen, precision=precision, v_mode="in_ladder") as sol:
            sol.set_t2(t2)
            sol.step(0.5)
            dmx = sol.chain(solver_mod.CHAIN_DIFF_PPHH)
    scale = float(np.max(np.abs(d64)))
    err = float(np.max(np.abs(dmx - d64)))
    print(f"{name} {precision} generated V: max|dD| = {err:.3e}, rel {err / scale:.3e}")
    assert scale > 0
    assert err <= LADDER_RTOL_LONG_K[precision] * scale


@pytest.mark.parametrize("precision", ["mixed_bf16", "mixed_bf16x3"])
@pytest.mark.parametrize("name", ["eg14_s19", "eg54_s19", "pnm14_s4", "pairing_gm1.0"])
def test_mixed_solve_matches_reference(name, precision):
    g = golden(name)
    e_ref = float(g["energies"][-1])
    with system_for(g) as s, CCDSolver(s, precision=precision) as sol:
        n = s.n_particles
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        t2 = sol.t2()
    de_n = abs(res.e_corr - e_ref) / n
    t2_err = float(np.max(np.abs(t2_sample(g, t2) - g["t2"])))
    print(f"{name} {precision}: |dE/N| = {de_n:.3e}, T2 max-abs = {t2_err:.3e}, "
          f"iterations {res.iterations} (polish {res.polish_iterations}) vs {len(g['energies'])}")
    assert res.converged
    assert res.polish_iterations >= 1
    assert de_n <= E_PER_N_RTOL * abs(e_ref / n)
    assert t2_err <= T2_ATOL


def test_mixed_stops_within_1e7_per_particle():
    """The headline stop rule |dE| <= 1e-8 N lands within 1e-7 per particle of the fully
    converged FP64 energy, with the mixed solver as with the FP64 one."""
    g = golden("eg54_s19")
    e_ref = float(g["energies"][-1])
    with system_for(g) as s:
        n = s.n_particles
        for prec in ["mixed_bf16", "fp64"]:
            with CCDSolver(s, precision=prec) as sol:
                res = sol.solve(tol=1e-8 * n, max_iters=100, mixing=0.5)
            assert res.converged
            assert abs(res.e_corr - e_ref) / n <= 1e-7


def test_batch_solve_matches_individual_solves():
    """ccdgpu_solve_batch: several systems (different N, r_s, cutoff, precision) in flight at
    once give exactly the results of separate solves."""
    from coupled_cluster_doubles_b200 import System, solve_batch
    specs = [dict(r_s=1.0, n_shells=19, n_particle_shells=2), dict(r_s=2.0, n_shells=15, n_particle_shells=3),
             dict(r_s=0.5, n_shells=19, n_particle_shells=4)]
    systems = [System.electron_gas(**p, load_v_pppp=False) for p in specs]
    try:
        precs = ["mixed_bf16", "fp64", "mixed_bf16"]
        solos = []
        for s, pr in zip(systems, precs):
            with CCDSolver(s, v_mode="on_the_fly", precision=pr) as sol:
                solos.append((sol.solve(tol=1e-10), sol.t2()))
        sols = [CCDSolver(s, v_mode="on_the_fly", precision=pr) for s, pr in zip(systems, precs)]
        try:
            res = solve_batch(sols, tol=1e-10)
            for (r0, t0), r, sol in zip(solos, res, sols):
                assert r.iterations == r0.iterations and r.e_corr == r0.e_corr
                np.testing.assert_array_equal(sol.t2(), t0)
        finally:
            for sol in sols:
                sol.close()
    finally:
        for s in systems:
            s.close()
