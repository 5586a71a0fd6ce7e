"""V_pppp generated on the device from the model (CCDGPU_V_ON_THE_FLY, the counterpart of the
reference's saveMemory mode, calc.cpp:233-504 / load.cpp:112-318).

The host builds no V_pppp (System(..., load_v_pppp=False)).  Electron-gas and pairing elements
are generated with the reference's own expressions and are bit-identical to the stored ones,
so results agree with the stored-V solve to the same FP64 tolerance as the reference goldens
(1e-10 relative in E, 1e-9 in T2).  Neutron-matter elements use CUDA's exp and may differ by an
ulp; the same tolerances hold.
"""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver
from helpers import golden, system_for, t2_sample

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["eg14_s19", "eg54_s19", "pnm14_s4", "pairing_gm1.0", "pairing_gp0.5"])
def test_on_the_fly_matches_reference(name):
    g = golden(name)
    e_ref = float(g["energies"][-1])
    with system_for(g, load_v_pppp=False) as s, CCDSolver(s, v_mode="on_the_fly") as sol:
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
        t2 = sol.t2()
    assert abs(res.iterations - len(g["energies"])) <= 1
    assert abs(res.e_corr - e_ref) <= 1e-10 * abs(e_ref) + 1e-14
    assert np.max(np.abs(t2_sample(g, t2) - g["t2"])) < 1e-9


@pytest.mark.parametrize("name", ["eg14_s19", "pairing_gm0.5"])
def test_on_the_fly_ladder_equals_stored(name):
    """Bit-identical V elements give the same ladder intermediate as uploaded V."""
    g = golden(name)
    with system_for(g) as s_stored, system_for(g, load_v_pppp=False) as s_gen:
        with CCDSolver(s_stored) as a, CCDSolver(s_gen, v_mode="on_the_fly") as b:
            for _ in range(3):
                ea, eb = a.step(0.5), b.step(0.5)
                assert ea == eb
            np.testing.assert_array_equal(a.t2(), b.t2())


@pytest.mark.parametrize("name", ["eg14_s19", "eg54_s19"])
def test_on_the_fly_tc_images_equal_stored(name):
    """The tensor-core ladder's bf16 V images generated on the device equal the ones tiled from
    uploaded V (the same doubles, split the same way): three mixed iterations agree bit for bit."""
    g = golden(name)
    with system_for(g) as s_stored, system_for(g, load_v_pppp=False) as s_gen:
        with CCDSolver(s_stored, precision="mixed_bf16") as a, \
                CCDSolver(s_gen, v_mode="on_the_fly", precision="mixed_bf16") as b:
            for _ in range(3):
                ea, eb = a.step(0.5), b.step(0.5)
                assert ea == eb
            np.testing.assert_array_equal(a.t2(), b.t2())


@pytest.mark.parametrize("name", ["eg14_s19", "eg54_s19", "pairing_gm1.0"])
def test_on_the_fly_mixed_solve_equals_stored(name):
    """A mixed handle with generated V writes its FP64 tiles and its bf16 images from one
    evaluation of each element; a whole mixed solve, FP64 polish included, equals the solve
    with uploaded V bit for bit."""
    g = golden(name)
    with system_for(g) as s_stored, system_for(g, load_v_pppp=False) as s_gen:
        with CCDSolver(s_stored, precision="mixed_bf16") as a, \
                CCDSolver(s_gen, v_mode="on_the_fly", precision="mixed_bf16") as b:
            ra = a.solve(tol=g["tol"], max_iters=100, mixing=0.5)
            rb = b.solve(tol=g["tol"], max_iters=100, mixing=0.5)
            assert (ra.iterations, ra.polish_iterations) == (rb.iterations, rb.polish_iterations)
            if name.startswith("eg"):
                assert ra.polish_iterations >= 1
            assert ra.e_corr == rb.e_corr
            np.testing.assert_array_equal(a.t2(), b.t2())


def test_on_the_fly_mixed_precision():
    g = golden("eg54_s19")
    e_ref = float(g["energies"][-1])
    with system_for(g, load_v_pppp=False) as s, \
            CCDSolver(s, v_mode="on_the_fly", precision="mixed_bf16") as sol:
        res = sol.solve(tol=g["tol"], max_iters=100, mixing=0.5)
    assert res.converged and res.polish_iterations >= 1
    assert abs(res.e_corr - e_ref) / s.n_particles <= 1e-7 * abs(e_ref / s.n_particles)


def test_on_the_fly_requires_model():
    g = golden("eg14_s19")
    with system_for(g, load_v_pppp=False) as s:
        with pytest.raises(Exception):
            CCDSolver(s)  # stored mode without V_pppp
