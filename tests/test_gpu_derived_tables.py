"""Remap tables derived on the device.

A problem built without the eight loadMaps tables (load.cpp:389-532; ccdgpu_problem.maps all
NULL) makes ccdgpu_create derive them from the channel maps, as loadMaps does.  The flat
tables must equal the converted host tables entry for entry, so every solve through them is
bit-identical to the solve through the host's tables: same iteration count, same energy
history, same amplitudes.
"""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, System
from helpers import SMALL, golden, system_for

pytestmark = pytest.mark.gpu


def _no_tables(g, load_v_pppp=True):
    return getattr(System, g["kind"])(**g["params"], load_v_pppp=load_v_pppp, tables=False)


def _same_solve(a, b, g):
    ra = a.solve(tol=g["tol"], max_iters=100, mixing=0.5)
    rb = b.solve(tol=g["tol"], max_iters=100, mixing=0.5)
    assert ra.iterations == rb.iterations
    np.testing.assert_array_equal(a.energy_history(), b.energy_history())
    np.testing.assert_array_equal(a.t2(), b.t2())
    return ra


@pytest.mark.parametrize("path", ["fused", "tables"])
@pytest.mark.parametrize("name", SMALL + ["eg54_s19"])
def test_derived_tables_solve_bit_identical(name, path):
    g = golden(name)
    with system_for(g) as s1, _no_tables(g) as s2, \
            CCDSolver(s1, path=path) as a, CCDSolver(s2, path=path) as b:
        r = _same_solve(a, b, g)
        assert abs(r.e_corr - g["energies"][-1]) <= 1e-10 * abs(g["energies"][-1]) + 1e-14


def test_derived_tables_mixed_precision_on_the_fly_v():
    """Nothing but the channel maps, dimensions, energies and model from the host: V_pppp is
    generated and the tables derived on the device."""
    g = golden("eg14_s19")
    with system_for(g, load_v_pppp=False) as s1, _no_tables(g, load_v_pppp=False) as s2, \
            CCDSolver(s1, precision="mixed_bf16", v_mode="on_the_fly") as a, \
            CCDSolver(s2, precision="mixed_bf16", v_mode="on_the_fly") as b:
        _same_solve(a, b, g)


@pytest.mark.parametrize("precision", ["fp64", "mixed_bf16"])
@pytest.mark.parametrize("name", SMALL + ["eg54_s19"])
def test_nothing_but_structure_from_the_host(name, precision):
    """No V block and no remap table from the host: ccdgpu_create generates every V block from
    the model (load.cpp:112-318 elements) and derives the tables.  Pairing and electron-gas
    elements are bit-identical to the host's, so the solve is too; the Minnesota elements use
    CUDA's exp/pow and may differ by an ulp, so the PNM solve is held to the reference energy."""
    g = golden(name)
    with system_for(g) as s1, \
            getattr(System, g["kind"])(**g["params"], tables=False, v_blocks=False) as s2, \
            CCDSolver(s1, precision=precision) as a, \
            CCDSolver(s2, precision=precision, v_mode="on_the_fly") as b:
        if g["kind"] == "inf_matter":
            rb = b.solve(tol=g["tol"], max_iters=100, mixing=0.5)
            ref = g["energies"][-1]
            rtol = 1e-10 if precision == "fp64" else 1e-6
            assert abs(rb.e_corr - ref) <= rtol * abs(ref) + 1e-14
        else:
            _same_solve(a, b, g)
        assert b.mbpt2() == pytest.approx(float(g["scalars"][1]), rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("name", SMALL + ["eg54_s19"])
def test_table_path_on_generated_v(name):
    """The table path (the reference's stage structure) with every V block, the three-body V
    included, generated on the device and the tables derived there."""
    g = golden(name)
    with system_for(g) as s1, \
            getattr(System, g["kind"])(**g["params"], tables=False, v_blocks=False) as s2, \
            CCDSolver(s1, path="tables") as a, \
            CCDSolver(s2, path="tables", v_mode="on_the_fly") as b:
        if g["kind"] == "inf_matter":
            rb = b.solve(tol=g["tol"], max_iters=100, mixing=0.5)
            ref = g["energies"][-1]
            assert abs(rb.e_corr - ref) <= 1e-10 * abs(ref) + 1e-14
        else:
            _same_solve(a, b, g)
