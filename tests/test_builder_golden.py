"""The host problem builder reproduces the reference's inputs bit for bit.

Compares, per golden configuration, the builder's orbital energies, channel dimensions,
channel / three-body maps, the 8 loadMaps remap tables (load.cpp:389-532) and every V chain
(load.cpp:112-318) with FNV-1a hashes of the reference's own dumps, and E_ref / E_MBPT2 for
exact equality.
"""
import pytest

from helpers import EXTRA, MAPS, SMALL, STRUCT, VKINDS, golden, system_for
from oracle.oracle import fnv1a


@pytest.mark.parametrize("name", SMALL + ["eg54_s19"] + EXTRA)
def test_builder_matches_reference(name):
    g = golden(name)
    with system_for(g) as s:
        assert s.n_sp == int(g["header"][0])
        assert s.n_particles == int(g["header"][1])
        assert s.n_channels == int(g["header"][2])
        assert s.reference_energy == float(g["scalars"][0])
        assert s.mbpt2 == float(g["scalars"][1])
        for k, n in enumerate(STRUCT):
            assert fnv1a(s.array(n)) == int(g["struct_hashes"][k]), n
        for k, n in enumerate(MAPS):
            assert fnv1a(s.array(n)) == int(g["map_hashes"][k]), n
        for k, n in enumerate(VKINDS):
            assert fnv1a(s.array(n)) == int(g["v_hashes"][k]), n


def test_builder_without_v_pppp_keeps_everything_else():
    g = golden("eg14_s19")
    with system_for(g, load_v_pppp=False) as s:
        assert s.array("v_pppp").size == 0
        assert not s.problem.contents.v_pppp
        for k, n in enumerate(MAPS):
            assert fnv1a(s.array(n)) == int(g["map_hashes"][k]), n


@pytest.mark.parametrize("name", ["pairing_gp0.5", "pnm14_s4", "eg14_s19"])
def test_builder_without_tables_keeps_everything_else(name):
    """CCDHOST_NO_TABLES: no remap tables and NULL ccdgpu_problem.maps (the solver derives
    them on the device); every other input stays bit-identical to the reference's."""
    from coupled_cluster_doubles_b200 import System
    g = golden(name)
    with getattr(System, g["kind"])(**g["params"], tables=False) as s:
        p = s.problem.contents
        assert all(not p.maps[k] for k in range(8))
        assert s.reference_energy == float(g["scalars"][0])
        for n in MAPS:
            assert s.array(n).size == 0, n
        for k, n in enumerate(STRUCT):
            assert fnv1a(s.array(n)) == int(g["struct_hashes"][k]), n
        for k, n in enumerate(VKINDS):
            assert fnv1a(s.array(n)) == int(g["v_hashes"][k]), n


@pytest.mark.parametrize("name", ["pairing_gp0.5", "pnm14_s4", "eg14_s19"])
def test_builder_without_v_blocks(name):
    """CCDHOST_NO_V: every ccdgpu_problem.v_* is NULL (the solver generates the blocks on the
    device); E_ref, E_MBPT2 (evaluated element by element) and the structure stay bit-identical
    to the reference's."""
    from coupled_cluster_doubles_b200 import System
    g = golden(name)
    with getattr(System, g["kind"])(**g["params"], tables=False, v_blocks=False) as s:
        p = s.problem.contents
        assert not any([p.v_hhhh, p.v_hhpp, p.v_pppp, p.v_hpph_mod, p.v_hphp_mod, p.v_h_hpp,
                        p.v_phh_p])
        assert s.reference_energy == float(g["scalars"][0])
        assert s.mbpt2 == float(g["scalars"][1])
        for n in VKINDS:
            assert s.array(n).size == 0, n
        for k, n in enumerate(STRUCT):
            assert fnv1a(s.array(n)) == int(g["struct_hashes"][k]), n


@pytest.mark.parametrize("args", [dict(xi=1.0, g=0.5, n_pair_states=4, n_particles=8),
                                  dict(xi=1.0, g=0.5, n_pair_states=0, n_particles=0)])
def test_builder_rejects_bad_pairing_input(args):
    from coupled_cluster_doubles_b200 import System
    from coupled_cluster_doubles_b200.system import BuildError
    with pytest.raises(BuildError):
        System.pairing(**args)


def test_builder_rejects_bad_plane_wave_input():
    from coupled_cluster_doubles_b200 import System
    from coupled_cluster_doubles_b200.system import BuildError
    with pytest.raises(BuildError):
        System.electron_gas(r_s=1.0, n_shells=2, n_particle_shells=4)
    with pytest.raises(BuildError):
        System.inf_matter(density=0.08, tz_max=3, n_shells=4, n_particle_shells=2)


def test_device_channels_without_a_gpu_is_an_error():
    """CCDHOST_DEVICE_CHANNELS has no host fallback: without a GPU the build fails with
    CCDGPU_ERR_NO_DEVICE (-6)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from coupled_cluster_doubles_b200 import System
    from coupled_cluster_doubles_b200.system import BuildError
    with pytest.raises(BuildError, match="status -6"):
        System.pairing(xi=1.0, g=0.5, n_pair_states=4, n_particles=4, device_channels=True)
