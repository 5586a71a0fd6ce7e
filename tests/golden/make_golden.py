"""Regenerates the golden fixtures in this directory from the reference itself.

Runs oracle/_ref/ref_harness (the unmodified reference sources compiled by oracle/ref/Makefile,
see oracle/build.py) for each configuration and stores, per configuration, an .npz with:
  energies      corrCCD after every iteration (stored-V loop of main.cpp:589-670)
  scalars       E_ref, E_MBPT2, final corrCCD, tolerance
  t2            converged t2_pphh data (full for small systems, every 97th element otherwise)
  t2_sumsq      sum of squares of the full converged t2
  map_hashes    FNV-1a of the 8 loadMaps tables (u64 channel,row,column triples, pphh order)
  struct_hashes FNV-1a of chan_dims, chan_mod_dims (hp, ph), three_body_dims, pp/hh/ph/hp maps,
                hpp/phh maps, sp_energy
  v_hashes      FNV-1a of the V chains over amplitude-carrying channels
Usage: python tests/golden/make_golden.py [name ...]   (needs the reference build)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.refdump import read_dump  # noqa: E402
from oracle.oracle import fnv1a  # noqa: E402

# name -> (reference CLI, builder kind, builder params, full t2?)
CONFIGS = {
    "pairing_gm1.0": (["--pairing", "-l", "8", "-n", "8", "-x", "1.0", "-g", "-1.0", "-t", "1e-12"],
                      "pairing", dict(xi=1.0, g=-1.0, n_pair_states=8, n_particles=8), True),
    "pairing_gm0.5": (["--pairing", "-l", "8", "-n", "8", "-x", "1.0", "-g", "-0.5", "-t", "1e-12"],
                      "pairing", dict(xi=1.0, g=-0.5, n_pair_states=8, n_particles=8), True),
    "pairing_gp0.5": (["--pairing", "-l", "8", "-n", "8", "-x", "1.0", "-g", "0.5", "-t", "1e-12"],
                      "pairing", dict(xi=1.0, g=0.5, n_pair_states=8, n_particles=8), True),
    "pairing_gp1.0": (["--pairing", "-l", "8", "-n", "8", "-x", "1.0", "-g", "1.0", "-t", "1e-12"],
                      "pairing", dict(xi=1.0, g=1.0, n_pair_states=8, n_particles=8), True),
    "pnm14_s4": (["--infMatter", "-d", "0.08", "-z", "1", "-s", "4", "-p", "2", "-t", "1e-8"],
                 "inf_matter", dict(density=0.08, tz_max=1, n_shells=4, n_particle_shells=2), True),
    # Symmetric nuclear matter (both isospins): one particle shell, which converges (with two
    # the reference's iteration runs to its cap or to NaN at these densities).
    "snm4_s4": (["--infMatter", "-d", "0.16", "-z", "2", "-s", "4", "-p", "1", "-t", "1e-8"],
                "inf_matter", dict(density=0.16, tz_max=2, n_shells=4, n_particle_shells=1), True),
    "eg14_s19": (["--electronGas", "-r", "1.0", "-s", "19", "-p", "2", "-t", "1e-12"],
                 "electron_gas", dict(r_s=1.0, n_shells=19, n_particle_shells=2), True),
    "eg54_s19": (["--electronGas", "-r", "1.0", "-s", "19", "-p", "4", "-t", "1e-12"],
                 "electron_gas", dict(r_s=1.0, n_shells=19, n_particle_shells=4), False),
    # More pins of the builder and the oracle (CPU tests).
    "eg14_r05": (["--electronGas", "-r", "0.5", "-s", "19", "-p", "2", "-t", "1e-12"],
                 "electron_gas", dict(r_s=0.5, n_shells=19, n_particle_shells=2), True),
    "eg14_r2": (["--electronGas", "-r", "2.0", "-s", "19", "-p", "2", "-t", "1e-12"],
                "electron_gas", dict(r_s=2.0, n_shells=19, n_particle_shells=2), True),
    "pnm14_d016": (["--infMatter", "-d", "0.16", "-z", "1", "-s", "4", "-p", "2", "-t", "1e-10"],
                   "inf_matter", dict(density=0.16, tz_max=1, n_shells=4, n_particle_shells=2),
                   True),
    "pairing_l6n4": (["--pairing", "-l", "6", "-n", "4", "-x", "1.0", "-g", "0.3", "-t", "1e-12"],
                     "pairing", dict(xi=1.0, g=0.3, n_pair_states=6, n_particles=4), True),
    "eg38_s16": (["--electronGas", "-r", "1.0", "-s", "16", "-p", "3", "-t", "1e-10"],
                 "electron_gas", dict(r_s=1.0, n_shells=16, n_particle_shells=3), False),
    # The large workloads: 1850 spin-orbitals (|n|^2 <= 36), hh up to 54 / 66.
    "eg54c36_r2": (["--electronGas", "-r", "2.0", "-s", "32", "-p", "4", "-t", "1e-12"],
                   "electron_gas", dict(r_s=2.0, n_shells=32, n_particle_shells=4), False),
    "eg54c36_r05": (["--electronGas", "-r", "0.5", "-s", "32", "-p", "4", "-t", "1e-12"],
                    "electron_gas", dict(r_s=0.5, n_shells=32, n_particle_shells=4), False),
    "pnm66_s32": (["--infMatter", "-d", "0.08", "-z", "1", "-s", "32", "-p", "5", "-t", "1e-12"],
                  "inf_matter", dict(density=0.08, tz_max=1, n_shells=32, n_particle_shells=5),
                  False),
}

STRUCT = ["chan_dims", "chan_mod_dims", "three_body_dims", "pp_map", "hh_map", "ph_mod_map",
          "hp_mod_map", "hpp_map", "phh_map", "sp_energy"]
MAPS = ["map_iab_j", "map_jab_i", "map_a_bij", "map_b_aij", "map_ai_jb", "map_aj_ib",
        "map_bi_ja", "map_bj_ia"]


def struct_view(name, arr):
    # The builder only fills the hp/ph columns of modified channel dims meaningfully for the
    # solver; the reference also counts pp/hh pairs there, which the tests compare as well.
    return np.ascontiguousarray(arr)


def generate(name):
    cli, kind, params, full = CONFIGS[name]
    harness = os.path.join(REPO, "oracle", "_ref", "ref_harness")
    with tempfile.TemporaryDirectory() as td:
        dump = os.path.join(td, "dump.bin")
        env = dict(os.environ, CCD_DUMP=dump, OPENBLAS_NUM_THREADS="1",
                   # The reference's pairing basis builds its 3-body maps correctly only
                   # single-threaded (SPBasis.cpp:227-255 runs outside any omp-for).
                   OMP_NUM_THREADS="1" if kind == "pairing" else str(os.cpu_count()))
        subprocess.run([harness, *cli], check=True, env=env, stdout=subprocess.DEVNULL)
        d = read_dump(dump)
    t2 = d["t2"]
    out = dict(
        energies=d["energies"], scalars=d["scalars"], header=d["header"],
        t2=t2 if full else t2[::97].copy(), t2_full=np.array([1 if full else 0]),
        t2_sumsq=np.array([float(np.dot(t2, t2))]),
        map_hashes=np.array([fnv1a(d[m]) for m in MAPS], dtype=np.uint64),
        struct_hashes=np.array([fnv1a(struct_view(s, d[s])) for s in STRUCT], dtype=np.uint64),
        v_hashes=d["v_hashes"],
        kind=np.array(kind), params=np.array(repr(params)), cli=np.array(" ".join(cli)),
    )
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


if __name__ == "__main__":
    names = sys.argv[1:] or list(CONFIGS)
    for n in names:
        o = generate(n)
        print(n, "iterations", len(o["energies"]), "E", repr(float(o["scalars"][2])))
