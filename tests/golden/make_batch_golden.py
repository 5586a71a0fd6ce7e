"""Regenerates tests/golden/batch24.npz: the reference's own outcome for each member of the
batched electron-gas sweep that bench.py --config batch24 solves (bench.batch_specs: N in
{14, 38, 54} x r_s in {0.5, 1, 2, 3, 4, 5, 6, 8}, cutoffs drawn from a fixed seed), at the
sweep's one stop threshold |dE| <= 1.4e-7 (1e-8 N for the smallest N).

Runs oracle/_ref/ref_harness (the unmodified reference sources, see oracle/build.py) per
member and stores, per member: r_s, n_shells, n_particle_shells, N, the iterations the
reference loop ran (main.cpp:508-519: at most 101), its final corrCCD, and the outcome:
  converged  |dE| <= tol before the cap
  capped     101 iterations, energy still finite
  diverged   the energy became non-finite (the reference loop then runs on to its cap)
Usage: python tests/golden/make_batch_golden.py   (needs the reference build)
"""
import math
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from bench import batch_specs  # noqa: E402
from oracle.refdump import read_dump  # noqa: E402

TOL = 1.4e-7
N_OF_P = {2: 14, 3: 38, 4: 54}


def outcome(energies):
    e = float(energies[-1])
    if not math.isfinite(e):
        return "diverged"
    if len(energies) >= 101 and abs(float(energies[-1]) - float(energies[-2])) > TOL:
        return "capped"
    return "converged"


def run(spec):
    cli = ["--electronGas", "-r", repr(float(spec["r_s"])), "-s", str(spec["n_shells"]),
           "-p", str(spec["n_particle_shells"]), "-t", repr(TOL)]
    harness = os.path.join(REPO, "oracle", "_ref", "ref_harness")
    with tempfile.TemporaryDirectory() as td:
        dump = os.path.join(td, "dump.bin")
        env = dict(os.environ, CCD_DUMP=dump, OPENBLAS_NUM_THREADS="1",
                   OMP_NUM_THREADS=str(os.cpu_count()))
        subprocess.run([harness, *cli], check=True, env=env, stdout=subprocess.DEVNULL)
        return read_dump(dump)["energies"]


if __name__ == "__main__":
    rows = []
    for spec in batch_specs():
        en = run(spec)
        st = outcome(en)
        rows.append((spec, len(en), float(en[-1]), st))
        print(spec, "N", N_OF_P[spec["n_particle_shells"]], "iterations", len(en), "E",
              float(en[-1]), st, flush=True)
    np.savez_compressed(
        os.path.join(HERE, "batch24.npz"),
        r_s=np.array([r[0]["r_s"] for r in rows]),
        n_shells=np.array([r[0]["n_shells"] for r in rows]),
        n_particle_shells=np.array([r[0]["n_particle_shells"] for r in rows]),
        n=np.array([N_OF_P[r[0]["n_particle_shells"]] for r in rows]),
        iterations=np.array([r[1] for r in rows]),
        e_final=np.array([r[2] for r in rows]),
        status=np.array([r[3] for r in rows]),
        tol=np.array([TOL]))
