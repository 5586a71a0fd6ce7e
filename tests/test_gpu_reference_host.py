"""The boundary against the reference itself: the reference's own host objects drive the library.

oracle/_ref/gpu_host links the unmodified reference objects (built from its sources by
oracle/ref/Makefile) and runs main.cpp's set-up for one rank (argp options, SPBasis, channel
construction in ffdBalance order, loadVnn_*, loadMaps); it then hands the reference's own
arrays (chanDims, chanMaps, threeBodyChanDims, Chain<T>::get blocks, ChainIndex maps) to
ccdgpu_create exactly as INTEGRATION.md's patch does, solves with ccdgpu_solve, copies T2 back
into t2_pphh and prints main.cpp's result lines.  The energies must match the reference's
goldens to 1e-10 relative (FP64), the iteration count to one, and the checksum of the T2 the
host received the golden's sum of squares.
"""
import os
import re
import subprocess

import pytest

from helpers import golden

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(REPO, "oracle", "_ref", "gpu_host")


def _run(cli, env_extra=None):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/gpu_host not built (needs the reference sources)")
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", **(env_extra or {}))
    out = subprocess.run([EXE, *cli.split()], env=env, capture_output=True, text=True,
                         timeout=600, check=True).stdout
    val = {k: float(v) for k, v in re.findall(r"^([A-Za-z0-9_/]+): ([-0-9.eE+]+)", out, re.M)}
    return val


@pytest.mark.parametrize("name", ["eg14_s19", "pnm14_s4", "pairing_gm1.0"])
def test_reference_host_through_c_abi_matches_reference(name):
    g = golden(name)
    val = _run(str(g["cli"]))
    e_ref = float(g["energies"][-1])
    assert abs(val["iterations"] - len(g["energies"])) <= 1
    assert abs(val["CCDCorr"] - e_ref) <= 1e-10 * abs(e_ref)
    assert abs(val["t2_sumsq"] - float(g["t2_sumsq"][0])) <= 1e-8 * float(g["t2_sumsq"][0])


def test_reference_host_readme_known_answer():
    # src/README.md:8-10: E_CCD/A = 10.155078 for neutron matter at 0.08 fm^-3, 14 neutrons.
    val = _run("--infMatter -d 0.08 -z 1 -s 4 -p 2 -t 1e-8")
    assert round(val["E_CCD/A"], 6) == 10.155078


def test_reference_host_mixed_precision():
    g = golden("eg14_s19")
    val = _run(str(g["cli"]), {"CCD_GPU_PRECISION": "mixed_bf16"})
    e_ref = float(g["energies"][-1])
    assert abs(val["CCDCorr"] - e_ref) / 14 <= 1e-7 * abs(e_ref / 14)
