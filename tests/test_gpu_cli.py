"""The command-line front end on the GPU: the reference's output lines and energies, a batch
file solved together, and a checkpoint / restart of T2."""
import io

import pytest

from coupled_cluster_doubles_b200 import cli
from helpers import golden

pytestmark = pytest.mark.gpu


def _values(text):
    out = {}
    for line in text.splitlines():
        if ":" in line and not line.startswith("system"):
            k, v = line.split(":", 1)
            out.setdefault(k.strip(), []).append(float(v))
    return out


@pytest.mark.parametrize("name", ["eg14_s19", "pnm14_s4", "pairing_gp0.5"])
def test_cli_reproduces_reference_energy(name):
    g = golden(name)
    buf = io.StringIO()
    assert cli.main(str(g["cli"]).split() + ["-v", "1"], out=buf) == 0
    v = _values(buf.getvalue())
    ref = float(g["energies"][-1])
    assert abs(v["CCDCorr"][0] - ref) <= 1e-10 * abs(ref)
    assert abs(v["Reference Energy"][0] - float(g["scalars"][0])) <= 1e-12 * abs(g["scalars"][0])
    assert abs(v["MBPT2Corr"][0] - float(g["scalars"][1])) <= 1e-12 * abs(g["scalars"][1])
    assert abs(v["iterations"][0] - len(g["energies"])) <= 1


@pytest.mark.parametrize("name", ["eg14_s19", "pairing_gp0.5"])
def test_cli_save_memory_mode(name):
    """-m 1 (saveMemory): no V block from the host, every one generated on the device."""
    g = golden(name)
    buf = io.StringIO()
    assert cli.main(str(g["cli"]).split() + ["-m", "1", "-v", "1"], out=buf) == 0
    v = _values(buf.getvalue())
    ref = float(g["energies"][-1])
    assert abs(v["CCDCorr"][0] - ref) <= 1e-10 * abs(ref)
    assert abs(v["MBPT2Corr"][0] - float(g["scalars"][1])) <= 1e-12 * abs(g["scalars"][1])


def test_cli_batch_and_restart(tmp_path):
    eg, pnm = golden("eg14_s19"), golden("pnm14_s4")
    bf = tmp_path / "sweep.txt"
    bf.write_text(f"{str(eg['cli'])}\n{str(pnm['cli'])}\n")
    buf = io.StringIO()
    assert cli.main(["--batch", str(bf)], out=buf) == 0
    v = _values(buf.getvalue())
    # The batch runs at the strictest tolerance (1e-12); the PNM golden stopped at 1e-8.
    assert abs(v["CCDCorr"][0] - float(eg["energies"][-1])) <= 1e-10 * abs(eg["energies"][-1])
    assert abs(v["CCDCorr"][1] - float(pnm["energies"][-1])) <= 1e-7
    # A loose solve checkpointed, then resumed to the golden tolerance.
    ck = tmp_path / "t2.npy"
    first = io.StringIO()
    cli.main(str(eg["cli"]).split()[:-2] + ["-t", "1e-4", "--checkpoint", str(ck)], out=first)
    resumed = io.StringIO()
    cli.main(str(eg["cli"]).split() + ["--restart", str(ck)], out=resumed)
    v1, v2 = _values(first.getvalue()), _values(resumed.getvalue())
    ref = float(eg["energies"][-1])
    assert abs(v2["CCDCorr"][0] - ref) <= 1e-10 * abs(ref)
    # Resuming continues the same fixed-point iteration: about the iterations that were left.
    assert v2["iterations"][0] <= len(eg["energies"]) - v1["iterations"][0] + 3
