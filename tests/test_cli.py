"""The command-line front end: the reference's options, defaults and config-file rule
(parse.cpp:128-229, main.cpp:34-39), checked without a GPU."""
from coupled_cluster_doubles_b200 import cli


def test_defaults_are_the_references():
    o = cli.parse_args([])
    assert o["basis"] == "inf_matter"
    assert (o["density"], o["g"], o["r_s"], o["xi"], o["tolerance"]) == (0.08, 0.5, 0.5, 1.0, 1e-8)
    assert (o["nParticleShells"], o["nParticles"], o["nPairStates"], o["nShells"], o["tzMax"]) == \
        (2, 4, 4, 4, 1)
    assert o["saveMemory"] == 0 and o["verbose"] == 0 and o["precision"] == "fp64"


def test_short_and_long_options():
    o = cli.parse_args("--electronGas -r 1.0 -s 19 -p 2 -t 1e-12".split())
    assert o["basis"] == "electron_gas" and o["r_s"] == 1.0 and o["nShells"] == 19
    assert o["nParticleShells"] == 2 and o["tolerance"] == 1e-12
    o = cli.parse_args("--pairing --nPairStates 8 --nParticles 8 --xi 1.0 --g -0.5".split())
    assert (o["basis"], o["nPairStates"], o["nParticles"], o["g"]) == ("pairing", 8, 8, -0.5)


def test_config_file_then_command_line(tmp_path):
    cfg = tmp_path / "run.cfg"
    cfg.write_text("--electronGas -r 2.0\n-s 32\t-p 4\n-t 1e-10\n")
    o = cli.parse_args(["-c", str(cfg)])
    assert (o["basis"], o["r_s"], o["nShells"], o["nParticleShells"], o["tolerance"]) == \
        ("electron_gas", 2.0, 32, 4, 1e-10)
    # The command line overrides the file, the basis flag included.
    o = cli.parse_args(["-c", str(cfg), "-r", "0.5", "--infMatter", "-d", "0.16"])
    assert (o["basis"], o["r_s"], o["density"], o["nShells"]) == ("inf_matter", 0.5, 0.16, 32)


def test_system_spec_per_basis():
    kind, kw = cli.system_spec(cli.parse_args("--infMatter -d 0.08 -z 1 -s 4 -p 2".split()))
    assert kind == "inf_matter"
    assert kw == dict(density=0.08, tz_max=1, n_shells=4, n_particle_shells=2, load_v_pppp=True,
                      tables=False, v_blocks=True)
    kind, kw = cli.system_spec(cli.parse_args("--pairing -l 8 -n 8 -x 1.0 -g 0.5".split()))
    assert kind == "pairing"
    assert kw == dict(xi=1.0, g=0.5, n_pair_states=8, n_particles=8, load_v_pppp=True,
                      tables=False, v_blocks=True)
    kind, kw = cli.system_spec(cli.parse_args("--electronGas -r 1 -s 19 -p 2 -m 1".split()))
    assert kind == "electron_gas" and kw["load_v_pppp"] is False  # saveMemory: V on the device
    assert kw["v_blocks"] is False


def test_batch_file_lines_on_top_of_command_line(tmp_path):
    bf = tmp_path / "sweep.txt"
    bf.write_text("# sweep\n--electronGas -r 1.0 -s 19 -p 2\n\n-r 2.0   # same basis, other r_s\n"
                  "--pairing -l 8 -n 8\n")
    base = cli.parse_args(["--electronGas", "-s", "15", "-t", "1e-9", "--batch", str(bf)])
    specs = cli.batch_specs(str(bf), base)
    assert len(specs) == 3
    assert (specs[0]["r_s"], specs[0]["nShells"], specs[0]["tolerance"]) == (1.0, 19, 1e-9)
    assert (specs[1]["basis"], specs[1]["r_s"], specs[1]["nShells"]) == ("electron_gas", 2.0, 15)
    assert specs[2]["basis"] == "pairing" and specs[2]["nPairStates"] == 8
