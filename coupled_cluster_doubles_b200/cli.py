"""Command-line front end with the reference's options (parse.cpp:15-229) and output lines
(main.cpp:478-700), running the solve on the GPU through the C ABI.

    python -m coupled_cluster_doubles_b200.cli --electronGas -r 1.0 -s 19 -p 2 -t 1e-12

Reference options and defaults (parse.cpp:128-196, main.cpp:34-39):
  --pairing | --infMatter (default) | --electronGas     basis
  -d/--density 0.08  -g/--g 0.5  -p/--nParticleShells 2  -n/--nParticles 4
  -l/--nPairStates 4  -r/--r_s 0.5  -s/--nShells 4  -t/--tolerance 1e-8  -z/--tzMax 1
  -x/--xi 1.0  -m/--saveMemory 0 (1: every V block generated on the device)  -v/--verbose 0
  -c/--config FILE   whitespace-separated options read first; the command line overrides them
The reference's load-balancer timing options (-T, -W, -M) have no counterpart (one GPU per
system).  Additions: --precision (fp64, mixed_bf16, mixed_bf16x3), --device, --max-iters,
--checkpoint FILE (T2 after the solve, .npy, the reference's t2_pphh order), --restart FILE
(start from a checkpoint instead of T2 = 0), --batch FILE (one system per line, each line
options as above on top of the command line's; all lines solved together with
ccdgpu_solve_batch).
"""
import argparse
import shlex
import sys

PRECISIONS = ("fp64", "mixed_bf16", "mixed_bf16x3")


def _parser():
    ap = argparse.ArgumentParser(prog="coupled_cluster_doubles_b200.cli", add_help=True,
                                 description="CCD on the GPU with the reference's options")
    # Basis flags: the last one given wins (a config file's choice can be overridden).
    ap.add_argument("--pairing", dest="basis", action="store_const", const="pairing")
    ap.add_argument("--infMatter", dest="basis", action="store_const", const="inf_matter")
    ap.add_argument("--electronGas", dest="basis", action="store_const", const="electron_gas")
    ap.add_argument("-c", "--config", metavar="FILE")
    ap.add_argument("-d", "--density", type=float)
    ap.add_argument("-g", "--g", type=float)
    ap.add_argument("-p", "--nParticleShells", type=int)
    ap.add_argument("-n", "--nParticles", type=int)
    ap.add_argument("-l", "--nPairStates", type=int)
    ap.add_argument("-r", "--r_s", type=float)
    ap.add_argument("-s", "--nShells", type=int)
    ap.add_argument("-t", "--tolerance", type=float)
    ap.add_argument("-z", "--tzMax", type=int)
    ap.add_argument("-x", "--xi", type=float)
    ap.add_argument("-m", "--saveMemory", type=int)
    ap.add_argument("-v", "--verbose", type=int)
    ap.add_argument("--precision", choices=PRECISIONS)
    ap.add_argument("--device", type=int)
    ap.add_argument("--max-iters", type=int)
    ap.add_argument("--checkpoint", metavar="FILE")
    ap.add_argument("--restart", metavar="FILE")
    ap.add_argument("--batch", metavar="FILE")
    return ap


DEFAULTS = dict(basis="inf_matter", density=0.08, g=0.5, nParticleShells=2, nParticles=4,
                nPairStates=4, r_s=0.5, nShells=4, tolerance=1e-8, tzMax=1, xi=1.0,
                saveMemory=0, verbose=0, precision="fp64", device=0, max_iters=100,
                checkpoint=None, restart=None, batch=None, config=None)


def _read_tokens(path):
    with open(path) as f:
        return f.read().split()


def parse_args(argv, base=None):
    """Options as the reference reads them: defaults, then the config file's tokens, then the
    command line (a later value wins).  `base` (a dict) replaces the defaults."""
    ap = _parser()
    first = ap.parse_args(argv)
    tokens = list(argv)
    if first.config:
        tokens = _read_tokens(first.config) + tokens
    ns = ap.parse_args(tokens)
    opts = dict(DEFAULTS if base is None else base)
    for k, v in vars(ns).items():
        if v is not None:
            opts[k] = v
    return opts


def system_spec(opts):
    """(System factory name, keyword arguments) of the basis the options describe."""
    if opts["basis"] == "pairing":
        kw = dict(xi=opts["xi"], g=opts["g"], n_pair_states=opts["nPairStates"],
                  n_particles=opts["nParticles"])
    elif opts["basis"] == "inf_matter":
        kw = dict(density=opts["density"], tz_max=opts["tzMax"], n_shells=opts["nShells"],
                  n_particle_shells=opts["nParticleShells"])
    else:
        kw = dict(r_s=opts["r_s"], n_shells=opts["nShells"],
                  n_particle_shells=opts["nParticleShells"])
    kw["load_v_pppp"] = not opts["saveMemory"]
    kw["tables"] = False  # the remap tables are derived on the device at create
    # saveMemory: every V block is generated on the device from the model, none on the host.
    kw["v_blocks"] = not opts["saveMemory"]
    return opts["basis"], kw


def batch_specs(path, opts):
    """One option set per non-empty, non-comment line of a batch file, on top of `opts`."""
    out = []
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if line:
                out.append(parse_args(shlex.split(line), base=opts))
    return out


def _report(system, res, verbose, out):
    a = system.n_particles
    eref, e2 = system.reference_energy, system.mbpt2
    if verbose >= 1:
        print(f"Reference Energy: {eref:.17g}", file=out)
        print(f"Reference Energy/A: {eref / a:.17g}", file=out)
        print(f"MBPT2Corr: {e2:.17g}", file=out)
        print(f"MBPT2Corr/A: {e2 / a:.17g}", file=out)
        print(f"E_mbpt2: {eref + e2:.17g}", file=out)
        print(f"E_mbpt2/A: {(eref + e2) / a:.17g}", file=out)
    print(f"iterations: {res.iterations}", file=out)
    print(f"CCDCorr: {res.e_corr:.17g}", file=out)
    print(f"CCDCorr/A: {res.e_corr / a:.17g}", file=out)
    print(f"E_CCD: {eref + res.e_corr:.17g}", file=out)
    print(f"E_CCD/A: {(eref + res.e_corr) / a:.17g}", file=out)
    print(f"cc_diagrams_time: {res.seconds:f}", file=out)


def main(argv=None, out=None):
    import numpy as np

    from .solver import CCDSolver, solve_batch
    from .system import System

    out = out or sys.stdout
    opts = parse_args(sys.argv[1:] if argv is None else argv)
    v_mode = "on_the_fly" if opts["saveMemory"] else "stored"
    if opts["batch"]:
        specs = batch_specs(opts["batch"], opts)
        systems = [getattr(System, system_spec(o)[0])(**system_spec(o)[1]) for o in specs]
        solvers = [CCDSolver(s, precision=o["precision"], device=o["device"],
                             v_mode="on_the_fly" if o["saveMemory"] else "stored")
                   for s, o in zip(systems, specs)]
        try:
            tol = min(o["tolerance"] for o in specs)
            results = solve_batch(solvers, tol=tol, max_iters=opts["max_iters"], check=False)
            for k, (s, r) in enumerate(zip(systems, results)):
                print(f"system {k}:", file=out)
                _report(s, r, opts["verbose"], out)
        finally:
            for x in solvers + systems:
                x.close()
        return 0
    kind, kw = system_spec(opts)
    with getattr(System, kind)(**kw) as s, \
            CCDSolver(s, precision=opts["precision"], device=opts["device"], v_mode=v_mode) as sol:
        if opts["restart"]:
            sol.set_t2(np.load(opts["restart"]))
        res = sol.solve(tol=opts["tolerance"], max_iters=opts["max_iters"], mixing=0.5)
        if opts["checkpoint"]:
            np.save(opts["checkpoint"], sol.t2())
        _report(s, res, opts["verbose"], out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
