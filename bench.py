"""Benchmark: CCD iterations/s and time-to-converge of the B200 solver.

One "step" is one complete CCD solve of the workload from T2 = 0 with the reference's stop
rule (|dE| <= tol on the total correlation energy, at most 101 iterations, mixing 0.5) and
tol = 1e-8 N, which keeps the energy within 1e-7 per particle of the converged value.
`value` = iterations of all timed steps / their device time (inputs resident in HBM, L2
flushed before every step).  `e2e` runs the same solve through the C ABI from host buffers:
create (upload of the problem) + solve + read-back of T2 + destroy, every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config eg54c36] [--impl reference]

Default workload: the 3D electron gas with N=54, r_s=2.0, |n|^2 <= 36 (1850 spin-orbitals),
V_pppp generated on the device from the model, mixed precision (split-bf16 tensor-core pp
ladder, FP64 polish) as the headline arm beside the plain FP64 solver.

--impl reference times the reference's own loop (oracle/_ref/ref_harness: the unmodified
reference sources, one MPI rank, all host cores as OpenMP threads) on the same workload, stop
rule and `config`: one set-up, then each step is a bounded sample of the solve.

With --gpus N under torchrun every rank solves its own replica of the workload (the CCD
iteration of one system is not sharded); value sums the iterations of all ranks over the
maximum device time.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "CCD iter/s & time-to-converge, mixed vs FP64 on 1 B200 at |ΔE/N|≤1e-7; %peak"

# name -> description, builder kind, builder params, reference CLI, particles, golden fixture
# (tests/golden, a reference run at tol 1e-12), V_pppp mode of the GPU arm, iterations per
# reference-arm step (a bounded sample: one step stays around a second of host time).
CONFIGS = {
    "eg54c36": dict(desc="3D electron gas, N=54, r_s=2.0, |n|^2<=36 (1850 spin-orbitals)",
                    kind="electron_gas", params=dict(r_s=2.0, n_shells=32, n_particle_shells=4),
                    cli=["--electronGas", "-r", "2.0", "-s", "32", "-p", "4"], n=54,
                    golden="eg54c36_r2", v_mode="on_the_fly", ref_iters=3),
    "eg54c36r05": dict(desc="3D electron gas, N=54, r_s=0.5, |n|^2<=36 (1850 spin-orbitals)",
                       kind="electron_gas",
                       params=dict(r_s=0.5, n_shells=32, n_particle_shells=4),
                       cli=["--electronGas", "-r", "0.5", "-s", "32", "-p", "4"], n=54,
                       golden="eg54c36_r05", v_mode="on_the_fly", ref_iters=3),
    "pnm66": dict(desc="pure neutron matter, N=66, rho=0.08 fm^-3, |n|^2<=36 (1850 "
                       "spin-orbitals)", kind="inf_matter",
                  params=dict(density=0.08, tz_max=1, n_shells=32, n_particle_shells=5),
                  cli=["--infMatter", "-d", "0.08", "-z", "1", "-s", "32", "-p", "5"], n=66,
                  golden="pnm66_s32", v_mode="stored", ref_iters=3),
    "eg14": dict(desc="3D electron gas, N=14, r_s=1.0, |n|^2<=20 (778 spin-orbitals)",
                 kind="electron_gas", params=dict(r_s=1.0, n_shells=19, n_particle_shells=2),
                 cli=["--electronGas", "-r", "1.0", "-s", "19", "-p", "2"], n=14,
                 golden="eg14_s19", v_mode="stored", ref_iters=101),
    "eg54c20": dict(desc="3D electron gas, N=54, r_s=1.0, |n|^2<=20 (778 spin-orbitals)",
                    kind="electron_gas", params=dict(r_s=1.0, n_shells=19, n_particle_shells=4),
                    cli=["--electronGas", "-r", "1.0", "-s", "19", "-p", "4"], n=54,
                    golden="eg54_s19", v_mode="stored", ref_iters=10),
    "pairing": dict(desc="pairing model, 8 levels, 4 pairs, g=-1.0", kind="pairing",
                    params=dict(xi=1.0, g=-1.0, n_pair_states=8, n_particles=8),
                    cli=["--pairing", "-l", "8", "-n", "8", "-x", "1.0", "-g", "-1.0"], n=8,
                    golden="pairing_gm1.0", v_mode="stored", ref_iters=101),
}
DEFAULT_CONFIG = "eg54c36"
MIXING = 0.5
MAX_ITERS = 100  # the reference's cap: at most 101 iterations (main.cpp:509-519)


def stop_tol(n_particles):
    """|dE| bound of the stop rule that keeps the converged energy within 1e-7 per particle
    of the fully converged value (a factor-10 margin over the linear convergence tail;
    the achieved error is measured against the reference and reported)."""
    return 1e-8 * n_particles


def config_dict(name):
    """The workload description, identical in the GPU arm's and the reference arm's lines."""
    c = CONFIGS[name]
    return {"workload": c["desc"], "reference_cli": " ".join(c["cli"]),
            "stop_rule": f"|dE| <= 1e-8 N = {stop_tol(c['n']):g} on the total correlation "
                         "energy (keeps |dE/N| <= 1e-7)",
            "start": "T2 = 0", "mixing": MIXING, "max_iterations": MAX_ITERS + 1,
            "l2": "GPU arm: flushed (256 MiB write) before every step"}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def combine_ranks(dev_ms, iters, device, world):
    """Replicas: the job's time is the slowest rank's device time (MAX) and its work the
    iterations of all ranks (SUM); returns (max_ms, total_iterations)."""
    import torch
    ms = torch.tensor([float(dev_ms)], dtype=torch.float64, device=device)
    it = torch.tensor([float(iters)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(ms, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(it, op=torch.distributed.ReduceOp.SUM)
    return float(ms.item()), float(it.item())


def dram_traffic():
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch per (workload,
    kernel), from ncu captures (bench_dram_traffic.json beside this file)."""
    try:
        with open(os.path.join(REPO, "bench_dram_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_gemm_peak(device, n=8192, reps=3):
    """FP64 GEMM throughput of this GPU (cuBLAS DGEMM n^3 through torch), TF/s: the FP64
    denominator of the ladder rooflines, measured in the run."""
    import torch
    a = torch.rand(n, n, dtype=torch.float64, device=device)
    b = torch.rand(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (ms / 1e3) / 1e12


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def reference_threads(name):
    # The reference's pairing basis builds its three-body maps correctly only single-threaded
    # (SPBasis.cpp:227-255 appends inside an omp parallel region without omp for).
    return 1 if CONFIGS[name]["kind"] == "pairing" else (os.cpu_count() or 1)


def reference_bench(name, steps, timeout):
    """The reference's own loop (oracle/_ref/ref_harness, bench mode) on this host: one
    set-up, then `steps` solves from T2 = 0, each a bounded sample of at most ref_iters
    iterations at the GPU arm's stop rule.  Returns ([(iterations, seconds, e_corr)],
    setup seconds, threads) or raises."""
    c = CONFIGS[name]
    exe = os.path.join(REPO, "oracle", "_ref", "ref_harness")
    threads = reference_threads(name)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1",
               CCD_BENCH=f"{steps},{c['ref_iters']},{stop_tol(c['n'])!r}")
    out = subprocess.run([exe, *c["cli"]], env=env, capture_output=True, text=True,
                         timeout=timeout, check=True).stdout
    rows = [(int(a), float(b), float(e)) for a, b, e in
            re.findall(r"^bench_step: (\d+) ([0-9.eE+-]+) (\S+)", out, re.M)]
    setup = sum(float(x) for x in re.findall(r"^(?:setup|load)_time: ([0-9.eE+-]+)", out, re.M))
    if len(rows) != steps:
        raise RuntimeError("reference harness printed %d of %d steps" % (len(rows), steps))
    return rows, setup, threads


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    c = CONFIGS[args.config]
    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ref_harness")):
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference build oracle/_ref/ref_harness missing (built from the "
                          "reference sources by oracle/build.py)"}))
        return
    rows, setup, threads = reference_bench(args.config, args.warmup + args.steps, timeout=3000)
    timed = rows[args.warmup:]
    its = sum(r[0] for r in timed)
    secs = sum(r[1] for r in timed)
    value = its / secs
    sample = (f"{args.steps} timed steps after {args.warmup} warm-up steps in one process "
              f"after one set-up ({setup:.1f} s, untimed); each step a solve from T2 = 0 "
              f"capped at {c['ref_iters']} iterations of the reference loop "
              f"({its} iterations timed)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iter/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args.config),
        "time": "per step: wall time of the reference loop (its cc_diagrams_time span), "
                "1 MPI rank, OMP threads = host cores, OpenBLAS single-threaded",
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


PRECISIONS = {"mixed": "mixed_bf16", "fp64": "fp64"}
FP64_PEAK_FALLBACK = 35.47  # cuBLAS DGEMM 8192^3 measured on this pool's B200 (FP64 pipe)


def golden_reference(name):
    """The reference's converged energy and sampled T2 (every 97th element) for a workload,
    from the committed fixture of a reference run at tol 1e-12; None if there is none."""
    import numpy as np
    path = os.path.join(REPO, "tests", "golden", CONFIGS[name]["golden"] + ".npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    return {"e_corr": float(g["energies"][-1]), "t2": g["t2"], "full": bool(g["t2_full"][0])}


def quad_count(system):
    """Quads of the fused assembly: (strict particle pair a < b, strict hole pair i < j) per
    channel, summed over the channels."""
    import numpy as np
    d = system.chan_dims().astype(np.int64)
    pp = system.array("pp_map").reshape(-1, 2)
    hh = system.array("hh_map").reshape(-1, 2)
    ps = np.concatenate([[0], np.cumsum((pp[:, 0] < pp[:, 1]).astype(np.int64))])
    hs = np.concatenate([[0], np.cumsum((hh[:, 0] < hh[:, 1]).astype(np.int64))])
    po = np.concatenate([[0], np.cumsum(d[:, 0])])
    ho = np.concatenate([[0], np.cumsum(d[:, 1])])
    return int(((ps[po[1:]] - ps[po[:-1]]) * (hs[ho[1:]] - hs[ho[:-1]])).sum())


def assemble_bytes(n_quads, nt):
    """Algorithmic bytes of one fused assembly launch, per quad (four amplitudes (ab,ij),
    (ab,ji), (ba,ij), (ba,ji)): read t, V and D at (ab,ij), R and the int32 phhp index at the
    four positions (72 B); write the four amplitudes and their phhp copies (64 B) and the next
    iteration's operand-image entries of row ab, columns ij and ji, in both images: nt bf16
    terms each (mixed) or one FP64 value."""
    return n_quads * (136.0 + (8.0 * nt if nt else 32.0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default=DEFAULT_CONFIG, choices=list(CONFIGS) + ["batch24"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="fused", choices=["fused", "tables"])
    ap.add_argument("--precision", default="mixed", choices=list(PRECISIONS),
                    help="headline arm; the other precision is timed beside it")
    ap.add_argument("--v-mode", default=None, choices=["stored", "on_the_fly", "in_ladder"],
                    help="stored: V_pppp built on the host and uploaded; on_the_fly: generated "
                         "on the device from the model at create; in_ladder: as on_the_fly, and "
                         "the electron gas's tensor-core ladder regenerates it every iteration "
                         "(default: the workload's own setting)")
    ap.add_argument("--no-device-loop", action="store_true",
                    help="replay per-iteration graphs instead of the device solve loop (for "
                         "profilers, which cannot see kernels inside graph WHILE nodes)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default pp-ladder schedule instead of autotuning it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--single-arm", action="store_true",
                    help="time only the headline precision (for profiler launch lists)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.config == "batch24":
        run_batch(args)
        return

    import numpy as np
    import torch

    from coupled_cluster_doubles_b200 import CCDSolver, System

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg = CONFIGS[args.config]
    v_mode = args.v_mode or cfg["v_mode"]
    kind, params = cfg["kind"], cfg["params"]
    system = getattr(System, kind)(**params, load_v_pppp=v_mode == "stored")
    n_part = system.n_particles
    tol = stop_tol(n_part)
    if args.path == "tables" and args.precision == "mixed":
        args.precision = "fp64"  # the table path is FP64 only
    arms = [args.precision] + ([p for p in PRECISIONS if p != args.precision]
                               if args.path == "fused" and not args.single_arm else [])
    solvers = {a: CCDSolver(system, device=local, path=args.path, precision=PRECISIONS[a],
                            v_mode=v_mode, device_loop=not args.no_device_loop)
               for a in arms}
    stream = {a: torch.cuda.ExternalStream(solvers[a].stream_ptr(), device=local) for a in arms}
    # Autotuner: each arm's pp-ladder schedule picked by timing the candidates (untimed setup).
    tuned = {a: (solvers[a].autotune(reps=3) if not args.no_autotune else
                 (solvers[a].schedule(), None, None)) for a in arms}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    gold = golden_reference(args.config)

    for a in arms:
        for _ in range(args.warmup):
            solvers[a].reset()
            solvers[a].solve(tol=tol, max_iters=MAX_ITERS, mixing=MIXING)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # Timed region per arm: K solves from T2 = 0, L2 flushed (256 MiB write) before each, on
    # the solver's own stream; device time between CUDA events on that stream.
    timing = {}
    launches0 = {a: solvers[a].profile()["launches"] for a in arms}
    with ClockSampler(local) as clocks:
        for a in arms:
            sol, st = solvers[a], stream[a]
            iters, dev_ms, last = 0, 0.0, None
            barrier()
            torch.cuda.synchronize()
            for _ in range(args.steps):
                with torch.cuda.stream(st):
                    flush.fill_(1.0)
                sol.reset()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                torch.cuda.nvtx.range_push("timed_solve")  # profilers: ncu --nvtx-include
                last = sol.solve(tol=tol, max_iters=MAX_ITERS, mixing=MIXING)
                torch.cuda.nvtx.range_pop()
                e1.record(st)
                e1.synchronize()
                dev_ms += e0.elapsed_time(e1)
                iters += last.iterations
            torch.cuda.synchronize()
            barrier()
            max_ms, total_it = combine_ranks(dev_ms, iters, f"cuda:{local}", world)
            t2 = sol.t2()
            acc = {}
            if gold is not None:
                t2s = t2 if gold["full"] else t2[::97]
                acc = {"abs_de_per_particle_vs_reference":
                       abs(last.e_corr - gold["e_corr"]) / n_part,
                       "t2_max_abs_vs_reference": float(np.max(np.abs(t2s - gold["t2"])))}
            timing[a] = {"max_ms": max_ms, "iters": total_it,
                         "iters_per_solve": last.iterations,
                         "polish_per_solve": last.polish_iterations,
                         "e_corr": last.e_corr, **acc,
                         "launches": solvers[a].profile()["launches"] - launches0[a]}

    # Kernel-level pass per arm: one solve with CUDA events around every kernel family.
    prof, work = {}, {}
    for a in arms:
        sol = solvers[a]
        sol.reset()
        sol.enable_profiling(True)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        sol.solve(tol=tol, max_iters=MAX_ITERS, mixing=MIXING)
        prof[a] = sol.profile()
        sol.enable_profiling(False)
        work[a] = sol.work_per_iteration()
    # Live schedule of one iteration inside the device solve loop: when the first and the last
    # CTA of every kernel started and when the last one finished (%globaltimer, us), relative
    # to the earliest start.
    trace = {}
    for a in arms:
        sol = solvers[a]
        sol.reset()
        sol.trace_arm(5)
        sol.solve(tol=tol, max_iters=MAX_ITERS, mixing=MIXING)
        trace[a] = {k: [round(f / 1e3, 2), round(l / 1e3, 2),
                        round(e / 1e3, 2) if e is not None else None]
                    for k, (f, l, e) in sorted(sol.trace_read(with_end=True).items(),
                                               key=lambda x: x[1][0])}
        sol.trace_arm(-1)
    ladder_cls = {a: solvers[a].ladder_profile(reps=5) for a in arms}
    other_cls = solvers[arms[0]].kernel_profile(reps=5)  # shared by both arms
    n_t2 = solvers[arms[0]].n_t2
    n_quads = quad_count(system)
    nt_of = {"mixed": 2, "fp64": 0}

    # e2e (headline arm): the public API from host buffers, every step: create (H2D upload)
    # + solve + T2 read-back + destroy.  The problem carries no loadMaps tables: create derives
    # them on the device, as a caller that skips loadMaps would have it; with V generated on
    # the device it carries no V block either.
    host_t2 = np.empty(n_t2)
    e2e_secs, e2e_iters = 0.0, 0
    stored = v_mode == "stored"
    system_e2e = getattr(System, kind)(**params, load_v_pppp=stored, tables=False,
                                       v_blocks=stored)
    h2d = _problem_bytes(system_e2e, with_v_pppp=stored, with_tables=False, with_v=stored)
    phase_s = np.zeros(4)  # create, solve (graph capture included), T2 read-back, destroy
    create_ms = np.zeros(5)  # ccdgpu_create by phase (host metadata, uploads, device set-up, schedules, all)
    graph_ms = 0.0  # building of the device-loop graph (inside create, beside the set-up kernels)
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s2 = CCDSolver(system_e2e, device=local, path=args.path, precision=PRECISIONS[arms[0]],
                       v_mode=v_mode, device_loop=not args.no_device_loop)
        ta = time.perf_counter()
        if k >= args.warmup:
            create_ms += np.array(s2.profile()["ms_create"])
        r2 = s2.solve(tol=tol, max_iters=MAX_ITERS, mixing=MIXING)
        tb = time.perf_counter()
        if k >= args.warmup:
            graph_ms += s2.profile()["ms_loop_graph"]
        s2.t2(host_t2)
        tc = time.perf_counter()
        s2.close()
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_secs += t1 - t0
            e2e_iters += r2.iterations
            phase_s += np.array([ta - t0, tb - ta, tc - tb, t1 - tc])
    system_e2e.close()
    e2e_secs_max, e2e_iters_all = combine_ranks(e2e_secs, e2e_iters, f"cuda:{local}", world)
    fp64_peak, fp64_peak_src = FP64_PEAK_FALLBACK, "fallback (cuBLAS DGEMM measured earlier)"
    try:
        fp64_peak = fp64_gemm_peak(torch.device(f"cuda:{local}"))
        fp64_peak_src = "cuBLAS DGEMM 8192^3 measured in this run"
    except RuntimeError:
        pass

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        hbm = peaks["hbm_gbs"]
        traffic = dram_traffic()
        per_it = {}
        for a in arms:
            p = prof[a]
            it_p = max(p["iterations"], 1)
            per_it[a] = {"pp_ladder": p["ms_ladder"] / it_p, "hh_ladder": p["ms_hh_ladder"] / it_p,
                         "ring": p["ms_ring"] / it_p, "onebody": p["ms_onebody"] / it_p,
                         "assemble_energy": p["ms_assemble"] / it_p,
                         "iteration": p["ms_total"] / it_p}
        head = arms[0]
        t = timing[head]
        value = t["iters"] / (t["max_ms"] / 1000.0)

        def cls_bytes(*names):
            return sum(other_cls[n][2] for n in names if n in other_cls)

        def cls_flops(*names):
            return sum(other_cls[n][1] for n in names if n in other_cls)

        # Per kernel family of one iteration: algorithmic bytes (and flops) per launch over its
        # average device time in the profiled solve (events around each family on its stream).
        def kernel_rooflines(a):
            nt = nt_of[a]
            lad = "pp_ladder_tc_kernel<2>" if a == "mixed" else "pp_ladder_kernel<0,1,2>"
            fams = [
                ("pp_ladder", lad, work[a]["ladder_bytes"], work[a]["ladder_flops"]),
                ("assemble_energy", "assemble_fused_kernel", assemble_bytes(n_quads, nt), 0.0),
                ("ring", "phhp_gather_kernel + ring_small_kernel + ring16_kernel<32/48/64>",
                 cls_bytes("ring_small", "ring_mid", "ring_large"),
                 cls_flops("ring_small", "ring_mid", "ring_large")),
                ("hh_ladder", "hh_mma_kernel<2> + hh_slice_kernel + hh_reduce_kernel",
                 cls_bytes("hh_small", "hh_large", "hh_reduce"),
                 cls_flops("hh_small", "hh_large")),
                ("onebody", "onebody_fused_kernel", cls_bytes("onebody"), 0.0),
            ]
            out = {}
            for fam, kname, by, fl in fams:
                ms = per_it[a][fam]
                if ms <= 0 or by <= 0:
                    continue
                gbs = by / (ms / 1e3) / 1e9
                tr = traffic.get(f"{args.config}|{v_mode}|{a}|{kname}")
                out[fam] = {"kernel": kname, "bound": "hbm", "achieved": gbs, "peak": hbm,
                            "unit": "GB/s", "frac": gbs / hbm, "traffic": tr,
                            "algorithmic_bytes_per_launch": by, "avg_launch_ms": ms}
                if fl > 0:
                    out[fam]["fp64_tflops"] = fl / (ms / 1e3) / 1e12
            return out

        roof = {a: kernel_rooflines(a) for a in arms}
        # The table path has no per-family events (its stages are separate calls): no roofline.
        dominant = (max(roof[head], key=lambda f: roof[head][f]["avg_launch_ms"])
                    if roof[head] else None)
        arms_out = {}
        for a in arms:
            ta = timing[a]
            lms = per_it[a]["pp_ladder"]
            arms_out[a] = {
                "iter_per_s": ta["iters"] / (ta["max_ms"] / 1000.0),
                "time_to_converge_ms": ta["max_ms"] / args.steps,
                "iterations_per_solve": ta["iters_per_solve"],
                "polish_iterations_per_solve": ta["polish_per_solve"],
                "e_corr": ta["e_corr"],
                "abs_de_per_particle_vs_reference": ta.get("abs_de_per_particle_vs_reference"),
                "t2_max_abs_vs_reference": ta.get("t2_max_abs_vs_reference"),
                "kernel_ms_per_iteration": per_it[a],
                "trace_iteration5_us": trace[a],
                "kernel_rooflines": roof[a],
                # (None on the table path, whose stages have no per-family events.)
                "pp_ladder_tflops_algorithmic": (work[a]["ladder_flops"] / (lms / 1000.0) / 1e12
                                                 if lms > 0 else None),
                "gpu_launches": int(ta["launches"]),
                "schedule": tuned[a][0],
                "schedule_source": "autotuned" if not args.no_autotune else "default",
            }
            # Each ladder class alone: executed rate (packed rows a<=b, K over c<d and hh) and
            # bandwidth; the FP64 wide class holds the largest channels (hh 36..72).
            cls = {}
            for name, (ms, fl, by) in ladder_cls[a].items():
                cls[name] = {"ms": ms, "tflops_executed": fl / (ms / 1000.0) / 1e12,
                             "gbs": by / (ms / 1000.0) / 1e9}
                if name.startswith("fp64"):
                    cls[name]["frac_of_fp64_peak"] = cls[name]["tflops_executed"] / fp64_peak
                else:
                    cls[name]["frac_of_hbm_peak"] = cls[name]["gbs"] / hbm
            arms_out[a]["pp_ladder_classes_alone"] = cls
        # Ring / hh ladder / one-body classes alone (the same kernels in both arms).
        shared = {}
        for name, (ms, fl, by) in other_cls.items():
            shared[name] = {"ms": ms, "gbs": by / (ms / 1000.0) / 1e9,
                            "frac_of_hbm_peak": by / (ms / 1000.0) / 1e9 / hbm}
            if fl > 0:
                shared[name]["tflops"] = fl / (ms / 1000.0) / 1e12
                shared[name]["frac_of_fp64_peak"] = shared[name]["tflops"] / fp64_peak
        cpu = None
        if not args.no_cpu_baseline:
            cpu = _cpu_baseline(args.config)
        result = {"precision": PRECISIONS[head], "path": args.path,
                  "v_pppp": {"stored": "uploaded from the host",
                             "on_the_fly": "generated on the device from the model at create",
                             "in_ladder": "regenerated inside the tensor-core ladder every "
                                          "iteration"}[v_mode],
                  "solve_loop": ("batched graph replay" if args.no_device_loop else
                                 "device (graph WHILE nodes)"),
                  "iterations_per_solve": t["iters_per_solve"],
                  "polish_iterations_per_solve": t["polish_per_solve"],
                  "time_to_converge_ms": t["max_ms"] / args.steps,
                  "e_corr_per_particle": t["e_corr"] / n_part,
                  "abs_de_per_particle_vs_reference": t.get("abs_de_per_particle_vs_reference"),
                  "t2_max_abs_vs_reference": t.get("t2_max_abs_vs_reference"),
                  "reference_golden": ("tests/golden/%s.npz (reference at tol 1e-12; T2 every "
                                       "97th element)" % cfg["golden"]) if gold else None,
                  "fp64_peak_tflops": fp64_peak, "fp64_peak_source": fp64_peak_src,
                  "parallelism": "replicas" if world > 1 else "single GPU"}
        if "fp64" in arms_out and head != "fp64":
            result["speedup_time_to_converge_vs_fp64"] = (
                arms_out["fp64"]["time_to_converge_ms"] / arms_out[head]["time_to_converge_ms"])
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t["max_ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("bf16 2-term split operands, f32 accumulate (pp ladder) + f64"
                      if head == "mixed" else "f64"),
            "data": "synthetic",
            "config": config_dict(args.config),
            "result": result,
            "arms": arms_out,
            "shared_kernels_alone": shared,
            "e2e": {"value": e2e_iters_all / e2e_secs_max, "unit": "iter/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8 * n_t2,
                    "what": "ccdgpu_create from host buffers (remap tables"
                            + ("" if stored else " and every V block")
                            + " made on the device) + ccdgpu_solve + ccdgpu_get_t2 + "
                              "ccdgpu_destroy",
                    "rank0_ms_per_step": dict(zip(["create", "solve", "get_t2", "destroy"],
                                                  (1e3 * phase_s / args.steps).round(3).tolist())),
                    "rank0_create_ms_by_phase": dict(zip(
                        ["host_metadata", "alloc_upload", "device_setup",
                         "schedules_and_loop_graph_during_device_setup", "total"],
                        (create_ms / args.steps).round(3).tolist())),
                    "rank0_loop_graph_build_ms": round(graph_ms / args.steps, 3)},
            "roofline": ({**roof[head][dominant], "family": dominant, "peak_source": peak_kind}
                         if dominant else None),
            "gpu_launches": int(t["launches"]),
            "clocks": clocks.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    for sol in solvers.values():
        sol.close()
    if world > 1:
        torch.distributed.destroy_process_group()


BATCH_SEED = 20261203


def batch_specs():
    """The batched electron-gas sweep: N in {14, 38, 54} x r_s in {0.5, 1, 2, 3, 4, 5, 6, 8},
    each with a cutoff |n|^2 in {16, 20, 24} (n_shells 15 / 19 / 22) drawn from a fixed seed."""
    import numpy as np
    rng = np.random.default_rng(BATCH_SEED)
    return [dict(r_s=rs, n_shells=int(rng.choice([15, 19, 22])), n_particle_shells=p)
            for p in (2, 3, 4) for rs in (0.5, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 8.0)]


def run_batch(args):
    """Config 4: 24 independent systems solved together (ccdgpu_solve_batch), mixed precision
    with V_pppp generated on the device; timed against the same 24 solved one after another.
    value = systems solved per second; each system stops at |dE| <= 1e-8 N."""
    import numpy as np
    import torch

    from coupled_cluster_doubles_b200 import CCDSolver, System, solve_batch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    specs = batch_specs()
    systems = [System.electron_gas(**sp, load_v_pppp=False) for sp in specs]
    ns = [s.n_particles for s in systems]
    tol = min(stop_tol(n) for n in ns)  # one stop threshold for the batch: the strictest
    mixed = [CCDSolver(s, device=local, precision="mixed_bf16", v_mode="on_the_fly") for s in systems]
    ref = [CCDSolver(s, device=local, v_mode="on_the_fly") for s in systems]
    # Low-density members of the sweep do not converge under the reference's iteration (capped
    # at 101 iterations or diverging to non-finite amplitudes); they are run and counted, and
    # errors are compared on the systems that converge in both precisions.
    e_conv = [r.e_corr for r in solve_batch(ref, tol=1e-12, check=False)]
    streams = [torch.cuda.ExternalStream(m.stream_ptr(), device=local) for m in mixed]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def timed(run):
        for m in mixed:
            m.reset()
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        res = run()
        ends = []
        for st in streams:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(st)
            ends.append(e1)
        torch.cuda.synchronize()
        return max(e0.elapsed_time(e1) for e1 in ends), res

    for _ in range(args.warmup):
        timed(lambda: solve_batch(mixed, tol=tol, check=False))
    batch_ms, seq_ms, res = [], [], None
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            ms, res = timed(lambda: solve_batch(mixed, tol=tol, check=False))
            batch_ms.append(ms)
        for _ in range(args.steps):
            ms, _ = timed(lambda: [solve_batch([m], tol=tol, check=False) for m in mixed])
            seq_ms.append(ms)
    b_ms = sum(batch_ms) / len(batch_ms)
    s_ms = sum(seq_ms) / len(seq_ms)
    import math
    iters = sum(r.iterations for r in res)
    status = ["diverged" if not math.isfinite(r.e_corr) else
              ("converged" if r.converged else "capped") for r in res]
    de = [abs(r.e_corr - e) / n for r, e, n, st in zip(res, e_conv, ns, status)
          if st == "converged" and math.isfinite(e)]
    if rank == 0:
        line = {
            "metric": METRIC, "value": len(systems) / (b_ms / 1000.0), "unit": "systems/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": b_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 2-term split operands, f32 accumulate (pp ladder) + f64",
            "data": "synthetic",
            "config": {"workload": "24 electron-gas systems, N in {14,38,54} x r_s in "
                                   "{0.5,1,2,3,4,5,6,8}, cutoff |n|^2 in {16,20,24} drawn with "
                                   f"numpy default_rng({BATCH_SEED})",
                       "systems": [dict(sp, N=n, status=st, iterations=r.iterations)
                                   for sp, n, st, r in zip(specs, ns, status, res)],
                       "converged": status.count("converged"), "capped": status.count("capped"),
                       "diverged": status.count("diverged"),
                       "precision": "mixed_bf16", "v_pppp": "generated on the device",
                       "stop_rule": f"|dE| <= {tol:g}", "iterations_total": iters,
                       "iter_per_s": iters / (b_ms / 1000.0),
                       "sequential_ms": s_ms, "batch_speedup_vs_sequential": s_ms / b_ms,
                       "max_abs_de_per_particle_vs_fp64_converged": max(de) if de else None,
                       "l2": "flushed (256 MiB write) before every step"},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    for m in mixed + ref:
        m.close()
    for s in systems:
        s.close()


def _problem_bytes(system, with_v_pppp=True, with_tables=True, with_v=True):
    """Bytes ccdgpu_create copies host -> device for this system: V blocks in their reference
    layouts (the a <= b rows of V_pppp, V_hhpp, V_hhhh of amplitude-carrying channels, both modified-channel V,
    the three-body V), the eight ChainIndex tables (24 bytes per entry) or, without them, the
    16-byte modified-pair lookup per (particle, hole), the energies and the O(sum pp) pair
    metadata.  with_v=False: no V block; the modified channels' pair lists (8 bytes a pair)
    instead, from which the device generates them."""
    import numpy as np
    d = system.chan_dims()
    act = (d[:, 0] > 0) & (d[:, 1] > 0)
    pp = d[act, 0].astype(np.int64)
    hh = d[act, 1].astype(np.int64)
    md = system.array("chan_mod_dims").reshape(-1, 4)
    hp = md[:, 2].astype(np.int64)
    ph = md[:, 3].astype(np.int64)
    n_t = int((pp * hh).sum())
    # V_pppp: only the rows a <= b of each block cross (pr rows of pp values).
    pm = system.array("pp_map").reshape(-1, 2)
    starts = np.concatenate([[0], np.cumsum(d[:, 0])[:-1]]).astype(np.int64)
    keep = (pm[:, 0] <= pm[:, 1]).astype(np.int64)
    pr_all = np.add.reduceat(keep, starts[d[:, 0] > 0]) if len(keep) else np.zeros(0, np.int64)
    pr = pr_all[(d[d[:, 0] > 0, 1] > 0)]
    v = 8 * int((pr * pp).sum() * (1 if with_v_pppp else 0) + n_t + (hh * hh).sum() +
                (ph * hp).sum() + (hp * hp).sum())
    v += 8 * 2 * n_t
    if not with_v:
        act_m = (ph > 0) & (hp > 0)
        v = 8 * int(ph[act_m].sum() + hp[act_m].sum()) + 40 * int(act_m.sum())
    meta = 24 * int(pp.sum()) + 16 * int(hh.sum()) + 8 * system.n_sp
    npart = system.n_sp - system.n_particles
    tables = 24 * 8 * n_t if with_tables else 16 * npart * system.n_particles
    return v + tables + meta


def _cpu_baseline(name, steps=2):
    """The reference's loop on this host's cores (oracle/_ref, bench mode): one set-up, then
    `steps` bounded samples of the workload's solve; None when the reference build is
    missing or fails."""
    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ref_harness")):
        return None
    try:
        rows, setup, threads = reference_bench(name, steps, timeout=900)
    except (subprocess.SubprocessError, RuntimeError, OSError, ValueError):
        return None
    it = sum(r[0] for r in rows)
    secs = sum(r[1] for r in rows)
    return {"value": it / secs, "unit": "iter/s", "cores": threads, "kind": "reference",
            "sample": f"{steps} solves from T2 = 0 of the workload, each capped at "
                      f"{CONFIGS[name]['ref_iters']} iterations ({it} iterations, {secs:.3f} s "
                      f"of loop time) by the reference build after one set-up ({setup:.1f} s, "
                      f"untimed); OMP threads = {threads}, 1 MPI rank"}


if __name__ == "__main__":
    main()
