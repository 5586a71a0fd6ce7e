"""Benchmark: CCD iterations/s and time-to-converge of the B200 solver.

One "step" is one complete CCD solve of the workload from T2 = 0 with the reference's stop
rule (|dE| <= tol on the total correlation energy, at most 101 iterations, mixing 0.5).
`value` = iterations of all timed steps / their device time (inputs resident in HBM, L2
flushed before every step).  `e2e` runs the same solve through the C ABI from host buffers:
create (upload of V, maps, energies) + solve + read-back of T2, every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config eg14] [--impl reference]

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

# name -> (description, builder kind, builder params, reference CLI, tol)
CONFIGS = {
    "eg14": ("3D electron gas, N=14, r_s=1.0, |n|^2<=20 (778 spin-orbitals)", "electron_gas",
             dict(r_s=1.0, n_shells=19, n_particle_shells=2),
             ["--electronGas", "-r", "1.0", "-s", "19", "-p", "2"], 1e-12),
    "eg54c20": ("3D electron gas, N=54, r_s=1.0, |n|^2<=20 (778 spin-orbitals)", "electron_gas",
                dict(r_s=1.0, n_shells=19, n_particle_shells=4),
                ["--electronGas", "-r", "1.0", "-s", "19", "-p", "4"], 1e-12),
    "eg54c36": ("3D electron gas, N=54, r_s=2.0, |n|^2<=36 (1850 spin-orbitals)", "electron_gas",
                dict(r_s=2.0, n_shells=32, n_particle_shells=4),
                ["--electronGas", "-r", "2.0", "-s", "32", "-p", "4"], 1e-12),
    "pnm66": ("pure neutron matter, N=66, rho=0.08 fm^-3, |n|^2<=36 (1850 spin-orbitals)",
              "inf_matter", dict(density=0.08, tz_max=1, n_shells=32, n_particle_shells=5),
              ["--infMatter", "-d", "0.08", "-z", "1", "-s", "32", "-p", "5"], 1e-12),
    "pairing": ("pairing model, 8 levels, 4 pairs, g=-1.0", "pairing",
                dict(xi=1.0, g=-1.0, n_pair_states=8, n_particles=8),
                ["--pairing", "-l", "8", "-n", "8", "-x", "1.0", "-g", "-1.0"], 1e-12),
}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


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


def reference_run(cfg, cores, timeout=600):
    """Runs the reference executable (oracle/_ref/ccd.exe) once; returns (iterations, loop s)."""
    exe = os.path.join(REPO, "oracle", "_ref", "ccd.exe")
    _, kind, _, cli, tol = CONFIGS[cfg]
    env = dict(os.environ, OMP_NUM_THREADS=str(1 if kind == "pairing" else cores),
               OPENBLAS_NUM_THREADS="1")
    out = subprocess.run([exe, *cli, "-t", repr(tol)], env=env, capture_output=True, text=True,
                         timeout=timeout, check=True).stdout
    it = int(re.findall(r"^iterations: (\d+)", out, re.M)[-1])
    secs = float(re.findall(r"cc_diagrams_time: ([0-9.eE+-]+)", out)[-1])
    return it, secs, out


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    desc, kind, _, cli, tol = CONFIGS[args.config]
    exe = os.path.join(REPO, "oracle", "_ref", "ccd.exe")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference build oracle/_ref/ccd.exe missing (built from the reference "
                          "sources by oracle/build.py)"}))
        return
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        reference_run(args.config, cores)
    its, secs = 0, 0.0
    for _ in range(args.steps):
        i, s, _ = reference_run(args.config, cores)
        its += i
        secs += s
    value = its / secs
    used = 1 if kind == "pairing" else cores
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iter/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "tol": tol, "cli": " ".join(cli),
                   "time": "reference cc_diagrams_time (CCD loop only), 1 MPI rank"},
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": used, "kind": "reference",
                         "sample": f"{args.steps} full solves ({its} iterations) of the workload"},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="eg14", choices=list(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="fused", choices=["fused", "tables"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import numpy as np
    import torch

    from coupled_cluster_doubles_b200 import CCDSolver, System

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    desc, kind, params, cli, tol = CONFIGS[args.config]
    system = getattr(System, kind)(**params)
    solver = CCDSolver(system, device=local, path=args.path)
    stream = torch.cuda.ExternalStream(solver.stream_ptr(), device=local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def one_solve():
        solver.reset()
        return solver.solve(tol=tol, max_iters=100, mixing=0.5)

    for _ in range(args.warmup):
        one_solve()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # Timed region: K solves, L2 flushed (256 MiB write) before each on the solver's stream.
    iters = 0
    dev_ms = 0.0
    results = []
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            solver.reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = solver.solve(tol=tol, max_iters=100, mixing=0.5)
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
            iters += r.iterations
            results.append(r)
        torch.cuda.synchronize()
        barrier()
    ms = torch.tensor([dev_ms], dtype=torch.float64, device=f"cuda:{local}")
    it_t = torch.tensor([float(iters)], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        torch.distributed.all_reduce(ms, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(it_t, op=torch.distributed.ReduceOp.SUM)
    max_ms = float(ms.item())
    total_iters = float(it_t.item())
    value = total_iters / (max_ms / 1000.0)
    launches = solver.profile()["launches"]

    # Kernel-level pass: the same solve with CUDA events around every kernel family.
    solver.reset()
    solver.enable_profiling(True)
    flush.fill_(1.0)
    torch.cuda.synchronize()
    rp = solver.solve(tol=tol, max_iters=100, mixing=0.5)
    prof = solver.profile()
    solver.enable_profiling(False)
    work = solver.work_per_iteration()
    n_t2 = solver.n_t2

    # e2e: the public API from host buffers, every step: create (H2D) + solve + T2 read-back.
    host_t2 = np.empty(n_t2)
    e2e_secs, e2e_iters = 0.0, 0
    h2d = _problem_bytes(system)
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s2 = CCDSolver(system, device=local, path=args.path)
        r2 = s2.solve(tol=tol, max_iters=100, mixing=0.5)
        s2.t2(host_t2)
        s2.close()
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_secs += t1 - t0
            e2e_iters += r2.iterations
    e2e_t = torch.tensor([e2e_secs], dtype=torch.float64, device=f"cuda:{local}")
    e2e_i = torch.tensor([float(e2e_iters)], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(e2e_i, op=torch.distributed.ReduceOp.SUM)

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        it_p = max(prof["iterations"], 1)
        ladder_ms = prof["ms_ladder"] / it_p
        # Algorithmic bytes of one pp-ladder launch: antisymmetry-packed V_pppp (rows a<=b,
        # columns c<d), the T and X operands and D written in full.
        ladder_bytes = work["ladder_bytes"]
        achieved = ladder_bytes / (ladder_ms / 1000.0) / 1e9
        cpu = None
        if not args.no_cpu_baseline:
            cpu = _cpu_baseline(args.config)
        r0 = results[-1]
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "precision": "fp64", "path": args.path,
                       "tol": tol, "iterations_per_solve": r0.iterations,
                       "e_corr": r0.e_corr, "e_corr_per_particle": r0.e_corr / system.n_particles,
                       "time_to_converge_ms": max_ms / args.steps,
                       "l2": "flushed (256 MiB write) before every step",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "e2e": {"value": e2e_i.item() / e2e_t.item(), "unit": "iter/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8 * n_t2,
                    "what": "ccdgpu_create from host buffers + ccdgpu_solve + ccdgpu_get_t2"},
            "roofline": {"kernel": "pp_ladder_kernel", "bound": "hbm", "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "peak_source": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_launch": ladder_bytes,
                         "avg_launch_ms": ladder_ms,
                         "flops_per_launch": work["ladder_flops"],
                         "tflops": work["ladder_flops"] / (ladder_ms / 1000.0) / 1e12},
            "kernel_ms_per_iteration": {
                "pp_ladder": ladder_ms, "hh_ladder": prof["ms_hh_ladder"] / it_p,
                "ring": prof["ms_ring"] / it_p, "onebody": prof["ms_onebody"] / it_p,
                "assemble_energy": prof["ms_assemble"] / it_p,
                "iteration": prof["ms_total"] / it_p},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    solver.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def _problem_bytes(system):
    """Bytes ccdgpu_create copies host -> device for this system: V blocks in their reference
    layouts (V_pppp, V_hhpp, V_hhhh of amplitude-carrying channels, both modified-channel V,
    the three-body V), the eight ChainIndex tables (24 bytes per entry), the energies and the
    O(sum pp) pair metadata."""
    import numpy as np
    d = system.chan_dims()
    act = (d[:, 0] > 0) & (d[:, 1] > 0)
    pp = d[act, 0].astype(np.int64)
    hh = d[act, 1].astype(np.int64)
    md = system.array("chan_mod_dims").reshape(-1, 4)
    hp = md[:, 2].astype(np.int64)
    ph = md[:, 3].astype(np.int64)
    n_t = int((pp * hh).sum())
    v = 8 * int((pp * pp).sum() + n_t + (hh * hh).sum() + (ph * hp).sum() + (hp * hp).sum())
    v += 8 * 2 * n_t
    meta = 24 * int(pp.sum()) + 16 * int(hh.sum()) + 8 * system.n_sp
    return v + 24 * 8 * n_t + meta


def _cpu_baseline(cfg):
    exe = os.path.join(REPO, "oracle", "_ref", "ccd.exe")
    if not os.path.exists(exe):
        return None
    cores = os.cpu_count() or 1
    kind = CONFIGS[cfg][1]
    try:
        it, secs, _ = reference_run(cfg, cores, timeout=120)
    except (subprocess.SubprocessError, IndexError, OSError):
        return None
    return {"value": it / secs, "unit": "iter/s", "cores": 1 if kind == "pairing" else cores,
            "kind": "reference",
            "sample": f"one full solve of the workload by the reference build ({it} iterations, "
                      f"cc_diagrams_time {secs:.3f} s, OMP threads = cores, 1 MPI rank)"}


if __name__ == "__main__":
    main()
