"""The multi-GPU path of bench.py is replicas: every rank solves its own system, the job's
time is the slowest rank's device time and its work the iterations of all ranks.  Checked
with two gloo ranks on the CPU (world size 2), and the rank rule of the reference arm (only
rank 0 runs it)."""
import multiprocessing as mp
import os
import socket
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, REPO)
    import datetime

    import torch
    import bench
    torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r: 10 + 5 r ms of device time, 20 + r iterations.
        q.put((rank, bench.combine_ranks(10.0 + 5.0 * rank, 20 + rank, "cpu", world)))
    finally:
        torch.distributed.destroy_process_group()


def test_replicas_combine_max_time_and_summed_work():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # Every rank sees the same job-wide figures: the slowest time, the summed iterations.
    assert out[0] == out[1] == (15.0, 41.0)
    max_ms, iters = out[0]
    assert abs(iters / (max_ms / 1000.0) - 41.0 / 0.015) < 1e-6


def test_single_process_is_unchanged():
    sys.path.insert(0, REPO)
    import bench
    assert bench.combine_ranks(7.5, 12, "cpu", 1) == (7.5, 12.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, REPO)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        config = "eg14"
    bench.run_reference_arm(Args())  # returns at once on a non-zero rank
    assert capsys.readouterr().out == ""
