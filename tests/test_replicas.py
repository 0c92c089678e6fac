"""The N > 1 path of `bench.py` on the CPU: one process per GPU, each an
independent replica of the workload (the path has no exchange step), timed
as the slowest rank. Two `gloo` ranks stand in for two GPUs: the max over
ranks, the whole-job rate, and the reference arm running on rank 0 only."""

import importlib.util
import os
import socket
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", REPO / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(REPO / "rang-core_b200"))
    bench = _bench()
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, l = bench.replica_env()
        ms = 100.0 + 25.0 * r  # the slower replica sets the job's time
        slowest = bench.max_over_ranks(ms, dist, torch.device("cpu"))
        rate = bench.job_rate(w, 1_000_000, 3, slowest / 1e3)
        # a leg that needs every rank (pinned host memory): one refusal skips it everywhere
        both = bench.all_ranks(True, dist, torch.device("cpu"))
        one_refused = bench.all_ranks(r != 1, dist, torch.device("cpu"))
        out.put((r, w, l, slowest, rate, both, one_refused))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_report_the_slowest_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in results] == [(0, 2, 0), (1, 2, 1)]
    assert all(r[3] == 125.0 for r in results)
    # 2 replicas x 1 M units x 3 steps in 0.125 s
    assert all(r[4] == pytest.approx(48.0) for r in results)
    assert all(r[5] is True and r[6] is False for r in results)


def test_one_process_needs_no_collective():
    bench = _bench()
    assert bench.max_over_ranks(7.5, None, None) == 7.5
    assert bench.all_ranks(True, None, None) and not bench.all_ranks(False, None, None)
    assert bench.job_rate(1, 2_000_000, 2, 0.5) == pytest.approx(8.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    bench = _bench()
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        workload = "ms2dirty 16.5M vis 1024^2"

    assert bench.run_reference(Args()) is None  # returns before any work
    assert capsys.readouterr().out == ""


def test_reference_sample_is_as_large_as_the_run_allows():
    bench = _bench()
    assert bench.reference_stride(20, 3) == 16
    assert bench.reference_stride(40, 3) == 32
    assert bench.reference_stride(100, 5) == 64
