"""The multi-rank path of bench.py on CPU: two gloo ranks (torchrun-style
environment) take the job time as the slowest rank's, report the whole-job
rate of the replicas, and only rank 0 of the reference arm does work."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_init("gloo")
    t = bench.max_over_ranks(1.0 + r, w, "cpu")  # rank r "took" 1 + r seconds
    dist.barrier()
    out.put((r, w, t, bench.job_rate(100.0, w, t)))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, t, rate in got:
        assert w == 2 and t == 2.0          # the slowest rank's time on every rank
        assert rate == pytest.approx(100.0)  # 2 replicas x 100 units / 2 s


def test_reference_arm_rank_nonzero_does_nothing(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup = 1, 0

    bench.run_reference(A())
    assert capsys.readouterr().out == ""


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.job_rate(10.0, 1, 2.0) == 5.0
    json.dumps({"ok": True})
