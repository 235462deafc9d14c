"""CPU tests of the multi-rank bench path.  `bench.py --gpus N` runs N independent
replicas (the solve path does not shard); their device-timed regions are combined
as the max over ranks and the whole-job value is N x steps over that time.  Two
gloo ranks on the CPU check the combination; the reference arm runs on rank 0
only."""
import importlib.util
import os
import socket
from datetime import timedelta
from pathlib import Path
from types import SimpleNamespace

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times_ms, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t_max, value = _bench().replicas_throughput(torch, dist, times_ms[rank], steps, world, "cpu")
        q.put((rank, t_max, value))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("times_ms", [(1234.0, 2000.0), (2500.0, 900.0)])
def test_two_gloo_replicas_report_the_slowest_rank(times_ms):
    world, steps = 2, 3
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times_ms, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    slowest = max(times_ms)
    assert [r for r, _, _ in results] == [0, 1]
    for _, t_max, value in results:
        assert t_max == slowest
        assert value == pytest.approx(world * steps / (slowest * 1e-3))


def test_single_rank_needs_no_process_group():
    t_max, value = _bench().replicas_throughput(torch, None, 500.0, 2, 1, "cpu")
    assert t_max == 500.0 and value == pytest.approx(4.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    args = SimpleNamespace(gpus=2, steps=3, warmup=3, n=None, cpu_sample_n=8192)
    _bench().run_reference_arm(args, rank=1, world=2)
    assert capsys.readouterr().out == ""
