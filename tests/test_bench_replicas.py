"""Host logic of the N-replica bench on CPU: two gloo ranks agree on the slowest rank's time,
the whole-job throughput counts every replica's builds, and only rank 0 prints the reference
arm's line."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    sys.path.insert(0, str(ROOT))
    import datetime

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        t = bench.max_over_ranks(dist, times[rank], "cpu")
        out.put((rank, t, bench.replica_throughput(world, 10, t)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, times = 2, [0.25, 0.75]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in res:
        assert t == 0.75
        assert v == pytest.approx(2 * 10 / 0.75)


def test_single_rank_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, 1.5, "cpu") == 1.5
    assert bench.replica_throughput(1, 4, 2.0) == 2.0


def test_reference_arm_prints_only_on_rank_0(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(gpus=2, steps=3, warmup=3, impl="reference")
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    assert buf.getvalue() == ""
