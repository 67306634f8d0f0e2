"""The bench's multi-rank host side on the CPU: two gloo ranks as torchrun
would start them (one process per GPU on the box), with nothing on a GPU.

The device path shards as independent replicas with no exchange, so the
collectives are the timing barrier and the max over ranks; the whole-job
figure divides all ranks' units by the slowest rank's time, and the
reference arm runs on rank 0 alone.
"""

from __future__ import annotations

import argparse
import contextlib
import io
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    ranks = bench.Ranks("gloo", timeout_s=60)
    # this rank's own timing: rank 1 is the slow one
    slowest = ranks.max_over_ranks(2.0 + 3.0 * rank)
    ranks.barrier()
    rate = bench.whole_job_rate(1000.0, slowest, ranks.world)
    ranks.close()
    out.put((rank, ranks.world, slowest, rate))


def test_two_ranks_agree_on_the_slowest_time_and_the_whole_job_rate():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for _, world, slowest, rate in got:
        assert world == 2
        assert slowest == 5.0  # the max over ranks, seen by both
        assert rate == 1000.0 * 2 / 5.0  # both ranks' units over the slowest time


def test_one_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, str(ROOT))
    import bench

    ranks = bench.Ranks("gloo")
    assert ranks.world == 1 and ranks.dist is None
    assert ranks.max_over_ranks(3.5) == 3.5
    ranks.barrier()
    ranks.close()


def test_the_reference_arm_runs_on_rank_zero_alone(monkeypatch):
    # under torchrun every rank starts the reference arm; all but rank 0 leave
    # at once, printing nothing and running nothing
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(size=4096, steps=1, warmup=0, gpus=2)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args)
    assert buf.getvalue() == ""


def test_the_metric_names_the_plane_it_ran():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.metric_for(4096) == bench.METRIC
    assert bench.metric_for(128) == "site-updates/s (plain 2D sweep, 128^2)"
