"""The multi-GPU form is replicas: one process per GPU, each analysing its own seeded sequence, with no
collective on the data path; the ranks meet only at the timed region's barriers and in the max over ranks
of its time. These tests run that host side as two gloo ranks on the CPU (127.0.0.1 rendezvous)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    # each rank's own time: the job's is the slowest rank's, on every rank
    got = bench.max_over_ranks(1.5 + rank, world, torch.device("cpu"))
    q.put((rank, got))
    dist.destroy_process_group()


def test_max_over_ranks_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert sorted(q.get() for _ in range(2)) == [(0, 2.5), (1, 2.5)]


def test_replicas_analyse_their_own_sequences():
    sys.path.insert(0, ROOT)
    import bench

    a, b = bench.make_frames(0, 2), bench.make_frames(1, 2)
    assert a.shape == b.shape == (2, 1080, 1920)
    assert not np.array_equal(a, b)
    assert np.array_equal(a, bench.make_frames(0, 2))  # seeded: the same rank sees the same pictures


def test_reference_arm_under_torchrun_prints_one_line():
    """`bench.py --impl reference` launched as two ranks: rank 0 times the oracle and prints the line,
    rank 1 exits without work, and both exit 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def _split_main(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    from ironav_b200.synth import batch_streams

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    mine = bench.split_streams(batch_streams(64), rank, world)
    nmb = sum(((w + 15) // 16) * ((h + 15) // 16) for (w, h, _, _) in mine)
    total = bench.sum_over_ranks(nmb, world, torch.device("cpu"))
    q.put((rank, [s[3] for s in mine], nmb, total))
    dist.destroy_process_group()


def test_batched_streams_split_and_summed_on_two_gloo_ranks():
    """The batched workloads' only multi-GPU form: the 64 streams split across ranks with no collective on
    the data path. Every stream goes to exactly one rank, the shares of macroblocks are balanced, and the
    job's macroblock count is the sum over ranks (not rank 0's share times the rank count)."""
    from ironav_b200.synth import batch_streams

    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_split_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get() for _ in range(2))
    streams = batch_streams(64)
    all_mb = sum(((w + 15) // 16) * ((h + 15) // 16) for (w, h, _, _) in streams)
    seeds = sorted(got[0][1] + got[1][1])
    assert seeds == sorted(s[3] for s in streams)  # each stream on exactly one rank
    assert got[0][3] == got[1][3] == all_mb        # the job's count is the sum over ranks
    assert got[0][2] + got[1][2] == all_mb
    assert abs(got[0][2] - got[1][2]) <= 8160      # balanced within one 1080p stream
