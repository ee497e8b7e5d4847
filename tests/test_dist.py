"""The multi-rank layout on CPU: two gloo ranks (no GPU), as the benchmark and
esp_sharded run them on GPUs with NCCL."""
from __future__ import annotations

import os

import numpy as np
import pytest

from fastesp_b200.shard import shard_range


def test_shard_ranges_cover_once():
    for n in (0, 1, 7, 30000, 30001):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, b = shard_range(n, r, world)
                seen += list(range(a, b))
                assert b - a in (n // world, n // world + 1)
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        from fastesp_b200.shard import esp_sharded, max_over_ranks, rank_info
        assert rank_info() == (rank, world, rank)
        t = max_over_ranks(10.0 + rank)
        pts = np.arange(3 * 11, dtype=np.float64).reshape(11, 3)
        # a stand-in evaluator: any per-point function of the point
        vals = esp_sharded(lambda p: p.sum(axis=1) * (1.0 + 0.0 * rank), pts)
        q.put((rank, t, vals.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.arange(33, dtype=np.float64).reshape(11, 3).sum(axis=1)
    for rank, t, vals in res:
        assert t == 11.0                                  # the max over ranks
        np.testing.assert_array_equal(vals, expect)       # every point once, in order


def test_rank_point_sets_differ(small_system):
    from fastesp_b200.shard import rank_points
    wfn = small_system[0]
    a = rank_points(wfn.symbols, wfn.coords, 50, 0)
    b = rank_points(wfn.symbols, wfn.coords, 50, 1)
    assert a.shape == b.shape == (50, 3) and not np.array_equal(a, b)


def test_bench_launches_one_rank_per_gpu():
    """``bench.py --gpus 2`` without a launcher re-executes itself under
    torch.distributed.run as two ranks; each sees its own RANK / LOCAL_RANK
    (checked here without touching CUDA)."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--gpus", "2", "--print-ranks"],
                       capture_output=True, text=True, timeout=180, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    ranks = sorted((json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")),
                   key=lambda d: d["rank"])
    assert [(d["rank"], d["local_rank"], d["world_size"]) for d in ranks] == [(0, 0, 2), (1, 1, 2)]


def test_launcher_command_line():
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).resolve().parents[1]))
    import bench
    argv = bench.launcher_argv(4, ["--gpus", "4", "--steps", "5"], 29512)
    assert argv[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in argv and "--master-addr=127.0.0.1" in argv
    assert "--master-port=29512" in argv and argv[-4:] == ["--gpus", "4", "--steps", "5"]
