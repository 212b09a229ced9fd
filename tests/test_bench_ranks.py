"""The multi-rank host logic of bench.py on CPU: two gloo ranks, the timings reduced to their
maximum on every rank (weak scaling of independent replicas: the job is as slow as its slowest
rank), and the reference arm printing on rank 0 only."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    mine = [10.0 + rank, 5.0 - rank, 7.0 * (rank + 1)]
    out[rank] = bench.max_over_ranks(mine, "cpu", world)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        assert out[0] == out[1] == [11.0, 5.0, 14.0]


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.0, 2.0], "cpu", 1) == [1.0, 2.0]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "engine")), reason="reference engine not built")
def test_reference_arm_rank1_prints_nothing():
    """Under torchrun every rank but 0 of the reference arm exits 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
