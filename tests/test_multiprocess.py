"""Host logic of bench.py's multi-rank runs on CPU (gloo, world size 2).

Under torchrun every rank advects its own replica; the bench reduces the
timed-region milliseconds by max and the point updates by sum over ranks,
and the reference arm runs on rank 0 only.
"""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch

    sys.path.insert(0, ROOT)
    import bench

    torch.distributed.init_process_group(
        "gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
        timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms, updates = bench.reduce_over_ranks(10.0 + 5.0 * rank, 1000 * (rank + 1), "cpu")
        q.put((rank, ms, updates))
    finally:
        torch.distributed.destroy_process_group()


def test_reduce_over_ranks_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, updates in got:
        assert ms == 15.0  # max over ranks
        assert updates == 3000.0  # sum over ranks


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1",
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
