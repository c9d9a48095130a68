"""Spatial sharding of one level set over several shards (viennals_b200/
shard.py): z slabs with ghost planes, a halo exchange after every step and
the time step / alphas / moved flag all-reduced inside every stage.  The
sharded run must give the unsharded run's result bit for bit: the same
defined points and values, time steps and point-update counts.

CPU: slab slicing and joining of the exchange format, the partition, and a
world-size-2 run over gloo with the oracle as each shard's engine.  GPU: two
libvlsgpu contexts as two shards (threads of one process, WENO5 + RK3)
against one context advancing the whole level set."""
import os
import socket
import sys
import threading

import numpy as np
import pytest

from parity_cases import egg_velocity, params, sphere_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slices_join_back_to_the_domain():
    from viennals_b200.shard import concat_z, slice_z

    g, lss = sphere_case(3.0, 0.3)
    d = lss[0]
    cuts = [-(1 << 19), -4, 0, 3, 1 << 19]
    parts = [slice_z(d, a, b) for a, b in zip(cuts[:-1], cuts[1:])]
    j = concat_z(parts)
    assert np.array_equal(j.idx, d.idx) and np.array_equal(j.values, d.values)
    # the joined runs give every cell the sign the original runs give it
    from oracle import oracle as O

    a, b = O.OracleLS(g, d), O.OracleLS(g, j)
    rng = np.random.default_rng(1)
    q = rng.integers(-14, 15, size=(4000, 3)).astype(np.int32)
    assert np.array_equal(np.sign(a.values_at(q)), np.sign(b.values_at(q)))


def test_partition_balances_points():
    from viennals_b200.shard import Z_MAX, Z_MIN, partition_z

    z = np.concatenate([np.full(100, 0), np.arange(-50, 50), np.full(300, 20)])
    b = partition_z(z, 4, min_planes=2)
    assert b[0] == Z_MIN and b[-1] == Z_MAX and all(x < y for x, y in zip(b, b[1:]))
    counts = [int(((z >= lo) & (z < hi)).sum()) for lo, hi in zip(b[:-1], b[1:])]
    assert sum(counts) == len(z) and max(counts) <= 2 * len(z) / 4 + 100


def _unsharded(grid, dom, vel, p, steps):
    from oracle import oracle as O

    ls = O.OracleLS(grid, dom)
    t = 0.0
    upd = 0
    for _ in range(steps):
        r = O.advect([ls], p, vel)
        t += r.advected_time
        upd += r.point_updates
    idx, val = ls.points(0)
    return idx, val, t, upd


def _case():
    g, lss = sphere_case(6.0, 0.3)  # radius 20 cells
    return g, lss[0], egg_velocity(), params(0, 0, 0.0)  # EO1, FE, one step per call


def _gloo_rank(rank, world, port, q, steps):
    import datetime

    import torch

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from shard_support import OracleEngine
    from viennals_b200.shard import ShardedAdvect

    torch.distributed.init_process_group(
        "gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
        timeout=datetime.timedelta(seconds=120))
    try:
        g, dom, v, p = _case()
        sh = ShardedAdvect(OracleEngine(g, v), dom, p, rank, world)
        for _ in range(steps):
            sh.step()
        whole = sh.gather()
        q.put((rank, whole.idx, whole.values, sh.advected_time, sh.point_updates,
               list(sh.bounds), sh.halo))
    finally:
        torch.distributed.destroy_process_group()


def test_sharded_oracle_over_gloo_equals_unsharded():
    import torch.multiprocessing as mp

    steps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q, steps)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = sorted([q.get(timeout=600) for _ in procs], key=lambda x: x[0])
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    g, dom, v, p = _case()
    idx, val, t, upd = _unsharded(g, dom, v, p, steps)
    (_, i0, v0, t0, u0, bounds, halo), (_, i1, v1, t1, u1, _, _) = got
    lo, hi = bounds[1] - halo, bounds[1] + halo
    # the cut lies inside the band with ghost planes on both sides
    assert (dom.idx[:, 2] < lo).any() and (dom.idx[:, 2] >= hi).any()
    for ii, vv in ((i0, v0), (i1, v1)):
        assert np.array_equal(ii, idx)
        assert np.array_equal(vv.view(np.int64), val.view(np.int64))
    assert t0 == t1 == t
    assert u0 + u1 == upd


@pytest.mark.gpu
def test_two_gpu_contexts_as_shards_equal_one_context():
    """WENO5 + RK3 on a sphere of radius 100 cells cut at z = 0: two contexts
    (two shards) against one context, bit for bit in FP64."""
    from shard_support import LocalComm
    from viennals_b200.advect import Context
    from viennals_b200.shard import ShardEngine, ShardedAdvect

    g, lss = sphere_case(5.0, 0.05)
    dom, v = lss[0], egg_velocity()
    p = params(11, 2, 0.0, cfl=0.4)
    steps = 3
    whole = Context(0, 0)
    whole.set_grid(g)
    whole.set_level_set_count(1)
    whole.upload(0, dom)
    whole.set_velocity(v.descriptor())
    t_ref, upd_ref = 0.0, 0
    for _ in range(steps):
        r = whole.advect(p)
        t_ref += r.advected_time
        upd_ref += r.point_updates
    ref_idx, ref_val, _ = whole.download(0)

    comm = LocalComm(2)
    out = [None, None]

    def run(rank):
        sh = ShardedAdvect(ShardEngine(0, 0, g, v), dom, p, rank, 2, comm=comm.for_rank(rank))
        for _ in range(steps):
            sh.step()
        out[rank] = (sh.gather(), sh.advected_time, sh.point_updates, sh.bounds, sh.halo)

    th = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert out[0] is not None and out[1] is not None
    (w0, t0, u0, bounds, halo), (w1, t1, u1, _, _) = out
    assert (dom.idx[:, 2] < bounds[1] - halo).any() and (dom.idx[:, 2] >= bounds[1] + halo).any()
    for w in (w0, w1):
        assert np.array_equal(w.idx, ref_idx)
        assert np.array_equal(w.values.view(np.int64), ref_val.view(np.int64))
    assert t0 == t1 == t_ref
    assert u0 + u1 == upd_ref
