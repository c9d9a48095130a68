"""Test stand-ins for the sharded advection (viennals_b200/shard.py): an
engine that runs the oracle (CPU) and an in-process communicator for shards
driven from threads of one process."""
import threading

import numpy as np

from viennals_b200.domain import Domain, make_runs


class OracleEngine:
    """The oracle as a shard's engine: the slab uploaded into an oracle level
    set, advected with the owned slab and the reduction, and exported in the
    exchange format (runs from the oracle's sign queries)."""

    def __init__(self, grid, velocity):
        self.grid, self.velocity = grid, velocity
        self.own = (-1, 0, 0)
        self.reduce = None

    def upload(self, dom):
        from oracle import oracle as O

        self.ls = O.OracleLS(self.grid, dom)

    def set_owned_region(self, axis, lo, hi):
        self.own = (axis, lo, hi)

    def set_reduction_callback(self, fn):
        self.reduce = fn

    def advect(self, params):
        from oracle import oracle as O

        O.set_shard(*self.own, reduce=self.reduce)
        try:
            return O.advect([self.ls], params, self.velocity)
        finally:
            O.set_shard()

    def download_domain(self):
        idx, vals = self.ls.points(0)
        lo = idx.min(axis=0) - 1 if len(idx) else np.zeros(3, np.int64)
        hi = idx.max(axis=0) + 1 if len(idx) else np.zeros(3, np.int64)

        def sign(x, y, z):
            q = np.stack([x, y, z], 1).astype(np.int32)
            return np.where(self.ls.values_at(q) < 0, -1, 1)

        rs, sg = make_runs(idx, sign, lo, hi)
        return Domain(self.grid, idx, vals, rs, sg, self.ls.width)


class LocalComm:
    """Point-to-point exchange and all-reduce between shards running as
    threads of one process (the torch.distributed calls of shard._Comm)."""

    def __init__(self, world):
        self.world = world
        self.barrier = threading.Barrier(world)
        self.lock = threading.Lock()
        self.box = {}
        self.red = [None] * world

    def for_rank(self, rank):
        outer = self

        class View:
            def allreduce(self, values, op):
                outer.red[rank] = np.array(values, np.float64)
                outer.barrier.wait(timeout=120)
                stack = np.stack(outer.red)
                values[:] = stack.min(axis=0) if op == 0 else stack.max(axis=0)
                outer.barrier.wait(timeout=120)

            def exchange(self, sends, recvs, grid, width):
                with outer.lock:
                    for r, dom in sends.items():
                        outer.box[(rank, r)] = dom
                outer.barrier.wait(timeout=120)
                with outer.lock:
                    got = {r: outer.box.pop((r, rank)) for r in recvs}
                outer.barrier.wait(timeout=120)
                return got

            def allgather_domains(self, dom, grid, width):
                with outer.lock:
                    outer.box[("all", rank)] = dom
                outer.barrier.wait(timeout=120)
                parts = [outer.box[("all", r)] for r in range(outer.world)]
                outer.barrier.wait(timeout=120)
                with outer.lock:
                    outer.box.pop(("all", rank), None)
                return parts

        return View()
