"""Spatial sharding of one level-set domain over several GPUs.

The reference advects one domain on one node; its only decomposition is the
OpenMP segmentation of the HRLE order (lsAdvect.hpp:464-477), re-balanced
after every rebuild (lsAdvect.hpp:426), with the per-segment time-step minima
and alpha maxima reduced in critical sections (lsAdvect.hpp:595-606,
:186-191).  Here the segments become z slabs, one per process and GPU:

* partition: the band's points are split into contiguous ranges of z planes
  (z is the slowest index of the HRLE order, so a slab is one contiguous run
  of the exchange format) holding equal numbers of points; `rebalance_every`
  steps the boundaries are recomputed from the current band;
* ghost layers: every shard advects its slab plus `halo` planes on each side
  taken from its neighbours.  A time step changes a value only through
  neighbours within the step's reach (the Expand widths, the stencil radius,
  the rebuild and the stage combinations, `halo_width`), so with at least
  that many ghost planes the slab's own values are exactly those of the
  unsharded run; the ghost planes themselves are refreshed from their owners
  after every step (the halo exchange);
* reductions: the time step (min), the Lax-Friedrichs alphas (max) and the
  stage combination's "moved down" flag (max) of each stage are all-reduced
  over the shards inside vlsg_advect (vlsg_set_reduction_callback), counting
  only the points a shard owns (vlsg_set_owned_region);
* the halo exchange and the reductions go through torch.distributed
  (point-to-point send/recv and all_reduce; NCCL between GPUs, gloo on CPU).

An engine is anything with upload(Domain), set_owned_region(axis, lo, hi),
set_reduction_callback(fn), advect(params) and download_domain(): the
library's `ShardEngine` below, or a CPU stand-in in the tests.
"""
import math

import numpy as np

from .domain import INF_INDEX, Domain

NI = -INF_INDEX  # start index of a run that begins before every cell of its row / plane
Z_MIN, Z_MAX = -(1 << 19), 1 << 19  # outside every grid index


def _keys(idx):
    """HRLE order keys (z slowest, x fastest) of (N, 3) indices."""
    i = np.asarray(idx, np.int64) + (1 << 20)
    return (i[:, 2] << 42) | (i[:, 1] << 21) | i[:, 0]


def slice_z(dom, a, b):
    """The part of `dom` in the planes a <= z < b as a Domain of its own: the
    points of those planes, the runs that start there, and a run at the start
    of plane a with the sign that covers that position in `dom` (the last run
    before it), unless a run starts exactly there."""
    pz = dom.idx[:, 2]
    pm = (pz >= a) & (pz < b)
    rz = dom.run_start[:, 2]
    rm = (rz >= a) & (rz < b)
    starts, signs = dom.run_start[rm], dom.run_sign[rm]
    head = np.array([[NI, NI, a]], np.int32)
    hk = _keys(head)[0]
    if not (len(starts) and _keys(starts[:1])[0] == hk):
        before = np.nonzero(_keys(dom.run_start) < hk)[0] if len(dom.run_start) else []
        sign = dom.run_sign[before[-1]] if len(before) else np.int8(1)
        starts = np.concatenate([head, starts])
        signs = np.concatenate([np.array([sign], np.int8), signs])
    out = Domain(dom.grid, dom.idx[pm], dom.values[pm], starts, signs, dom.width)
    return out


def concat_z(parts, grid=None, width=None):
    """Slabs in increasing z order (each from slice_z) joined into one Domain."""
    parts = [p for p in parts if p is not None]
    grid = grid if grid is not None else parts[0].grid
    width = width if width is not None else max(p.width for p in parts)
    cat = lambda name, shape, dt: (np.concatenate([getattr(p, name) for p in parts])
                                   if parts else np.zeros(shape, dt))
    return Domain(grid, cat("idx", (0, 3), np.int32), cat("values", (0,), np.float64),
                  cat("run_start", (0, 3), np.int32), cat("run_sign", (0,), np.int8), width)


def partition_z(z, world, min_planes=1):
    """Slab boundaries b_0 < ... < b_world over the points' z indices: slab r
    is [b_r, b_{r+1}), each holding about the same number of points and at
    least `min_planes` planes; b_0 and b_world lie outside every grid."""
    z = np.asarray(z, np.int64)
    if world == 1 or len(z) == 0:
        return [Z_MIN] + [Z_MAX] * world if world > 1 else [Z_MIN, Z_MAX]
    zs = np.sort(z)
    cuts = []
    for r in range(1, world):
        c = int(zs[min(len(zs) - 1, (r * len(zs)) // world)])
        lo = cuts[-1] + min_planes if cuts else int(zs[0]) + min_planes
        cuts.append(max(c, lo))
    return [Z_MIN] + cuts + [Z_MAX]


def halo_width(params):
    """Ghost planes one time step needs: per forward-Euler stage the Expand
    cycles to the scheme's width, the stencil reach and the rebuild; per
    stage combination the Expand to ceil(2 steps ratio + 1), the two Prune
    passes and the rebuild; plus one plane of margin."""
    s = int(params.spatial_scheme)
    width = {0: 3, 1: 5, 2: 3, 3: 5, 4: 7, 5: 3, 6: 5, 7: 7, 8: 9, 9: 8, 10: 5, 11: 7}[s]
    reach = {0: 1, 1: 2, 2: 1, 3: 2, 4: 2, 5: 1, 6: 2, 7: 2, 8: 3, 9: 2, 10: 2, 11: 3}[s]
    stages = {0: 1, 1: 2, 2: 3}[int(params.temporal_scheme)]
    combines = stages - 1
    e = math.ceil(2.0 * stages * params.time_step_ratio + 1)
    return stages * (width + reach + 1) + combines * (e + 3) + 1


class _Comm:
    """torch.distributed point-to-point of Domains and all-reduce of doubles
    on the process group's device (CUDA for NCCL, CPU for gloo)."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist

        self.torch, self.dist, self.group = torch, dist, group
        if device is None:
            device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        self.device = torch.device(device)

    def allreduce(self, values, op):
        t = self.torch.as_tensor(np.asarray(values, np.float64), device=self.device).clone()
        o = self.dist.ReduceOp.MIN if op == 0 else self.dist.ReduceOp.MAX
        self.dist.all_reduce(t, op=o, group=self.group)
        values[:] = t.cpu().numpy()

    def _tensors(self, dom):
        th = self.torch
        arrs = [dom.idx.astype(np.int32).reshape(-1), dom.values.astype(np.float64),
                dom.run_start.astype(np.int32).reshape(-1), dom.run_sign.astype(np.int32)]
        return [th.as_tensor(a, device=self.device) for a in arrs]

    def exchange(self, sends, recvs, grid, width):
        """sends: {rank: Domain}; recvs: ranks to receive one Domain from.
        Sizes first, then the arrays; non-blocking both ways."""
        th, dist = self.torch, self.dist
        reqs, hdr_in = [], {}
        for r, dom in sends.items():
            h = th.tensor([len(dom.values), len(dom.run_sign)], dtype=th.int64, device=self.device)
            reqs.append(dist.isend(h, r, group=self.group))
        for r in recvs:
            hdr_in[r] = th.zeros(2, dtype=th.int64, device=self.device)
            reqs.append(dist.irecv(hdr_in[r], r, group=self.group))
        for q in reqs:
            q.wait()
        reqs, bufs = [], {}
        for r, dom in sends.items():
            for t in self._tensors(dom):
                if t.numel():
                    reqs.append(dist.isend(t.contiguous(), r, group=self.group))
        for r in recvs:
            n, m = (int(v) for v in hdr_in[r].cpu())
            b = [th.empty(3 * n, dtype=th.int32, device=self.device),
                 th.empty(n, dtype=th.float64, device=self.device),
                 th.empty(3 * m, dtype=th.int32, device=self.device),
                 th.empty(m, dtype=th.int32, device=self.device)]
            bufs[r] = b
            for t in b:
                if t.numel():
                    reqs.append(dist.irecv(t, r, group=self.group))
        for q in reqs:
            q.wait()
        out = {}
        for r, b in bufs.items():
            idx, val, rs, sg = (t.cpu().numpy() for t in b)
            out[r] = Domain(grid, idx.reshape(-1, 3), val, rs.reshape(-1, 3),
                            sg.astype(np.int8), width)
        return out

    def allgather_domains(self, dom, grid, width):
        """Every rank's Domain, in rank order (for re-balancing and results)."""
        world = self.dist.get_world_size(self.group)
        rank = self.dist.get_rank(self.group)
        parts = [None] * world
        parts[rank] = dom
        for r in range(world):
            src = r
            got = self._broadcast_domain(dom if rank == src else None, src, grid, width)
            parts[r] = got
        return parts

    def _broadcast_domain(self, dom, src, grid, width):
        th, dist = self.torch, self.dist
        h = th.zeros(2, dtype=th.int64, device=self.device)
        if dom is not None:
            h = th.tensor([len(dom.values), len(dom.run_sign)], dtype=th.int64, device=self.device)
        dist.broadcast(h, src, group=self.group)
        n, m = (int(v) for v in h.cpu())
        if dom is not None:
            ts = self._tensors(dom)
        else:
            ts = [th.empty(3 * n, dtype=th.int32, device=self.device),
                  th.empty(n, dtype=th.float64, device=self.device),
                  th.empty(3 * m, dtype=th.int32, device=self.device),
                  th.empty(m, dtype=th.int32, device=self.device)]
        for t in ts:
            if t.numel():
                dist.broadcast(t, src, group=self.group)
        idx, val, rs, sg = (t.cpu().numpy() for t in ts)
        return Domain(grid, idx.reshape(-1, 3), val, rs.reshape(-1, 3), sg.astype(np.int8), width)


class ShardedAdvect:
    """One shard of a z-slab decomposition of a single level set (one per
    process; rank r of `world` owns the slab [bounds[r], bounds[r+1]))."""

    def __init__(self, engine, domain, params, rank, world, halo=None, group=None,
                 rebalance_every=0, comm=None):
        self.engine = engine
        self.params = params
        self.rank, self.world = rank, world
        self.grid = domain.grid
        self.width = domain.width
        self.halo = halo if halo is not None else halo_width(params)
        self.comm = comm if comm is not None else (_Comm(group) if world > 1 else None)
        self.rebalance_every = rebalance_every
        self.steps = 0
        self.point_updates = 0
        self.advected_time = 0.0
        self.bounds = partition_z(domain.idx[:, 2], world, min_planes=self.halo)
        self.own = slice_z(domain, *self._slab())
        if world > 1:
            self.engine.set_reduction_callback(self.comm.allreduce)

    def _slab(self, r=None):
        r = self.rank if r is None else r
        return self.bounds[r], self.bounds[r + 1]

    def _ghosts(self):
        """The neighbours' planes within `halo` of this slab."""
        lo, hi = self._slab()
        if self.world == 1:
            return None, None
        sends = {}
        if self.rank > 0:
            sends[self.rank - 1] = slice_z(self.own, lo, lo + self.halo)
        if self.rank + 1 < self.world:
            sends[self.rank + 1] = slice_z(self.own, hi - self.halo, hi)
        recvs = [r for r in (self.rank - 1, self.rank + 1) if 0 <= r < self.world]
        got = self.comm.exchange(sends, recvs, self.grid, self.width)
        below = slice_z(got[self.rank - 1], lo - self.halo, lo) if self.rank > 0 else None
        above = slice_z(got[self.rank + 1], hi, hi + self.halo) if self.rank + 1 < self.world else None
        return below, above

    def step(self):
        """One time step of the whole domain (vlsg_advect with
        advection_time 0 on every shard), then the halo exchange."""
        lo, hi = self._slab()
        below, above = self._ghosts()
        local = concat_z([below, self.own, above], self.grid, self.width)
        self.engine.upload(local)
        self.engine.set_owned_region(2 if self.world > 1 else -1, lo, hi)
        r = self.engine.advect(self.params)
        out = self.engine.download_domain()
        self.width = out.width
        self.own = slice_z(out, lo, hi)
        self.steps += 1
        self.point_updates += r.point_updates
        self.advected_time += r.advected_time
        if self.rebalance_every and self.steps % self.rebalance_every == 0 and self.world > 1:
            self.rebalance()
        return r

    def rebalance(self):
        """New slab boundaries from the current band (equal point counts)."""
        parts = self.comm.allgather_domains(self.own, self.grid, self.width)
        whole = concat_z(parts, self.grid, self.width)
        self.bounds = partition_z(whole.idx[:, 2], self.world, min_planes=self.halo)
        self.own = slice_z(whole, *self._slab())

    def gather(self):
        """The whole level set (every rank gets it)."""
        if self.world == 1:
            return self.own
        parts = self.comm.allgather_domains(self.own, self.grid, self.width)
        return concat_z(parts, self.grid, self.width)


class ShardEngine:
    """A libvlsgpu context as the engine of one shard: the slab and its ghost
    planes uploaded each step, advected with the owned region and the
    cross-shard reduction set, and downloaded again."""

    def __init__(self, device, precision, grid, velocity):
        from .advect import Context

        self.ctx = Context(device, precision)
        self.grid = grid
        self.ctx.set_grid(grid)
        self.ctx.set_level_set_count(1)
        desc = velocity.descriptor()
        if desc is None:
            self.ctx.set_velocity_callback(velocity)
        else:
            self.ctx.set_velocity(desc)

    def upload(self, dom):
        self.ctx.upload(0, dom)

    def set_owned_region(self, axis, lo, hi):
        self.ctx.set_owned_region(axis, lo, hi)

    def set_reduction_callback(self, fn):
        self.ctx.set_reduction_callback(fn)

    def advect(self, params):
        return self.ctx.advect(params)

    def download_domain(self):
        return self.ctx.download_domain(0, self.grid)
