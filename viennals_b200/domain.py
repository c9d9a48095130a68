"""Host-side level-set container in the exchange format of vlsg.h.

`Domain` mirrors what the C ABI moves across the boundary for one
viennals::Domain<T,3> (lsDomain.hpp:27-269): the grid (index bounds,
boundary conditions, gridDelta), the defined points with their values in
grid units, the undefined runs (start index, sign) that tile the rest of
the HRLE order, and levelSetWidth.
"""
import math

import numpy as np

from ._abi import BoundaryConditionEnum

# Index that stands for "minus infinity" in run starts; it fits the 21-bit
# per-axis keys the library and the oracle use.
INF_INDEX = (1 << 20) - 2


class Grid:
    """viennahrle::Grid built as Domain(bounds, boundaryConditions, gridDelta)
    does it: index bounds floor(min/dx) .. ceil(max/dx), lsDomain.hpp:68-78."""

    def __init__(self, bounds=None, boundary=None, grid_delta=1.0, dim=3,
                 index_min=None, index_max=None):
        self.dim = dim
        self.delta = float(grid_delta)
        if boundary is None:
            boundary = [BoundaryConditionEnum.INFINITE_BOUNDARY] * dim
        self.bc = [int(b) for b in boundary]
        if index_min is not None:
            self.min = [int(v) for v in index_min]
            self.max = [int(v) for v in index_max]
        elif bounds is not None:
            self.min = [math.floor(bounds[2 * i] / self.delta) for i in range(dim)]
            self.max = [math.ceil(bounds[2 * i + 1] / self.delta) for i in range(dim)]
        else:
            self.min = [0] * dim
            self.max = [0] * dim

    def map_index(self, d, c):
        """Periodic wrap (points min..max-1) / reflective mirror, vectorised."""
        c = np.asarray(c, dtype=np.int64)
        b = self.bc[d]
        lo, hi = self.min[d], self.max[d]
        if b == BoundaryConditionEnum.PERIODIC_BOUNDARY:
            n = hi - lo
            return lo + np.mod(c - lo, n)
        if b == BoundaryConditionEnum.REFLECTIVE_BOUNDARY:
            c = np.where(c < lo, 2 * lo - c, c)
            return np.where(c > hi, 2 * hi - c, c)
        if b == BoundaryConditionEnum.POS_INFINITE_BOUNDARY:
            return np.where(c < lo, 2 * lo - c, c)
        if b == BoundaryConditionEnum.NEG_INFINITE_BOUNDARY:
            return np.where(c > hi, 2 * hi - c, c)
        return c

    def is_periodic(self, d):
        return self.bc[d] == BoundaryConditionEnum.PERIODIC_BOUNDARY


class Domain:
    """Defined points + undefined runs of one level set."""

    def __init__(self, grid, idx=None, values=None, run_start=None,
                 run_sign=None, width=2):
        self.grid = grid
        d = grid.dim
        self.idx = np.zeros((0, d), np.int32) if idx is None else np.ascontiguousarray(idx, np.int32)
        self.values = np.zeros(0) if values is None else np.ascontiguousarray(values, np.float64)
        self.run_start = (np.zeros((0, d), np.int32) if run_start is None
                          else np.ascontiguousarray(run_start, np.int32))
        self.run_sign = (np.zeros(0, np.int8) if run_sign is None
                         else np.ascontiguousarray(run_sign, np.int8))
        self.width = int(width)
        # Domain::getPointData(): scalar arrays per defined point, by label
        self.point_data = {}

    @property
    def n_points(self):
        return len(self.values)

    def copy(self):
        return Domain(self.grid, self.idx.copy(), self.values.copy(),
                      self.run_start.copy(), self.run_sign.copy(), self.width)

    def sorted(self):
        """Points in HRLE order (x fastest, highest dimension slowest)."""
        order = np.lexsort(tuple(self.idx[:, d] for d in range(self.grid.dim)))
        return self.idx[order], self.values[order]

    def active_mask(self, cutoff=0.5):
        return np.abs(self.values) <= cutoff


def lex_order(idx):
    return np.lexsort(tuple(idx[:, d] for d in range(idx.shape[1])))


def make_runs_2d(idx, sign_fn, lo, hi):
    """HRLE-style undefined runs of a D = 2 point set (idx (N,2), sign_fn(x,
    y), lo/hi inclusive (x, y) box holding every defined point): the runs of
    make_runs for the one plane of the box, as (x, y) starts -- the region
    before the box, the rows of the box (heads, gaps, tails, empty rows) and
    the region after it."""
    idx = np.asarray(idx, np.int64).reshape(-1, 2)
    idx3 = np.concatenate([idx, np.zeros((len(idx), 1), np.int64)], 1)
    lo, hi = [int(lo[0]), int(lo[1])], [int(hi[0]), int(hi[1])]
    # make_runs over the plane z = 0 with no z levels outside it
    rs, sg = make_runs(idx3, lambda x, y, z: sign_fn(x, y), [lo[0], lo[1], 0], [hi[0], hi[1], 0],
                       planar=True)
    return np.ascontiguousarray(rs[:, :2]), sg


def make_runs(idx, sign_fn, lo, hi, planar=False):
    """HRLE-style undefined runs for a point set.

    idx: (N,3) defined points; sign_fn(x, y, z) -> array of +1/-1 for the
    undefined cells (vectorised, integer index arrays); lo/hi: inclusive
    index box that contains every defined point.  Emits a run at every start
    of an undefined stretch in HRLE order: row heads, gaps between points of
    a row, row tails, rows without points and the regions outside the box.
    """
    idx = np.asarray(idx, np.int64)
    lo = [int(v) for v in lo]
    hi = [int(v) for v in hi]
    ny = hi[1] - lo[1] + 1
    nz = hi[2] - lo[2] + 1
    order = lex_order(idx)
    p = idx[order]
    ev = []  # (x, y, z) arrays of event starts + cells to evaluate the sign at

    def add(xs, ys, zs, ex, ey, ez):
        ev.append((np.asarray(xs, np.int64), np.asarray(ys, np.int64),
                   np.asarray(zs, np.int64), np.asarray(ex, np.int64),
                   np.asarray(ey, np.int64), np.asarray(ez, np.int64)))

    cx = (lo[0] + hi[0]) // 2
    cy = (lo[1] + hi[1]) // 2
    NI = -INF_INDEX
    # region before the box (z < lo.z) and after it (z > hi.z); a planar
    # (D = 2) box has no z levels outside its plane
    if not planar:
        add([NI], [NI], [NI], [cx], [cy], [lo[2] - 1])
        add([NI], [NI], [hi[2] + 1], [cx], [cy], [hi[2] + 1])
    zs = np.arange(lo[2], hi[2] + 1)
    # rows before / after the box inside each plane
    add(np.full(nz, NI), np.full(nz, NI), zs, np.full(nz, cx), np.full(nz, lo[1] - 1), zs)
    add(np.full(nz, NI), np.full(nz, hi[1] + 1), zs, np.full(nz, cx), np.full(nz, hi[1] + 1), zs)
    # rows of the box
    if len(p):
        row = (p[:, 2] - lo[2]) * ny + (p[:, 1] - lo[1])
    else:
        row = np.zeros(0, np.int64)
    has = np.zeros(ny * nz, bool)
    has[row] = True
    empty = np.nonzero(~has)[0]
    ey_, ez_ = lo[1] + empty % ny, lo[2] + empty // ny
    add(np.full(len(empty), NI), ey_, ez_, np.full(len(empty), lo[0]), ey_, ez_)
    if len(p):
        first = np.ones(len(p), bool)
        first[1:] = row[1:] != row[:-1]
        last = np.ones(len(p), bool)
        last[:-1] = row[1:] != row[:-1]
        # head of each occupied row
        f = np.nonzero(first)[0]
        add(np.full(len(f), NI), p[f, 1], p[f, 2], p[f, 0] - 1, p[f, 1], p[f, 2])
        # gaps between consecutive points of a row, and the row tails
        gap = np.zeros(len(p), bool)
        gap[:-1] = (~last[:-1]) & (p[1:, 0] > p[:-1, 0] + 1)
        g = np.nonzero(gap | last)[0]
        add(p[g, 0] + 1, p[g, 1], p[g, 2], p[g, 0] + 1, p[g, 1], p[g, 2])
    xs = np.concatenate([e[0] for e in ev])
    ys = np.concatenate([e[1] for e in ev])
    zs_ = np.concatenate([e[2] for e in ev])
    sg = np.asarray(sign_fn(np.concatenate([e[3] for e in ev]),
                            np.concatenate([e[4] for e in ev]),
                            np.concatenate([e[5] for e in ev])), np.int64)
    o = np.lexsort((xs, ys, zs_))
    start = np.stack([xs[o], ys[o], zs_[o]], axis=1).astype(np.int32)
    sign = np.where(sg[o] < 0, -1, 1).astype(np.int8)
    # drop runs that repeat the previous sign with no defined point between
    if len(start) > 1:
        keys = (start[:, 2].astype(np.int64) << 42) + (start[:, 1].astype(np.int64) << 21) + start[:, 0]
        pk = ((p[:, 2] + (1 << 20)) << 42) + ((p[:, 1] + (1 << 20)) << 21) + (p[:, 0] + (1 << 20)) if len(p) else np.zeros(0, np.int64)
        kk = ((start[:, 2].astype(np.int64) + (1 << 20)) << 42) + ((start[:, 1].astype(np.int64) + (1 << 20)) << 21) + (start[:, 0].astype(np.int64) + (1 << 20))
        del keys
        npts_before = np.searchsorted(pk, kk)
        keep = np.ones(len(start), bool)
        keep[1:] = (sign[1:] != sign[:-1]) | (npts_before[1:] != npts_before[:-1])
        start, sign = start[keep], sign[keep]
    return start, sign
