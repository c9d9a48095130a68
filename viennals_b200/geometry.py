"""Synthetic level sets for tests and benchmarks.

These generate inputs; they are not part of the advection path.  The sphere
restates MakeGeometry::makeSphere (lsMakeGeometry.hpp:177-241): for every
index in the box around the sphere the value is the shortest distance along a
grid line to the sphere, kept when |d| <= gridDelta + 1e-5, stored as
d / gridDelta (width 2).  Undefined runs carry the geometric inside/outside
sign, which is what HRLE's FillDomainWithSignedDistance gives a valid width-2
band.
"""
import numpy as np

from .domain import Domain, make_runs, make_runs_2d


def _box_points(lo, hi):
    xs = np.arange(lo[0], hi[0] + 1, dtype=np.int64)
    ys = np.arange(lo[1], hi[1] + 1, dtype=np.int64)
    zs = np.arange(lo[2], hi[2] + 1, dtype=np.int64)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def sphere_distance(X, Y, Z, origin, radius, gd):
    """makeSphere's distance rule, lsMakeGeometry.hpp:199-213."""
    idx = (X, Y, Z)
    r2 = radius * radius
    distance = np.full(X.shape, np.finfo(np.float64).max)
    for i in range(3):
        y = idx[(i + 1) % 3] * gd - origin[(i + 1) % 3]
        z = idx[(i + 2) % 3] * gd - origin[(i + 2) % 3]
        x = r2 - y * y - z * z
        ok = ~(x < 0.0)
        with np.errstate(invalid="ignore"):
            dir_radius = np.abs(idx[i] * gd - origin[i]) - np.sqrt(np.where(ok, x, 0.0))
        upd = ok & (np.abs(dir_radius) < np.abs(distance))
        distance = np.where(upd, dir_radius, distance)
    return distance


def make_circle(grid, origin, radius):
    """makeSphere for D = 2 (lsMakeGeometry.hpp:177-241 with D = 2): the
    distance along the two grid lines through each index of the box around
    the circle, kept when |d| <= gridDelta + 1e-5, width 2."""
    gd = grid.delta
    ox, oy = float(origin[0]), float(origin[1])
    lo = [int((ox - radius) / gd - 1), int((oy - radius) / gd - 1)]
    hi = [int((ox + radius) / gd + 1), int((oy + radius) / gd + 1)]
    ys, xs = np.meshgrid(np.arange(lo[1], hi[1] + 1), np.arange(lo[0], hi[0] + 1), indexing="ij")
    X, Y = xs.ravel(), ys.ravel()
    last = (X == hi[0]) & (Y == hi[1])
    r2 = radius * radius
    idx = (X, Y)
    org = (ox, oy)
    distance = np.full(X.shape, np.finfo(np.float64).max)
    for i in range(2):
        y = idx[(i + 1) % 2] * gd - org[(i + 1) % 2]
        x = r2 - y * y
        ok = ~(x < 0.0)
        with np.errstate(invalid="ignore"):
            dir_radius = np.abs(idx[i] * gd - org[i]) - np.sqrt(np.where(ok, x, 0.0))
        upd = ok & (np.abs(dir_radius) < np.abs(distance))
        distance = np.where(upd, dir_radius, distance)
    keep = (np.abs(distance) <= 2.0 * 0.5 * gd + 1e-5) & ~last
    pts = np.stack([X[keep], Y[keep]], axis=1)
    vals = distance[keep] / gd
    for d in range(2):
        if grid.is_periodic(d):
            pts[:, d] = grid.map_index(d, pts[:, d])
    o = np.lexsort((pts[:, 0], pts[:, 1]))
    pts, vals = pts[o], vals[o]

    def sign_fn(x, y):
        dx = np.asarray(x) * gd - ox
        dy = np.asarray(y) * gd - oy
        return np.where(dx * dx + dy * dy < r2, -1, 1)

    rs, sg = make_runs_2d(pts, sign_fn, [lo[0] - 1, lo[1] - 1], [hi[0] + 1, hi[1] + 1])
    return Domain(grid, pts.astype(np.int32), vals, rs, sg, width=2)


def sdf_levelset_2d(grid, sdf, lo, hi, half_width=1.0):
    """Band of a 2D signed distance function (physical units) over the index
    box [lo, hi]: every index with |sdf| <= half_width * gridDelta, value
    sdf / gridDelta, undefined runs with the sign of sdf."""
    gd = grid.delta
    ys, xs = np.meshgrid(np.arange(lo[1], hi[1] + 1), np.arange(lo[0], hi[0] + 1), indexing="ij")
    X, Y = xs.ravel(), ys.ravel()
    v = sdf(X * gd, Y * gd) / gd
    keep = np.abs(v) <= half_width
    pts = np.stack([X[keep], Y[keep]], axis=1)
    vals = v[keep]
    for d in range(2):
        if grid.is_periodic(d):
            pts[:, d] = grid.map_index(d, pts[:, d])
    key = pts[:, 1].astype(np.int64) * (1 << 21) + pts[:, 0]
    _, first = np.unique(key, return_index=True)
    pts, vals = pts[first], vals[first]

    def sign_fn(x, y):
        return np.where(sdf(np.asarray(x) * gd, np.asarray(y) * gd) < 0, -1, 1)

    rs, sg = make_runs_2d(pts, sign_fn, [lo[0] - 1, lo[1] - 1], [hi[0] + 1, hi[1] + 1])
    return Domain(grid, pts.astype(np.int32), vals, rs, sg, width=int(round(2 * half_width)))


def make_sphere(grid, origin, radius):
    gd = grid.delta
    origin = [float(o) for o in origin] + [0.0] * (3 - len(origin))
    # C++ double -> int conversion truncates toward zero
    lo = [int((origin[i] - radius) / gd - 1) for i in range(3)]
    hi = [int((origin[i] + radius) / gd + 1) for i in range(3)]
    X, Y, Z = _box_points(lo, hi)
    # the generator loop stops before reaching endIndex itself
    last = (X == hi[0]) & (Y == hi[1]) & (Z == hi[2])
    dist = sphere_distance(X, Y, Z, origin, radius, gd)
    value_limit = 2.0 * 0.5 * gd + 1e-5
    keep = (np.abs(dist) <= value_limit) & ~last
    idx = np.stack([X[keep], Y[keep], Z[keep]], axis=1)
    vals = dist[keep] / gd
    for d in range(3):
        if grid.is_periodic(d):
            idx[:, d] = grid.map_index(d, idx[:, d])

    def sign_fn(x, y, z):
        dx = x * gd - origin[0]
        dy = y * gd - origin[1]
        dz = z * gd - origin[2]
        return np.where(dx * dx + dy * dy + dz * dz < radius * radius, -1, 1)

    rs, sg = make_runs(idx, sign_fn, [lo[0] - 1, lo[1] - 1, lo[2] - 1],
                       [hi[0] + 1, hi[1] + 1, hi[2] + 1])
    return Domain(grid, idx.astype(np.int32), vals, rs, sg, width=2)


def sdf_levelset(grid, sdf, lo, hi, lipschitz=1.0, half_width=1.0):
    """Band of a signed distance function (physical units), width 2 by default.

    Every cell of the index box [lo, hi] with |sdf| <= half_width * gridDelta
    is defined with value sdf / gridDelta (the level set's width is
    2 * half_width); undefined runs carry the sign of sdf.  Bricks of 8^3
    cells whose centre is further than their half diagonal (times
    `lipschitz`) plus half_width + 0.5 cells from the surface are skipped
    unevaluated.  sdf(x, y, z) takes float arrays of coordinates.
    """
    gd = grid.delta
    lo = [int(v) for v in lo]
    hi = [int(v) for v in hi]
    B = 8
    nb = [(hi[d] - lo[d]) // B + 1 for d in range(3)]
    bz, by, bx = np.meshgrid(np.arange(nb[2]), np.arange(nb[1]), np.arange(nb[0]), indexing="ij")
    cx = (lo[0] + bx * B + 3.5) * gd
    cy = (lo[1] + by * B + 3.5) * gd
    cz = (lo[2] + bz * B + 3.5) * gd
    dc = sdf(cx.ravel(), cy.ravel(), cz.ravel())
    reach = (np.sqrt(3.0) * 4.0 * lipschitz + half_width + 0.5) * gd
    near = np.nonzero(np.abs(dc) <= reach)[0]
    off = np.arange(B)
    oz, oy, ox = np.meshgrid(off, off, off, indexing="ij")
    ox, oy, oz = ox.ravel(), oy.ravel(), oz.ravel()
    idx_parts, val_parts = [], []
    chunk = 1 << 14
    for s in range(0, len(near), chunk):
        nbk = near[s:s + chunk]
        X = (lo[0] + bx.ravel()[nbk, None] * B + ox[None, :]).ravel()
        Y = (lo[1] + by.ravel()[nbk, None] * B + oy[None, :]).ravel()
        Z = (lo[2] + bz.ravel()[nbk, None] * B + oz[None, :]).ravel()
        inside = (X <= hi[0]) & (Y <= hi[1]) & (Z <= hi[2])
        X, Y, Z = X[inside], Y[inside], Z[inside]
        v = sdf(X * gd, Y * gd, Z * gd) / gd
        keep = np.abs(v) <= half_width
        idx_parts.append(np.stack([X[keep], Y[keep], Z[keep]], 1))
        val_parts.append(v[keep])
    idx = np.concatenate(idx_parts) if idx_parts else np.zeros((0, 3), np.int64)
    vals = np.concatenate(val_parts) if val_parts else np.zeros(0)
    for d in range(3):
        if grid.is_periodic(d):
            idx[:, d] = grid.map_index(d, idx[:, d])
    if len(idx):
        key = (idx[:, 2].astype(np.int64) << 42) + (idx[:, 1].astype(np.int64) << 21) + idx[:, 0]
        _, first = np.unique(key, return_index=True)
        idx, vals = idx[first], vals[first]

    def sign_fn(x, y, z):
        return np.where(sdf(np.asarray(x) * gd, np.asarray(y) * gd, np.asarray(z) * gd) < 0, -1, 1)

    rs, sg = make_runs(idx, sign_fn, [lo[0] - 1, lo[1] - 1, lo[2] - 1], [hi[0] + 1, hi[1] + 1, hi[2] + 1])
    return Domain(grid, idx.astype(np.int32), vals, rs, sg, width=int(round(2 * half_width)))


# signed distance helpers (physical units) ----------------------------------
def sdf_box(p, lo, hi):
    q = [np.maximum(lo[d] - p[d], p[d] - hi[d]) for d in range(3)]
    outside = np.sqrt(sum(np.maximum(qd, 0.0) ** 2 for qd in q))
    inside = np.minimum(np.maximum(np.maximum(q[0], q[1]), q[2]), 0.0)
    return outside + inside


def trench_etch_level_sets(grid, mask_thickness=0.5, opening=4.0):
    """Mask (material 0) and substrate-wrapping top (material 1) of a square
    trench etch: substrate below z = 0, a mask slab 0 < z < thickness with a
    centred square opening of the given width (periodic in x/y)."""
    h = opening / 2.0
    big = 1e9

    def mask(x, y, z):
        slab = np.maximum(-z, z - mask_thickness)
        hole = sdf_box((x, y, z), (-h, -h, -big), (h, h, big))
        return np.maximum(slab, -hole)

    def top(x, y, z):
        return np.minimum(z, mask(x, y, z))

    lo = [grid.min[0], grid.min[1], grid.min[2]]
    hi = [grid.max[0] - 1, grid.max[1] - 1, grid.max[2]]
    return sdf_levelset(grid, mask, lo, hi), sdf_levelset(grid, top, lo, hi)
