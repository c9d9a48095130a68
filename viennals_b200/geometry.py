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

from .domain import Domain, make_runs


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
