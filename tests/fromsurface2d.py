"""2D restatement of FromSurfaceMesh for line meshes (test input generator).

Follows lsFromSurfaceMesh.hpp:100-145 (gridline/segment intersection) and
:270-480 (distances along grid lines, clamped to +-1 with the 1e-7 shrink,
the smallest signed distance per point).  Used to rebuild the inputs of the
reference's BooleanOperationExactZero test (a box and a plane built by
MakeGeometry::makeBox / makePlane, lsMakeGeometry.hpp:245-419).
"""
import math

import numpy as np

from viennals_b200._abi import BoundaryConditionEnum as BC

# Index bound HRLE gives an INFINITE_BOUNDARY direction (the golden fixture's
# first run starts at -715827882 = -(2^31-1)/3).
HRLE_INFINITE_INDEX = 715827882
BOUNDARY_EPS = 1e-5
DISTANCE_EPS = 1e-4
SIGN_EPS = 1e-6


def _intersect(point, c, d):
    """calculateGridlineTriangleIntersection, 2D (lsFromSurfaceMesh.hpp:106-145)."""
    inside_pos = inside_neg = True
    dA = (d + 1) % 2
    A = [0.0, 0.0]
    for k in range(2):
        A[k] = c[(k + 1) % 2][dA] - point[dA]
        if k == d:
            A[k] = -A[k]
        if A[k] < 0:
            inside_pos = False
        if A[k] > 0:
            inside_neg = False
    if (not inside_pos and inside_neg) or (inside_pos and not inside_neg):
        s = A[0] + A[1]
        k = 0
        if inside_pos:
            if A[1] > A[0]:
                k = 1
        else:
            if A[1] < A[0]:
                k = 1
        inter = c[k][d] + (c[(k + 1) % 2][d] - c[k][d]) * (A[(k + 1) % 2] / s)
        return (1 if inside_pos else -1), inter
    return 0, None


def from_segments(grid, nodes, lines, remove_boundary_triangles=True):
    """Point list {index: value} of FromSurfaceMesh for a 2D line mesh."""
    gd = grid.delta
    D = 2
    gmin_idx = [-HRLE_INFINITE_INDEX if grid.bc[i] == BC.INFINITE_BOUNDARY else grid.min[i] for i in range(D)]
    gmax_idx = [HRLE_INFINITE_INDEX if grid.bc[i] == BC.INFINITE_BOUNDARY else grid.max[i] for i in range(D)]
    remove = [not (not remove_boundary_triangles and grid.is_periodic(i)) for i in range(D)]
    gmin = [gmin_idx[i] * gd for i in range(D)]
    gmax = [gmax_idx[i] * gd for i in range(D)]

    def max_grid_point(i):
        return gmax_idx[i] - 1 if grid.is_periodic(i) else gmax_idx[i]

    pts = {}
    for el in lines:
        c = [[float(nodes[el[q]][dim]) for dim in range(D)] for q in range(D)]
        center = [0.0, 0.0]
        flags = [True] * (2 * D)
        remove_el = False
        for dim in range(D):
            for q in range(D):
                if abs(c[q][dim] - gmin[dim]) < BOUNDARY_EPS * gd:
                    c[q][dim] = gmin[dim]
                if abs(c[q][dim] - gmax[dim]) < BOUNDARY_EPS * gd:
                    c[q][dim] = gmax[dim]
                if c[q][dim] > gmin[dim]:
                    flags[dim] = False
                if c[q][dim] < gmax[dim]:
                    flags[dim + D] = False
                center[dim] += c[q][dim]
            if remove[dim] and (flags[dim] or flags[dim + D]):
                remove_el = True
        if remove_el:
            continue
        center = [v / D for v in center]
        min_node = [min(c[0][i], c[1][i]) for i in range(D)]
        max_node = [max(c[0][i], c[1][i]) for i in range(D)]
        min_idx = [int(math.ceil(min_node[q] / gd)) for q in range(D)]
        max_idx = [int(math.floor(max_node[q] / gd)) for q in range(D)]
        for i in range(D):
            if remove[i]:
                min_idx[i] = max(min_idx[i], gmin_idx[i])
                max_idx[i] = min(max_idx[i], max_grid_point(i))
        for z in range(D):
            o = (z + 1) % D
            if min_idx[o] > max_idx[o]:
                continue
            for it in range(min_idx[o], max_idx[o] + 1):
                p = [0.0, 0.0]
                p[o] = it * gd
                status, inter = _intersect(p, c, z)
                if status == 0:
                    continue
                if remove[z] and inter > gd * gmax_idx[z]:
                    continue
                if remove[z] and inter < gmin_idx[z] * gd:
                    continue
                inter2 = inter / gd
                lo = int(math.floor(inter2 - DISTANCE_EPS))
                hi = int(math.ceil(inter2 + DISTANCE_EPS))
                lo = max(lo, min_idx[z] - 1)
                hi = min(hi, max_idx[z] + 1)
                lo = max(lo, gmin_idx[z])
                hi = min(hi, gmax_idx[z])
                t = [center[0], center[1]]
                t[z] -= inter
                t[o] -= p[o]
                nrm = math.sqrt(t[0] ** 2 + t[1] ** 2)
                # Normalize of a zero vector gives NaN in the reference
                t = [t[0] / nrm, t[1] / nrm] if nrm > 0 else [math.nan, math.nan]
                for iz in range(lo, hi + 1):
                    real = iz - inter2
                    sign_d = real - SIGN_EPS * t[z]
                    if status < 0:
                        real, sign_d = -real, -sign_d
                    if real < 0.0:
                        sign_d = -sign_d
                    real *= (1.0 - DISTANCE_EPS * 1e-3)
                    real = max(-1.0, min(1.0, real))
                    if real == 0.0:
                        real = 0.0
                    idx = [0, 0]
                    idx[z] = iz
                    idx[o] = it
                    key = tuple(int(grid.map_index(d, idx[d])) for d in range(D))
                    cur = pts.get(key)
                    if cur is None or (sign_d, real) < cur:
                        pts[key] = (sign_d, real)
    return {k: v[1] for k, v in pts.items()}


def box_mesh(lo, hi):
    """makeBox's 2D line loop, lsMakeGeometry.hpp:363-419."""
    c0 = [lo[0], lo[1]]
    c3 = [hi[0], hi[1]]
    c1 = [hi[0], lo[1]]
    c2 = [lo[0], hi[1]]
    return [c0, c1, c2, c3], [(0, 2), (2, 3), (3, 1), (1, 0)]


def plane_mesh(grid, origin, normal):
    """makePlane's 2D segment, lsMakeGeometry.hpp:245-360."""
    m = math.sqrt(sum(v * v for v in normal))
    n = [v / m for v in normal]
    i = [d for d in range(2) if grid.bc[d] == BC.INFINITE_BOUNDARY][0]
    j = (i + 1) % 2
    gd = grid.delta
    min_c = gd * (grid.min[j] - 1)
    max_c = gd * (grid.max[j] + 1)
    pts = []
    for cj in (min_c, max_c):
        num = (cj - origin[j]) * n[j]
        p = [0.0, 0.0]
        p[j] = cj
        p[i] = origin[i] - num / n[i]
        pts.append(p)
    line = (0, 1) if n[i] >= 0 else (1, 0)
    return pts, [line]
