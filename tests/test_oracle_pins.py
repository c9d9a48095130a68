"""The oracle against the reference's own pins (no GPU).

- TimeIntegration.cpp:177-313: Chamfer distance of an advected sphere to the
  analytic result, for EO1 / WENO3 / WENO5 x FE / RK2 / RK3.
- BooleanOperationExactZero (result.hpp): the golden run list of Box u Plane
  after the boolean operation's Prune passes (2D, reflective x).
- StencilLocalLaxFriedrichs.cpp:33-84: a sphere of radius 1 grown at v = 1
  for t = 0.5 with STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER, Chamfer distance
  to the radius-1.5 sphere < 0.035.
- LSTEST_ASSERT_VALID_LS (lsTestAsserts.hpp:11-23) after every advection.
- MarkVoidPoints.cpp:57-108: a plane at y = 0.35 with two circular holes of
  radius 5.1 centred at (+-8, -9.5) below it (2D, gridDelta 1, reflective x):
  exactly the defined points with y < -2 are voids.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from viennals_b200 import AdvectParams, BoundaryConditionEnum as BC, Domain, Grid
from viennals_b200.domain import make_runs
from viennals_b200.geometry import make_sphere
from viennals_b200.velocity import constant_vector

HERE = os.path.dirname(os.path.abspath(__file__))

# (spatial, temporal, threshold) -- TimeIntegration.cpp:177-313
TIME_INTEGRATION_PINS = [
    (0, 0, 0.08), (0, 1, 0.14), (0, 2, 0.14),
    (10, 0, 0.06), (10, 1, 0.016), (10, 2, 0.016),
    (11, 0, 0.04), (11, 1, 0.008), (11, 2, 0.008),
]


@pytest.fixture(scope="module")
def ti_setup():
    g = Grid([-5, 5, -5, 5, -5, 5], [BC.INFINITE_BOUNDARY] * 3, 0.15)
    start = O.OracleLS(g, make_sphere(g, [0, 0, 0], 1.5))
    ref = O.OracleLS(g, make_sphere(g, [0.5, 0, 0], 1.5))
    return start, ref


@pytest.mark.parametrize("spatial,temporal,threshold", TIME_INTEGRATION_PINS)
def test_time_integration_chamfer(ti_setup, spatial, temporal, threshold):
    start, ref = ti_setup
    ls = start.copy()
    p = AdvectParams.defaults()
    p.spatial_scheme = spatial
    p.temporal_scheme = temporal
    p.advection_time = 0.5
    res = O.advect([ls], p, constant_vector([1.0, 0.0, 0.0]))
    assert res.advected_time == pytest.approx(0.5)
    assert ls.check() == 0
    c = O.chamfer(ref, ls)
    assert c["chamfer"] < threshold


def test_stencil_llf_sphere_chamfer():
    from viennals_b200.velocity import constant_scalar

    g = Grid([-3, 3, -3, 3, -3, 3], [BC.INFINITE_BOUNDARY] * 3, 0.1)
    ls = O.OracleLS(g, make_sphere(g, [0, 0, 0], 1.0))
    ref = O.OracleLS(g, make_sphere(g, [0, 0, 0], 1.5))
    p = AdvectParams.defaults()
    p.spatial_scheme = 9  # STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER
    p.advection_time = 0.5
    res = O.advect([ls], p, constant_scalar(1.0))
    assert res.advected_time == pytest.approx(0.5)
    assert ls.check() == 0
    c = O.chamfer(ref, ls)
    assert c["chamfer"] < 0.035


def test_boolean_exact_zero_golden():
    from fromsurface2d import box_mesh, from_segments, plane_mesh

    g = Grid([-10, 10, -10, 10], [BC.REFLECTIVE_BOUNDARY, BC.INFINITE_BOUNDARY], 1.0, dim=2)

    def dom(pts, sign_fn):
        keys = sorted(pts, key=lambda k: (k[1], k[0]))
        idx = np.array(keys, np.int32)
        vals = np.array([pts[k] for k in keys])
        idx3 = np.concatenate([idx, np.zeros((len(idx), 1), np.int32)], 1)
        rs, sg = make_runs(idx3, lambda x, y, z: sign_fn(x, y), [-10, -12, 0], [10, 12, 0])
        return Domain(g, idx, vals, rs[:, :2], sg, width=2)

    bn, bl = box_mesh([-5, 1], [5, 10])
    box = from_segments(g, bn, bl, remove_boundary_triangles=False)
    pn, pl = plane_mesh(g, [0, 1], [0, 1])
    plane = from_segments(g, pn, pl)
    mask = O.OracleLS(g, dom(box, lambda x, y: np.where((x > -5) & (x < 5) & (y > 1) & (y < 10), -1, 1)))
    substrate = O.OracleLS(g, dom(plane, lambda x, y: np.where(y < 1, -1, 1)))
    substrate.boolean(mask, 1)  # UNION, then Prune(removeStrayZeros) + Prune

    gold = json.load(open(os.path.join(HERE, "golden", "boolean_exact_zero.json")))["runs"]
    di, dv = substrate.points(0)
    mine = {tuple(k): v for k, v in zip(di.tolist(), dv)}
    gdef = {tuple(r["index"]): r["value"] for r in gold if abs(r["value"]) < 1e300}
    assert set(mine) == set(gdef)
    for k, v in gdef.items():
        assert abs(mine[k] - v) < 1e-4, k
    und = [r for r in gold if abs(r["value"]) > 1e300]
    st = np.array([r["index"] for r in und], np.int32)
    st[:, 1] = np.clip(st[:, 1], -1000, 1000)
    got = substrate.values_at(st)
    for r, v in zip(und, got):
        assert abs(v) > 1e300
        assert (v < 0) == (r["value"] < 0), r


def test_mark_void_points_known_answer():
    # MarkVoidPoints.cpp:57-108 (default options; the geometry as a width-2
    # band of its signed distance: material below the plane minus the holes)
    g = Grid([-15, 15, -15, 15], [BC.REFLECTIVE_BOUNDARY, BC.INFINITE_BOUNDARY], 1.0, dim=2)

    def sdf(x, y):
        holes = [5.1 - np.hypot(x - cx, y + 9.5) for cx in (-8.0, 8.0)]
        return np.maximum(np.maximum(y - 0.35, holes[0]), holes[1])

    X, Y = np.meshgrid(np.arange(-15, 16), np.arange(-20, 6), indexing="xy")
    X, Y = X.ravel(), Y.ravel()
    v = sdf(X.astype(float), Y.astype(float))
    keep = np.abs(v) <= 1.0
    idx = np.stack([X[keep], Y[keep]], 1).astype(np.int32)  # y slowest, x fastest
    vals = v[keep]
    idx3 = np.concatenate([idx, np.zeros((len(idx), 1), np.int32)], 1)
    rs, sg = make_runs(idx3, lambda x, y, z: np.where(sdf(np.asarray(x, float),
                                                          np.asarray(y, float)) < 0, -1, 1),
                       [-15, -22, 0], [15, 8, 0])
    ls = O.OracleLS(g, Domain(g, idx, vals, rs[:, :2], sg, width=2))
    pi, _ = ls.points(0)
    marks = ls.void_markers()
    assert len(marks) == len(pi) and marks.any() and not marks.all()
    assert np.array_equal(marks, pi[:, 1] < -2)


def test_two_dimensional_generators_are_valid_level_sets():
    # the 2D inputs of tests/test_gpu_2d.py: makeSphere's rule in 2D (the
    # Advection2D.cpp circle) and a signed-distance band with periodic x; the
    # oracle's Check accepts both, and the circle grows under the
    # LAX_FRIEDRICHS_1ST_ORDER advection of Advection2D.cpp
    from viennals_b200.geometry import make_circle, sdf_levelset_2d
    from viennals_b200.velocity import constant_scalar

    g = Grid([-20, 20, -20, 20], [BC.REFLECTIVE_BOUNDARY, BC.REFLECTIVE_BOUNDARY], 0.5, dim=2)
    c = make_circle(g, [5.0, 0.0], 7.3)
    assert c.idx.shape[1] == 2 and c.run_start.shape[1] == 2
    ls = O.OracleLS(g, c)
    assert ls.check() == 0
    p = AdvectParams.defaults()
    p.spatial_scheme = 2  # LAX_FRIEDRICHS_1ST_ORDER
    p.advection_time = 1.0
    O.advect([ls], p, constant_scalar(1.0))
    assert ls.check() == 0
    assert len(ls.points(0)[1]) > len(c.values)
    g2 = Grid([-20, 20, -20, 20], [BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 1.0, dim=2)
    band = sdf_levelset_2d(g2, lambda x, y: y - 0.3 * x / 20.0, [g2.min[0], -6], [g2.max[0] - 1, 6])
    assert O.OracleLS(g2, band).check() == 0


def test_two_dimensional_runs_cover_every_undefined_cell():
    # make_runs_2d: every undefined cell of the box reads the sign of the last
    # run start at or before it in HRLE order (y slowest, x fastest), and no
    # run repeats its predecessor's sign with no defined point between them
    from viennals_b200.domain import INF_INDEX, make_runs_2d

    # a valid band: two circles' signed distance, defined where |d| <= 1 cell
    # (every sign change along a grid line then passes a defined point)
    lo, hi = [-9, -7], [11, 8]
    cells = [(x, y) for y in range(lo[1], hi[1] + 1) for x in range(lo[0], hi[0] + 1)]

    def sdf(x, y):
        x, y = np.asarray(x, float), np.asarray(y, float)
        return np.minimum(np.hypot(x - 3.2, y + 0.4) - 4.6, np.hypot(x + 5.1, y - 3.3) - 2.2)

    pts = np.array([c for c in cells if abs(sdf(*c)) <= 1.0], np.int64)

    def sign_fn(x, y):
        return np.where(sdf(x, y) < 0, -1, 1)

    rs, sg = make_runs_2d(pts, sign_fn, lo, hi)
    key = lambda x, y: (int(y) + INF_INDEX) * (1 << 22) + (int(x) + INF_INDEX)
    rk = [key(x, y) for x, y in rs]
    assert rk == sorted(rk)
    defined = {tuple(p) for p in pts.tolist()}
    for x, y in cells:
        if (x, y) in defined:
            continue
        j = np.searchsorted(rk, key(x, y), side="right") - 1
        assert j >= 0 and sg[j] == sign_fn(x, y), (x, y)
    pk = sorted(key(x, y) for x, y in defined)
    before = np.searchsorted(pk, rk)
    for i in range(1, len(sg)):
        assert sg[i] != sg[i - 1] or before[i] != before[i - 1]
