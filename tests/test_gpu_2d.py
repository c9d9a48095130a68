"""Advect<double,2> on the GPU (D = 2 held as the plane of a z-periodic grid
of period 1) against the oracle's 2D path: the same defined points, bit-
identical values, the same getters, and the undefined runs of the device's
exchange format equal to the host builder's for the same points.  The cases
follow the reference's 2D tests: a circle grown with reflective boundaries
(tests/Advection2D/Advection2D.cpp: LAX_FRIEDRICHS_1ST_ORDER, v = 1) and a
plane with a pillar moved by a vector velocity across a periodic boundary
(tests/PeriodicBoundary2D/PeriodicBoundary2D.cpp: v = (1, 0), single steps);
every scheme, the integration schemes, host velocity and alpha fields (asked
at the plane only), two materials and the FP32 form."""
import numpy as np
import pytest

from parity_cases import params
from viennals_b200 import BoundaryConditionEnum as BC, Grid
from viennals_b200.advect import Context
from viennals_b200.geometry import make_circle, sdf_levelset_2d
from viennals_b200.velocity import FunctorVelocity, VelocityField, constant_scalar, constant_vector

pytestmark = pytest.mark.gpu


def _oracle(grid, doms, vel, p, steps=1):
    from oracle import oracle as O

    ols = [O.OracleLS(grid, d) for d in doms]
    res = [O.advect(ols, p, vel) for _ in range(steps)]
    return ols, res


def _gpu(grid, doms, vel, p, steps=1, precision=0):
    ctx = Context(0, precision)
    ctx.set_grid(grid)
    ctx.set_level_set_count(len(doms))
    for i, d in enumerate(doms):
        ctx.upload(i, d)
    desc = vel.descriptor()
    if desc is None:
        ctx.set_velocity_callback(vel)
    else:
        ctx.set_velocity(desc)
    res = [ctx.advect(p) for _ in range(steps)]
    return ctx, res


def _same(grid, doms, vel, p, steps=1):
    ols, ores = _oracle(grid, doms, vel, p, steps)
    ctx, gres = _gpu(grid, doms, vel, p, steps)
    for a, b in zip(ores, gres):
        assert a.number_of_time_steps == b.number_of_time_steps
        assert a.advected_time == b.advected_time
        assert a.current_time_step == b.current_time_step
    for i, o in enumerate(ols):
        oi, ov = o.points(0)
        gi, gv, _ = ctx.download(i)
        assert gi.shape[1] == 2
        assert np.array_equal(oi, gi), i
        assert np.array_equal(ov.view(np.int64), gv.view(np.int64)), i
        dev = ctx.download_domain(i, grid)
        host = ctx.download_domain_host_runs(i, grid)
        assert np.array_equal(dev.run_start, host.run_start)
        assert np.array_equal(dev.run_sign, host.run_sign)
        assert o.check() == 0
    ctx.close()
    return ols


def _circle_case(bc=BC.REFLECTIVE_BOUNDARY):
    g = Grid([-20, 20, -20, 20], [bc, bc], 0.5, dim=2)
    return g, make_circle(g, [5.0, 0.0], 7.3)


def test_circle_growth_lax_friedrichs():
    # Advection2D.cpp: LAX_FRIEDRICHS_1ST_ORDER, v = 1 (t 20 there, 2 here)
    g, c = _circle_case()
    ols = _same(g, [c], constant_scalar(1.0), params(2, 0, 2.0))
    _, v = ols[0].points(0)
    assert len(v) > len(c.values)


@pytest.mark.parametrize("spatial,temporal", [(0, 0), (1, 1), (2, 1), (3, 0), (5, 2), (6, 1),
                                              (7, 2), (8, 0), (10, 1), (11, 2)])
def test_schemes(spatial, temporal):
    g, c = _circle_case()
    v = FunctorVelocity(1)
    v.set_rate(0, 0.8)
    v.set_linear(0, 1, 0.3)
    _same(g, [c], v, params(spatial, temporal, 0.9, cfl=0.4))


def test_periodic_plane_with_pillar_vector_velocity():
    # PeriodicBoundary2D.cpp: periodic x, infinite y; plane y = 0 united with
    # the box [5, 15] x [-1, 10]; v = (1, 0); single steps
    g = Grid([-20, 20, -20, 20], [BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 1.0, dim=2)

    def sdf(x, y):
        box = np.maximum(np.maximum(5.0 - x, x - 15.0), np.maximum(-1.0 - y, y - 10.0))
        return np.minimum(y, box)

    dom = sdf_levelset_2d(g, sdf, [g.min[0], -8], [g.max[0] - 1, 16])
    _same(g, [dom], constant_vector([1.0, 0.0, 0.0]), params(0, 0, 0.0), steps=12)


class _HostField(VelocityField):
    """A host velocity field of the coordinate and the normal."""

    def __init__(self):
        self.max_abs_z = 0.0

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        self.max_abs_z = max(self.max_abs_z, float(np.max(np.abs(coords[:, 2]), initial=0.0)),
                             float(np.max(np.abs(normals[:, 2]), initial=0.0)))
        scalar_out[:] = 0.5 + 0.02 * coords[:, 0] + 0.3 * normals[:, 1]
        vector_out[:] = 0.0


@pytest.mark.parametrize("spatial", [0, 7])
def test_host_velocity_field(spatial):
    g, c = _circle_case(BC.INFINITE_BOUNDARY)
    f = _HostField()
    _same(g, [c], f, params(spatial, 1, 0.7, cfl=0.4))
    assert f.max_abs_z == 0.0  # coordinates and normals of the plane


def test_two_materials():
    # a substrate below y = 0 under a mask slab with an opening (2D trench)
    g = Grid([-6, 6, -6, 6], [BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 0.2, dim=2)

    def substrate(x, y):
        return y

    def top(x, y):
        slab = np.maximum(y - 0.6, -y)
        opening = 1.5 - np.abs(x)
        return np.minimum(y, np.maximum(slab, opening))

    lo, hi = [g.min[0], -12], [g.max[0] - 1, 12]
    m = sdf_levelset_2d(g, substrate, lo, hi)
    t = sdf_levelset_2d(g, top, lo, hi)
    v = FunctorVelocity(2)
    v.set_rate(1, -1.0)
    v.set_linear(1, 1, -0.3)
    _same(g, [m, t], v, params(8, 2, 0.3))


def test_fp32_matches_fp64_points():
    g, c = _circle_case()
    p = params(11, 2, 1.5, cfl=0.4)
    c64, _ = _gpu(g, [c], constant_scalar(1.0), p, precision=0)
    c32, _ = _gpu(g, [c], constant_scalar(1.0), p, precision=1)
    i64, v64, _ = c64.download(0)
    i32, v32, _ = c32.download(0)
    assert np.array_equal(i64, i32)
    assert np.max(np.abs(v64 - v32)) < 1e-5
    c64.close()
    c32.close()


class _AlphaCallback(FunctorVelocity):
    """The functor's velocity and alphas through the host callbacks; records
    the directions the alpha callback is asked for."""

    def __init__(self, n):
        super().__init__(n)
        self.directions = set()

    def descriptor(self):
        return None

    def alpha_batch(self, directions, materials, central_differences, alpha_out):
        self.directions.update(int(d) for d in np.unique(directions))
        super().alpha_batch(directions, materials, central_differences, alpha_out)


@pytest.mark.parametrize("host", [False, True], ids=["functor", "callback"])
def test_llf_analytical(host):
    # LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER: the user's alphas of the 3x3
    # box in x and y (the z direction is never asked)
    g, c = _circle_case()
    v = _AlphaCallback(1) if host else FunctorVelocity(1)
    v.set_rate(0, 1.0)
    v.set_square(0, 0, 1.6, 0.4)
    v.set_dissipation_alpha(0, 0, 1.6)
    v.set_dissipation_alpha(0, 1, 1.0)
    v.set_dissipation_alpha(0, 2, 7.0)  # never asked in 2D: must not bound the step
    _same(g, [c], v, params(4, 2, 0.8, cfl=0.4))
    if host:
        assert v.directions == {0, 1}


class _CountingField(VelocityField):
    """A host velocity field of the normal; records the largest |z| of the
    coordinates and normals it is asked at."""

    def __init__(self):
        self.max_abs_z = 0.0

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        self.max_abs_z = max(self.max_abs_z, float(np.max(np.abs(coords[:, 2]), initial=0.0)),
                             float(np.max(np.abs(normals[:, 2]), initial=0.0)))
        scalar_out[:] = 1.0 + 0.4 * normals[:, 0] * normals[:, 0]
        vector_out[:] = 0.0


@pytest.mark.parametrize("host", [False, True], ids=["functor", "callback"])
def test_stencil_llf(host):
    # StencilLocalLaxFriedrichsScalar in 2D: the plane's 3x3 stencil and the
    # normal nudged in x and y; a host field is asked at the plane only
    g, c = _circle_case()
    if host:
        v = _CountingField()
    else:
        v = FunctorVelocity(1)
        v.set_rate(0, 1.0)
        v.set_square(0, 0, 0.4, 0.4)
    _same(g, [c], v, params(9, 0, 0.6, cfl=0.4))
    if host:
        assert v.max_abs_z == 0.0


@pytest.mark.parametrize("spatial", [7, 8])
def test_llf_box_sites_on_the_plane(spatial):
    # LocalLaxFriedrichs asks its box sites: in 2D the plane's 9, at z = 0
    g, c = _circle_case()
    f = _CountingField()
    _same(g, [c], f, params(spatial, 1, 0.5, cfl=0.4))
    assert f.max_abs_z == 0.0


def test_three_dimensional_only_forms_reject_2d_grids():
    # the batching form and owned z slabs (sharding) are three-dimensional
    from viennals_b200.advect import BatchContext

    g, c = _circle_case()
    b = BatchContext(0, 1)
    with pytest.raises(RuntimeError, match="three-dimensional"):
        b.set_domains([(g, c, constant_scalar(1.0))])
    b.close()
    ctx = Context(0, 0)
    ctx.set_grid(g)
    with pytest.raises(RuntimeError, match="D = 2"):
        ctx.set_owned_region(2, 0, 4)
    ctx.close()


class _Stateful(VelocityField):
    """A velocity that depends on what the velocity update callback saw."""

    def __init__(self):
        self.k = 0
        self.seen = []
        self.columns = set()

    def update(self, dom):
        self.columns.add(dom.idx.shape[1])
        self.seen.append((len(dom.values), float(np.sum(dom.values))))
        self.k = len(dom.values)
        return True

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        scalar_out[:] = 0.6 + 0.2 * normals[:, 1] + 1e-5 * self.k
        vector_out[:] = 0.0


def test_velocity_update_callback():
    # setVelocityUpdateCallback between the RK3 stages: the callback gets the
    # 2D top level set (two indices per point) and the result matches the
    # oracle's 2D path
    from oracle import oracle as O

    g, c = _circle_case()
    p = params(7, 2, 0.5, cfl=0.4)
    vo, vg = _Stateful(), _Stateful()
    ols = [O.OracleLS(g, c)]
    O.advect(ols, p, vo, update=vo.update)
    ctx = Context(0, 0)
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, c)
    ctx.set_velocity_callback(vg)
    ctx.set_velocity_update_callback(vg.update)
    ctx.advect(p)
    oi, ov = ols[0].points(0)
    gi, gv, _ = ctx.download(0)
    ctx.close()
    assert np.array_equal(oi, gi)
    assert np.array_equal(ov.view(np.int64), gv.view(np.int64))
    assert vo.seen == vg.seen and len(vg.seen) > 0
    assert vg.columns == {2}
