"""The exchange format built on the device (points in HRLE order and the
undefined runs, vlsg_download_levelset / vlsg_download_runs) against the
host builder of the same layout (make_runs over point queries), and the
upload -> download round trip through it."""
import numpy as np
import pytest

from parity_cases import sphere_growth_eo1, egg_velocity, params, run_gpu, sphere_case, trench_case
from viennals_b200 import BoundaryConditionEnum as BC, Grid

pytestmark = pytest.mark.gpu


def _check_runs(ctx, grid, slot=0):
    dev = ctx.download_domain(slot, grid)
    host = ctx.download_domain_host_runs(slot, grid)
    assert np.array_equal(dev.idx, host.idx)
    assert np.array_equal(dev.values, host.values)
    assert np.array_equal(dev.run_start, host.run_start)
    assert np.array_equal(dev.run_sign, host.run_sign)
    return dev


def test_runs_sphere_after_advect():
    g, lss, v, p = sphere_growth_eo1()
    ctx, _ = run_gpu(g, lss, v, p)
    dev = _check_runs(ctx, g)
    assert len(dev.run_sign) > 0 and len(dev.values) > 0


@pytest.mark.parametrize("precision", [0, 1])
def test_runs_egg_weno5(precision):
    g, lss = sphere_case(4.0, 0.3)
    ctx, _ = run_gpu(g, lss, egg_velocity(), params(11, 2, 0.6), precision=precision)
    _check_runs(ctx, g)


def test_runs_periodic_two_materials():
    g, lss, v, p = trench_case(8, 2, 0.2)
    ctx, _ = run_gpu(g, lss, v, p)
    for slot in range(2):
        _check_runs(ctx, g, slot)


def test_runs_reflective_plane():
    from viennals_b200.geometry import sdf_levelset
    from viennals_b200.velocity import constant_scalar

    g = Grid([-3, 3, -3, 3, -4, 4],
             [BC.REFLECTIVE_BOUNDARY, BC.REFLECTIVE_BOUNDARY, BC.INFINITE_BOUNDARY], 0.25)
    n = np.array([0.3, 0.2, 1.0])
    n /= np.linalg.norm(n)
    plane = sdf_levelset(g, lambda x, y, z: n[0] * x + n[1] * y + n[2] * z,
                         [g.min[0], g.min[1], -20], [g.max[0], g.max[1], 20])
    ctx, _ = run_gpu(g, [plane], constant_scalar(-1.0), params(1, 1, 0.5))
    _check_runs(ctx, g)


def test_runs_empty_level_set():
    from viennals_b200.advect import Context
    from viennals_b200.domain import Domain

    g = Grid([-5, 5, -5, 5, -5, 5], [BC.INFINITE_BOUNDARY] * 3, 0.5)
    empty = Domain(g, np.zeros((0, 3), np.int32), np.zeros(0),
                   np.array([[-100, -100, -100]], np.int32), np.array([1], np.int8), 2)
    ctx = Context()
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, empty)
    _check_runs(ctx, g)


def test_roundtrip_through_device_runs():
    from viennals_b200.advect import Context

    g, lss = sphere_case(5.0, 0.25)
    ctx, _ = run_gpu(g, lss, egg_velocity(), params(0, 0, 0.5))
    dom = ctx.download_domain(0, g)
    ctx2 = Context()
    ctx2.set_grid(g)
    ctx2.set_level_set_count(1)
    ctx2.upload(0, dom)
    again = ctx2.download_domain(0, g)
    assert np.array_equal(again.idx, dom.idx)
    assert np.array_equal(again.values, dom.values)
    assert np.array_equal(again.run_start, dom.run_start)
    assert np.array_equal(again.run_sign, dom.run_sign)
