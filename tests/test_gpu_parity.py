"""CUDA path (through the C ABI) against the oracle, FP64: identical defined
point sets and bit-identical values after every run (integer index work
bit-exact; FP64 phi within 0 ulp, which implies the 1e-9*gridDelta bound)."""
import numpy as np
import pytest

from parity_cases import (compare, sphere_growth_eo1, egg_velocity, params, run_gpu,
                          run_oracle, sphere_case, trench_case)
from viennals_b200 import BoundaryConditionEnum as BC, Grid
from viennals_b200.geometry import make_sphere, sdf_levelset
from viennals_b200.velocity import FunctorVelocity, constant_scalar, constant_vector

pytestmark = pytest.mark.gpu


def _parity(grid, lss, vel, p):
    ols, ro = run_oracle(grid, lss, vel, p)
    ctx, rg = run_gpu(grid, lss, vel, p)
    assert rg.number_of_time_steps == ro.number_of_time_steps
    assert rg.advected_time == ro.advected_time
    assert rg.current_time_step == ro.current_time_step
    assert rg.point_updates == ro.point_updates
    assert rg.kernel_launches > 0
    compare(ols, ctx)
    return ols, ctx, rg


def test_roundtrip_upload_download():
    g, lss = sphere_case(5.0, 0.25)
    from viennals_b200.advect import Context

    ctx = Context()
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, lss[0])
    idx, val, w = ctx.download(0)
    ref_i, ref_v = lss[0].sorted()
    assert w == 2
    assert np.array_equal(idx, ref_i)
    assert np.array_equal(val, ref_v)


def test_sphere_growth_eo1_fe():
    g, lss, v, p = sphere_growth_eo1()
    _parity(g, lss, v, p)


@pytest.mark.parametrize("spatial", [0, 10, 11])
@pytest.mark.parametrize("temporal", [0, 1, 2])
def test_time_integration_cases(spatial, temporal):
    g = Grid([-5, 5, -5, 5, -5, 5], [BC.INFINITE_BOUNDARY] * 3, 0.15)
    lss = [make_sphere(g, [0, 0, 0], 1.5)]
    _parity(g, lss, constant_vector([1.0, 0.0, 0.0]), params(spatial, temporal, 0.5))


@pytest.mark.parametrize("half,spatial,temporal", [(3.0, 11, 2), (1.5, 11, 1), (1.5, 0, 2),
                                                   (2.5, 8, 2), (1.0, 0, 2), (1.0, 5, 1)])
def test_band_width_and_saved_copy(half, spatial, temporal):
    # Uploaded bands of width 2 * half.  The RK copy of the top level set is
    # taken during the first stage's Expand when the band is narrower than the
    # stage combination's Expand width and its values stay within half of it,
    # otherwise at the step's start; both must match the reference's deep copy
    # at the step's start.
    g = Grid([-5, 5, -5, 5, -5, 5], [BC.INFINITE_BOUNDARY] * 3, 0.15)
    ls = sdf_levelset(g, lambda x, y, z: np.sqrt(x * x + y * y + z * z) - 1.5,
                      [-22] * 3, [22] * 3, half_width=half)
    assert ls.width == int(round(2 * half))
    _parity(g, [ls], constant_vector([1.0, 0.0, 0.0]), params(spatial, temporal, 0.3))


@pytest.mark.parametrize("spatial", [0, 1, 2, 3, 5, 6, 7, 8, 10, 11])
def test_all_schemes_egg_velocity(spatial):
    g = Grid(None, [BC.INFINITE_BOUNDARY] * 3, 0.6999999)
    lss = [make_sphere(g, [5.0, 0.0, 0.0], 7.3)]
    _parity(g, lss, egg_velocity(), params(spatial, 0, 0.5))


@pytest.mark.parametrize("spatial,temporal", [(8, 2), (7, 1), (5, 0)])
def test_trench_two_materials_periodic(spatial, temporal):
    g, lss, v, p = trench_case(spatial, temporal, 0.2)
    _parity(g, lss, v, p)


def test_periodic_extent_not_multiple_of_brick():
    # 50 x 46 points: the last brick of x and y hangs over the periodic end
    from viennals_b200.geometry import trench_etch_level_sets

    g = Grid([-2.5, 2.5, -2.3, 2.3, -1.6, 1.6],
             [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 0.1)
    m, t = trench_etch_level_sets(g, 0.5, 1.6)
    v = FunctorVelocity(2)
    v.set_rate(1, -1.0)
    v.set_linear(1, 2, -0.3)
    _parity(g, [m, t], v, params(11, 2, 0.15))


def test_multi_material_union_rk3():
    from oracle import oracle as O

    g = Grid(None, [BC.INFINITE_BOUNDARY] * 3, 0.25)
    s1 = make_sphere(g, [5.0, 0.0, 0.0], 4.5)
    s2 = make_sphere(g, [-1.0, 0.0, 0.0], 3.3)
    o1, o2 = O.OracleLS(g, s1), O.OracleLS(g, s2)
    o2.boolean(o1, 1)  # top wraps the lower one (MultiMaterialAdvection.cpp:75-77)
    from viennals_b200.domain import Domain, make_runs

    def dom(o):
        i, val = o.points(0)
        lo, hi = i.min(0) - 2, i.max(0) + 2
        rs, sg = make_runs(i, lambda x, y, z: np.where(
            o.values_at(np.stack([x, y, z], 1).astype(np.int32)) < 0, -1, 1), lo, hi)
        return Domain(g, i, val, rs, sg, width=o.width)

    v = FunctorVelocity(2)
    v.set_rate(0, -0.2)
    v.set_rate(1, 0.5)
    p = params(0, 2, 1.0, calculate_normal_vectors=0)
    _parity(g, [dom(o1), dom(o2)], v, p)


def test_three_materials_adaptive_etch():
    g = Grid([-3.2, 3.2, -3.2, 3.2, -3, 3],
             [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 0.2)
    lo = [g.min[0], g.min[1], -20]
    hi = [g.max[0] - 1, g.max[1] - 1, 20]
    sub = sdf_levelset(g, lambda x, y, z: z + 0.3, lo, hi)
    poly = sdf_levelset(g, lambda x, y, z: z - 0.55, lo, hi)
    mask = sdf_levelset(g, lambda x, y, z: np.maximum(np.maximum(z - 0.2, -0.3 - z), 1.2 - np.abs(x)),
                        lo, hi)
    v = FunctorVelocity(3)
    v.set_rate(0, 0.0).set_rate(1, -10.0).set_rate(2, -0.1)
    p = params(0, 0, 0.3, adaptive_time_stepping=1, adaptive_subdivisions=20)
    _parity(g, [mask, sub, poly], v, p)


def test_reflective_tilted_plane():
    g = Grid([-3, 3, -3, 3, -4, 4],
             [BC.REFLECTIVE_BOUNDARY, BC.REFLECTIVE_BOUNDARY, BC.INFINITE_BOUNDARY], 0.25)
    n = np.array([0.3, 0.2, 1.0])
    n /= np.linalg.norm(n)
    lss = [sdf_levelset(g, lambda x, y, z: n[0] * x + n[1] * y + n[2] * z,
                        [g.min[0], g.min[1], -20], [g.max[0], g.max[1], 20])]
    _parity(g, lss, constant_scalar(-1.0), params(1, 1, 0.5))


def test_empty_level_set():
    g = Grid([-2, 2, -2, 2, -2, 2], [BC.INFINITE_BOUNDARY] * 3, 0.5)
    from viennals_b200.domain import Domain

    d = Domain(g, np.zeros((0, 3), np.int32), np.zeros(0),
               np.array([[-100, -100, -100]], np.int32), np.array([1], np.int8), 2)
    _parity(g, [d], constant_scalar(1.0), params(0, 0, 0.5))


# Expand width per spatial scheme (the schemes' prepareLS)
SCHEME_WIDTH = {0: 3, 1: 5, 2: 3, 3: 5, 4: 7, 5: 3, 6: 5, 7: 7, 8: 9, 9: 8, 10: 5, 11: 7}


@pytest.mark.parametrize("spatial", [0, 3, 8, 9, 11])
def test_prepare_ls_matches_oracle_expand(spatial):
    # Advect::prepareLS (lsAdvect.hpp:972-1015) through vlsg_prepare_ls: the
    # top level set expanded to the scheme's width
    from oracle import oracle as O
    from viennals_b200.advect import Context

    g, lss = sphere_case(5.0, 0.25)
    ols = O.OracleLS(g, lss[0])
    ols.expand(SCHEME_WIDTH[spatial])
    ctx = Context()
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, lss[0])
    ctx.prepare_ls(spatial)
    assert ctx.download(0)[2] == ols.width == SCHEME_WIDTH[spatial]
    compare([ols], ctx)


def test_prepare_ls_unknown_scheme_is_an_error():
    from viennals_b200.advect import Context

    g, lss = sphere_case(5.0, 0.25)
    ctx = Context()
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, lss[0])
    with pytest.raises(RuntimeError, match="Discretization scheme not found"):
        ctx.prepare_ls(99)
