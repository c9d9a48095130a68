"""setIgnoreVoids (lsAdvect.hpp:899, :443-454, :510): points of the top
level set enclosed in a void (MarkVoidPoints, lsMarkVoidPoints.hpp, default
options) get no rates."""
import numpy as np
import pytest

from parity_cases import compare, params, run_gpu, run_oracle
from viennals_b200 import BoundaryConditionEnum as BC, Grid
from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
from viennals_b200.geometry import sdf_levelset
from viennals_b200.velocity import constant_scalar


def buried_void(delta=0.1, depth=1.0, radius=0.5):
    """A substrate below z = 0 (periodic in x/y) with a spherical void of the
    given radius whose centre lies `depth` below the surface."""
    g = Grid([-1.6, 1.6, -1.6, 1.6, -2.0, 1.0],
             [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], delta)

    def sdf(x, y, z):
        return np.maximum(z, radius - np.sqrt(x * x + y * y + (z + depth) ** 2))

    dom = sdf_levelset(g, sdf, [g.min[0], g.min[1], g.min[2]],
                       [g.max[0] - 1, g.max[1] - 1, g.max[2]])
    return g, dom


def test_oracle_voids_are_frozen():
    """Growth at v = 1: with ignoreVoids the bubble keeps its points (its
    surface does not move), without it the bubble shrinks."""
    g, dom = buried_void()
    deep = lambda o: o[0].points(0)[0][:, 2] < -3
    a, _ = run_oracle(g, [dom], constant_scalar(1.0), params(0, 0, 0.2, ignore_voids=0))
    b, _ = run_oracle(g, [dom], constant_scalar(1.0), params(0, 0, 0.2, ignore_voids=1))
    assert deep(b).sum() > 2 * deep(a).sum()


@pytest.mark.gpu
@pytest.mark.parametrize("spatial,temporal", [(S.ENGQUIST_OSHER_1ST_ORDER, TS.FORWARD_EULER),
                                              (S.WENO_5TH_ORDER, TS.RUNGE_KUTTA_3RD_ORDER),
                                              (S.LOCAL_LAX_FRIEDRICHS_1ST_ORDER,
                                               TS.RUNGE_KUTTA_2ND_ORDER)])
def test_gpu_ignore_voids(spatial, temporal):
    g, dom = buried_void()
    p = params(spatial, temporal, 0.2, ignore_voids=1)
    ols, ores = run_oracle(g, [dom], constant_scalar(1.0), p)
    ctx, gres = run_gpu(g, [dom], constant_scalar(1.0), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps


@pytest.mark.gpu
def test_gpu_ignore_voids_fp32_runs():
    g, dom = buried_void()
    p = params(S.WENO_5TH_ORDER, TS.RUNGE_KUTTA_3RD_ORDER, 0.2, ignore_voids=1)
    ctx, res = run_gpu(g, [dom], constant_scalar(1.0), p, precision=1)
    idx, val, _ = ctx.download(0)
    assert (idx[:, 2] < -3).sum() > 300
