"""The batching form (vlsg_batch_set_domains / vlsg_batch_advect): many
domains advanced together in one context, one kernel launch per pass, must
give every domain exactly what advancing it alone gives -- the same defined
points, bit-identical values, the same undefined runs and the same getters
(advected time, time step, point updates) -- for FP32 and FP64 and for the
integration schemes, over consecutive steps; unsupported set-ups are
rejected with an error."""
import numpy as np
import pytest

from parity_cases import params
from viennals_b200 import BoundaryConditionEnum as BC, Grid
from viennals_b200.advect import BatchContext, Context
from viennals_b200.synth import batch_domains

pytestmark = pytest.mark.gpu


def _loop(items, p, precision, steps):
    out = []
    for grid, dom, vel in items:
        c = Context(0, precision)
        c.set_grid(grid)
        c.set_level_set_count(1)
        c.upload(0, dom)
        c.set_velocity(vel.descriptor())
        res = [c.advect(p) for _ in range(steps)]
        out.append((res, c.download_domain(0, grid)))
        c.close()
    return out


def _batch(items, p, precision, steps):
    b = BatchContext(0, precision)
    b.set_domains(items)
    res = [b.advect(p) for _ in range(steps)]
    doms = [b.download_domain(d) for d in range(len(items))]
    launches = [r[0].kernel_launches for r in res]
    b.close()
    return res, doms, launches


def _same(items, p, precision, steps=1):
    loop = _loop(items, p, precision, steps)
    res, doms, _ = _batch(items, p, precision, steps)
    for d, (lres, ldom) in enumerate(loop):
        for s in range(steps):
            a, b = lres[s], res[s][d]
            assert a.advected_time == b.advected_time, (d, s)
            assert a.current_time_step == b.current_time_step, (d, s)
            assert a.point_updates == b.point_updates, (d, s)
            assert a.number_of_stages == b.number_of_stages
        bd = doms[d]
        assert np.array_equal(ldom.idx, bd.idx), d
        assert np.array_equal(ldom.values.view(np.int64), bd.values.view(np.int64)), d
        assert np.array_equal(ldom.run_start, bd.run_start), d
        assert np.array_equal(ldom.run_sign, bd.run_sign), d


@pytest.mark.parametrize("precision", [0, 1])
def test_small_domains_llf1_rk2(precision):
    items = batch_domains(12, seed=3, points_range=(1e3, 3e4))
    p = params(7, 1, 0.0)  # LOCAL_LAX_FRIEDRICHS_1ST_ORDER, RK2, one step
    _same(items, p, precision, steps=2)


@pytest.mark.parametrize("spatial,temporal", [(0, 0), (11, 2), (8, 1), (5, 2)])
def test_schemes(spatial, temporal):
    items = batch_domains(5, seed=11, points_range=(2e3, 2e4))
    _same(items, params(spatial, temporal, 0.0, cfl=0.4), 1, steps=1)


def test_launches_do_not_grow_with_domains():
    p = params(7, 1, 0.0)
    few = batch_domains(3, seed=5, points_range=(2e3, 5e3))
    many = batch_domains(24, seed=5, points_range=(2e3, 5e3))
    _, _, l3 = _batch(few, p, 1, 1)
    _, _, l24 = _batch(many, p, 1, 1)
    assert l3 == l24


def test_unsupported_setups_are_errors():
    items = batch_domains(2, seed=1, points_range=(2e3, 5e3))
    b = BatchContext(0, 1)
    # a domain that is not periodic in x
    g, d, v = items[0]
    bad = Grid(None, [BC.REFLECTIVE_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY],
               g.delta, index_min=g.min, index_max=g.max)
    with pytest.raises(RuntimeError):
        b.set_domains([(bad, d, v)])
    b.set_domains(items)
    with pytest.raises(RuntimeError):
        b.advect(params(2, 1, 0.0))  # global Lax-Friedrichs
    with pytest.raises(RuntimeError):
        b.advect(params(7, 1, 0.5))  # an advection time: one step per call only
    b.close()
