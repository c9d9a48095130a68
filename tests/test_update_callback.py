"""setVelocityUpdateCallback (lsAdvect.hpp:966-969): called by RK2 once and
RK3 twice per step with the top level set (lsAdvectIntegrationSchemes.hpp:
88-89, 129-130, 147-149); with a callback, stage 1 adjusts the lower layers
and an etching combination restores them."""
import numpy as np
import pytest

from parity_cases import compare, params, run_oracle, sphere_case, trench_case
from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
from viennals_b200.velocity import VelocityField


class Stateful(VelocityField):
    """A velocity that depends on what the update callback saw last."""

    def __init__(self):
        self.k = 0
        self.seen = []

    def update(self, dom):
        self.seen.append((len(dom.values), float(np.sum(dom.values))))
        self.k = len(dom.values)
        return True

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        m = materials.astype(np.float64)
        scalar_out[:] = (0.6 + 0.2 * normals[:, 2] + 1e-5 * self.k) * (1.0 - 1.6 * m)
        vector_out[:] = 0.0


def run_gpu_upd(grid, lss, vel, p):
    from viennals_b200.advect import Context

    ctx = Context(0, 0)
    ctx.set_grid(grid)
    ctx.set_level_set_count(len(lss))
    for i, d in enumerate(lss):
        ctx.upload(i, d)
    ctx.set_velocity_callback(vel)
    ctx.set_velocity_update_callback(vel.update)
    return ctx, ctx.advect(p)


@pytest.mark.parametrize("temporal,calls", [(TS.FORWARD_EULER, 0), (TS.RUNGE_KUTTA_2ND_ORDER, 1),
                                            (TS.RUNGE_KUTTA_3RD_ORDER, 2)])
def test_oracle_update_calls(temporal, calls):
    g, ls = sphere_case(3.0, 0.5)
    vel = Stateful()
    p = params(S.ENGQUIST_OSHER_1ST_ORDER, temporal, 0.0, single_step=1)
    from oracle import oracle as O

    ols = [O.OracleLS(g, d) for d in ls]
    O.advect(ols, p, vel, update=vel.update)
    assert len(vel.seen) == calls


@pytest.mark.gpu
@pytest.mark.parametrize("temporal", [TS.RUNGE_KUTTA_2ND_ORDER, TS.RUNGE_KUTTA_3RD_ORDER])
def test_gpu_update_callback_sphere(temporal):
    from oracle import oracle as O

    g, ls = sphere_case(4.0, 0.25)
    p = params(S.WENO_5TH_ORDER, temporal, 0.3)
    vo, vg = Stateful(), Stateful()
    ols = [O.OracleLS(g, d) for d in ls]
    ores = O.advect(ols, p, vo, update=vo.update)
    ctx, gres = run_gpu_upd(g, ls, vg, p)
    compare(ols, ctx)
    assert vo.seen == vg.seen
    assert gres.number_of_time_steps == ores.number_of_time_steps


@pytest.mark.gpu
@pytest.mark.parametrize("temporal", [TS.RUNGE_KUTTA_2ND_ORDER, TS.RUNGE_KUTTA_3RD_ORDER])
def test_gpu_update_callback_two_materials(temporal):
    from oracle import oracle as O

    g, ls, _, p = trench_case(S.LOCAL_LAX_FRIEDRICHS_1ST_ORDER, temporal, 0.15)
    vo, vg = Stateful(), Stateful()
    ols = [O.OracleLS(g, d) for d in ls]
    ores = O.advect(ols, p, vo, update=vo.update)
    ctx, gres = run_gpu_upd(g, ls, vg, p)
    compare(ols, ctx)
    assert vo.seen == vg.seen
    assert gres.number_of_time_steps == ores.number_of_time_steps


@pytest.mark.gpu
def test_gpu_update_callback_failure():
    g, ls = sphere_case(3.0, 0.5)

    class Bad(Stateful):
        def update(self, dom):
            raise RuntimeError("no")

    with pytest.raises(RuntimeError, match="callback"):
        run_gpu_upd(g, ls, Bad(), params(S.ENGQUIST_OSHER_1ST_ORDER, TS.RUNGE_KUTTA_2ND_ORDER,
                                         0.0, single_step=1))


@pytest.mark.gpu
def test_python_front_apply_with_update_callback():
    # the same run through viennals_b200.advect.Advect (the reference's Python
    # binding names): setters, the update callback, apply() and the written-back
    # Domain
    from oracle import oracle as O
    from viennals_b200.advect import Advect

    g, ls = sphere_case(4.0, 0.25)
    p = params(S.WENO_5TH_ORDER, TS.RUNGE_KUTTA_3RD_ORDER, 0.3)
    vo, vg = Stateful(), Stateful()
    ols = [O.OracleLS(g, d) for d in ls]
    ores = O.advect(ols, p, vo, update=vo.update)
    a = Advect(ls[0], vg)
    a.setSpatialScheme(S.WENO_5TH_ORDER)
    a.setTemporalScheme(TS.RUNGE_KUTTA_3RD_ORDER)
    a.setAdvectionTime(0.3)
    a.setVelocityUpdateCallback(vg.update)
    a.apply()
    assert vg.seen == vo.seen
    assert a.getNumberOfTimeSteps() == ores.number_of_time_steps
    assert a.getAdvectedTime() == ores.advected_time
    compare(ols, a.ctx)
    oi, ov = ols[0].points(0)
    assert np.array_equal(ls[0].idx, oi)
    assert np.array_equal(np.asarray(ls[0].values).view(np.int64), ov.view(np.int64))
