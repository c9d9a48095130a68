"""Point data through an advection (setSaveAdvectionVelocities,
setUpdatePointData): the top level set's per-point data is carried along the
source ids the reference's passes record (Expand lsExpand.hpp:110-150, Reduce
lsReduce.hpp:108-112, Prune lsPrune.hpp:164-168, the stage combination's
BooleanOperation lsBooleanOperation.hpp:104-114, rebuildLS lsAdvect.hpp:
318-410), and the value update saves each point's last rate and dissipation
(lsAdvect.hpp:764-767, 780-796).  The CUDA path against the oracle: the same
source ids and bit-identical FP64 velocities and dissipations."""
import numpy as np
import pytest

from parity_cases import compare, egg_velocity, params, run_gpu, run_oracle, sphere_case, trench_case


def _oracle_pd(grid, lss, vel, p):
    ols, ro = run_oracle(grid, lss, vel, p)
    return ols, ro, ols[-1].point_data()


def test_oracle_point_data_sources_and_velocities():
    """CPU: after a growing sphere's FE steps every point carries a source in
    range and the positive velocity of its last update; without
    updatePointData no point data is left (rebuildLS drops it)."""
    g, lss = sphere_case(3.0, 0.3)
    p = params(0, 0, 0.3, save_advection_velocities=1)
    ols, _, pd = _oracle_pd(g, lss, egg_velocity(), p)
    src, vel, diss = pd
    n0 = lss[0].n_points
    assert len(src) == len(ols[-1].points(0)[1])
    assert (src >= 0).all() and (src < n0).all()
    # EO has no dissipation; growth: every active point moved outwards
    assert (diss == 0).all() and (vel > 0).mean() > 0.3
    _, _, none = _oracle_pd(g, lss, egg_velocity(),
                            params(0, 0, 0.3, save_advection_velocities=1, update_point_data=0))
    assert none is None
    _, _, untracked = _oracle_pd(g, lss, egg_velocity(), params(0, 0, 0.3))
    assert untracked is None


CASES = [
    # (name, case builder, spatial, temporal)
    ("sphere EO1 FE", lambda: (*sphere_case(3.0, 0.3), egg_velocity()), 0, 0),
    ("sphere WENO5 RK3", lambda: (*sphere_case(3.0, 0.3), egg_velocity()), 11, 2),
    ("sphere LLF2 RK2", lambda: (*sphere_case(3.0, 0.3), egg_velocity()), 8, 1),
    ("trench LLF2 RK3", lambda: trench_case(8, 2, 0.1)[:3], 8, 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,spatial,temporal", CASES, ids=[c[0] for c in CASES])
def test_point_data_matches_oracle(name, make, spatial, temporal):
    g, lss, v = make()
    p = params(spatial, temporal, 0.15, save_advection_velocities=1)
    ols, ro, (src, vel, diss) = _oracle_pd(g, lss, v, p)
    ctx, rg = run_gpu(g, lss, v, p)
    assert rg.number_of_time_steps == ro.number_of_time_steps
    compare(ols, ctx)
    got = ctx.download_point_data(len(lss) - 1)
    assert got is not None
    gs, gv, gd = got
    assert np.array_equal(gs, src)
    assert np.array_equal(gv.view(np.int64), vel.view(np.int64))
    assert np.array_equal(gd.view(np.int64), diss.view(np.int64))
    if spatial == 8:
        assert (np.abs(gd) > 0).any()  # LLF dissipation saved


@pytest.mark.gpu
def test_point_data_dropped_without_update_and_untracked():
    g, lss = sphere_case(3.0, 0.3)
    ctx, _ = run_gpu(g, lss, egg_velocity(),
                     params(11, 2, 0.1, save_advection_velocities=1, update_point_data=0))
    assert ctx.download_point_data(0) is None
    ctx2, _ = run_gpu(g, lss, egg_velocity(), params(11, 2, 0.1))
    assert ctx2.download_point_data(0) is None


@pytest.mark.gpu
def test_python_front_translates_point_data():
    """A user array on the top level set follows its points through apply()
    (gathered by the source ids), and the saved velocities are attached."""
    from viennals_b200.advect import Advect

    g, lss = sphere_case(3.0, 0.3)
    dom = lss[0].copy()
    dom.point_data = {"tag": np.arange(dom.n_points, dtype=np.float64) * 2.0}
    adv = Advect(dom, egg_velocity())
    adv.setSpatialScheme(11)
    adv.setTemporalScheme(2)
    adv.setAdvectionTime(0.1)
    adv.setSaveAdvectionVelocities(True)
    adv.apply()
    ols, _, (src, vel, diss) = _oracle_pd(g, lss, egg_velocity(),
                                          params(11, 2, 0.1, save_advection_velocities=1))
    assert np.array_equal(dom.point_data["tag"], np.where(src >= 0, 2.0 * src, 0.0))
    assert np.array_equal(dom.point_data[Advect.velocityLabel], vel)
    assert np.array_equal(dom.point_data[Advect.dissipationLabel], diss)
