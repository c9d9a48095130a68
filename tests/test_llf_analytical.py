"""LocalLaxFriedrichsAnalytical (lsLocalLaxFriedrichsAnalytical.hpp:20-242):
the user's getDissipationAlpha at the 3x3x3 box, from the device functor
(alpha[material][direction]) or the host alpha callback."""
import numpy as np
import pytest

from parity_cases import compare, params, run_gpu, run_oracle, sphere_case, trench_case
from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
from viennals_b200.velocity import FunctorVelocity

LLFA = S.LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER


class Callback(FunctorVelocity):
    """The functor's velocity and alphas, asked through the host callbacks."""

    def descriptor(self):
        return None


def square_etch(cls=FunctorVelocity):
    """SquareEtch.cpp:45-83: material 1 etched at -|n_z| where n_z > 0, alpha
    |v| along z."""
    v = cls(2)
    v.set_abs(1, 2, -1.0, 0.0)
    v.set_dissipation_alpha(1, 2, 1.0)
    return v


def egg_alpha(cls=FunctorVelocity):
    v = cls(1)
    v.set_rate(0, 1.0)
    v.set_square(0, 0, 2.3, 0.5)
    for d, a in enumerate((2.3, 1.0, 1.0)):
        v.set_dissipation_alpha(0, d, a)
    return v


def test_oracle_alpha_callback_equals_functor():
    g, ls = sphere_case(3.0, 0.5)
    p = params(LLFA, TS.RUNGE_KUTTA_3RD_ORDER, 0.0, single_step=1)
    a, ra = run_oracle(g, ls, egg_alpha(), p)
    b, rb = run_oracle(g, ls, egg_alpha(Callback), p)
    assert np.array_equal(a[0].points(0)[1], b[0].points(0)[1])
    assert ra.current_time_step == rb.current_time_step


def test_oracle_llfa_dissipation_matters():
    """Larger alphas give a smaller time step (reduceTimeStepHamiltonJacobi)."""
    g, ls = sphere_case(3.0, 0.5)
    p = params(LLFA, TS.FORWARD_EULER, 0.0, single_step=1, time_step_ratio=0.45)
    small = egg_alpha()
    big = egg_alpha()
    for d in range(3):
        big.set_dissipation_alpha(0, d, 5.0)
    _, rs = run_oracle(g, ls, small, p)
    _, rb = run_oracle(g, ls, big, p)
    assert rb.current_time_step < rs.current_time_step


@pytest.mark.gpu
@pytest.mark.parametrize("temporal", [TS.FORWARD_EULER, TS.RUNGE_KUTTA_3RD_ORDER])
def test_gpu_llfa_sphere(temporal):
    g, ls = sphere_case(4.0, 0.25)
    p = params(LLFA, temporal, 0.6)
    ols, ores = run_oracle(g, ls, egg_alpha(), p)
    ctx, gres = run_gpu(g, ls, egg_alpha(), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps
    assert gres.advected_time == ores.advected_time


@pytest.mark.gpu
def test_gpu_llfa_square_etch_two_materials():
    g, ls, _, p = trench_case(LLFA, TS.RUNGE_KUTTA_2ND_ORDER, 0.3)
    ols, ores = run_oracle(g, ls, square_etch(), p)
    ctx, gres = run_gpu(g, ls, square_etch(), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps


class Everything(FunctorVelocity):
    """Velocity from the coordinates and the normal, alphas from the central
    differences (bounded, since a box can reach undefined neighbours whose
    sentinel values make the differences infinite)."""

    def __init__(self):
        super().__init__(2)

    def descriptor(self):
        return None

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        m = materials.astype(np.float64)
        scalar_out[:] = 0.8 + 0.1 * coords[:, 0] - 0.9 * m * np.abs(normals[:, 2])
        vector_out[:] = 0.0

    def alpha_batch(self, directions, materials, cd, out):
        d = directions.astype(np.int64)
        out[:] = 0.2 + 0.1 * materials + 0.02 * np.fmin(np.abs(cd[np.arange(len(d)), d]), 50.0)


def small_trench():
    from viennals_b200 import BoundaryConditionEnum as BC, Grid
    from viennals_b200.geometry import trench_etch_level_sets

    g = Grid([-1.2, 1.2, -1.2, 1.2, -0.8, 0.8],
             [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 0.1)
    return g, list(trench_etch_level_sets(g, 0.3, 0.8))


@pytest.mark.gpu
def test_gpu_llfa_callbacks():
    g, ls = small_trench()
    p = params(LLFA, TS.RUNGE_KUTTA_2ND_ORDER, 0.0, single_step=1)
    vel = Everything()
    ols, ores = run_oracle(g, ls, vel, p)
    ctx, gres = run_gpu(g, ls, vel, p)
    compare(ols, ctx)
    assert gres.current_time_step == ores.current_time_step
