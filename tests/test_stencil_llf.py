"""STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER (lsStencilLocalLaxFriedrichsScalar.hpp
:30-400): Toifl et al.'s stencil dissipation, rebuild to width 3 with cutoff
1.5 (lsAdvect.hpp:250-256), no lower-layer adjustment (:802-813), the time
step bounded by the last passing call's finalAlphas."""
import numpy as np
import pytest

from parity_cases import (compare, egg_velocity, params, run_gpu, run_oracle, sphere_case,
                          trench_case)
from viennals_b200 import BoundaryConditionEnum as BC, Grid
from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
from viennals_b200.geometry import make_sphere
from viennals_b200.velocity import FunctorVelocity, constant_scalar

SLLF = S.STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER


class Callback(FunctorVelocity):
    def descriptor(self):
        return None


def egg(cls=FunctorVelocity):
    v = cls(1)
    v.set_rate(0, 1.0)
    v.set_square(0, 0, 2.3, 0.5)
    v.set_vector(0, (0.1, 0.0, 0.0))
    return v


def square_etch():
    """SquareEtch.cpp:26-41: material 1 etched at -|n_z| where n_z > 0."""
    v = FunctorVelocity(2)
    v.set_abs(1, 2, -1.0, 0.0)
    return v


class Everything(FunctorVelocity):
    def __init__(self):
        super().__init__(1)

    def descriptor(self):
        return None

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        scalar_out[:] = 0.7 + 0.1 * coords[:, 1] + 0.4 * normals[:, 0] ** 2 + 1e-3 * (point_ids % 5)
        vector_out[:, 0] = 0.05
        vector_out[:, 1:] = 0.0


def test_oracle_callback_equals_functor():
    g, ls = sphere_case(3.0, 0.5)
    p = params(SLLF, TS.FORWARD_EULER, 0.0, single_step=1)
    a, ra = run_oracle(g, ls, egg(), p)
    b, rb = run_oracle(g, ls, egg(Callback), p)
    assert np.array_equal(a[0].points(0)[1], b[0].points(0)[1])
    assert ra.current_time_step == rb.current_time_step


@pytest.mark.gpu
@pytest.mark.parametrize("temporal", [TS.FORWARD_EULER, TS.RUNGE_KUTTA_2ND_ORDER,
                                      TS.RUNGE_KUTTA_3RD_ORDER])
def test_gpu_sllf_sphere(temporal):
    g, ls = sphere_case(4.0, 0.25)
    p = params(SLLF, temporal, 0.4)
    ols, ores = run_oracle(g, ls, egg(), p)
    ctx, gres = run_gpu(g, ls, egg(), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps
    assert gres.advected_time == ores.advected_time


@pytest.mark.gpu
def test_gpu_sllf_reference_case():
    """StencilLocalLaxFriedrichs.cpp:33-84 on the GPU: equal to the oracle and
    within the reference's Chamfer bound of the analytic sphere."""
    from oracle import oracle as O

    g = Grid([-3, 3, -3, 3, -3, 3], [BC.INFINITE_BOUNDARY] * 3, 0.1)
    ls = [make_sphere(g, [0, 0, 0], 1.0)]
    p = params(SLLF, TS.FORWARD_EULER, 0.5, cfl=0.4999)
    ols, ores = run_oracle(g, ls, constant_scalar(1.0), p)
    ctx, gres = run_gpu(g, ls, constant_scalar(1.0), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps
    ref = O.OracleLS(g, make_sphere(g, [0, 0, 0], 1.5))
    out = O.OracleLS(g, ctx.download_domain(0, g))
    assert out.check() == 0
    assert O.chamfer(ref, out)["chamfer"] < 0.035


@pytest.mark.gpu
def test_gpu_sllf_square_etch_two_materials():
    g, ls, _, p = trench_case(SLLF, TS.FORWARD_EULER, 0.3)
    ols, ores = run_oracle(g, ls, square_etch(), p)
    ctx, gres = run_gpu(g, ls, square_etch(), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps


@pytest.mark.gpu
def test_gpu_sllf_max_dissipation():
    g, ls = sphere_case(4.0, 0.25)
    p = params(SLLF, TS.FORWARD_EULER, 0.3, max_dissipation=0.3)
    ols, ores = run_oracle(g, ls, egg(), p)
    ctx, gres = run_gpu(g, ls, egg(), p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps


@pytest.mark.gpu
def test_gpu_sllf_callbacks():
    g, ls = sphere_case(3.0, 0.5)
    p = params(SLLF, TS.RUNGE_KUTTA_2ND_ORDER, 0.0, single_step=1)
    vel = Everything()
    ols, ores = run_oracle(g, ls, vel, p)
    ctx, gres = run_gpu(g, ls, vel, p)
    compare(ols, ctx)
    assert gres.current_time_step == ores.current_time_step


DEPO_PATTERNS = [[False, True], [True, True], [True, False], [False, False]]


@pytest.mark.parametrize("depo", DEPO_PATTERNS)
def test_oracle_prepare_finalize_valid(depo):
    from oracle import oracle as O

    g, ls, _, _ = trench_case()
    ols = [O.OracleLS(g, d) for d in ls]
    O.prepare_stencil_llf(ols, depo)
    assert ols[-1].check() == 0
    O.finalize_stencil_llf(ols)
    assert ols[-1].check() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("depo", DEPO_PATTERNS)
def test_gpu_prepare_finalize(depo):
    """PrepareStencilLocalLaxFriedrichs, then FinalizeStencilLocalLaxFriedrichs,
    on the GPU equal the oracle's."""
    from oracle import oracle as O
    from viennals_b200.advect import Context

    g, ls, _, _ = trench_case()
    ols = [O.OracleLS(g, d) for d in ls]
    ctx = Context(0, 0)
    ctx.set_grid(g)
    ctx.set_level_set_count(len(ls))
    for i, d in enumerate(ls):
        ctx.upload(i, d)
    O.prepare_stencil_llf(ols, depo)
    ctx.prepare_stencil_llf(depo)
    compare(ols, ctx)
    O.finalize_stencil_llf(ols)
    ctx.finalize_stencil_llf()
    compare(ols, ctx)


@pytest.mark.gpu
def test_gpu_stencil_workflow():
    """Prepare, advect with Stencil LLF (SquareEtch velocity), finalize."""
    from oracle import oracle as O
    from viennals_b200.advect import Context

    g, ls, _, p = trench_case(SLLF, TS.FORWARD_EULER, 0.2)
    depo = [False, True]
    ols = [O.OracleLS(g, d) for d in ls]
    O.prepare_stencil_llf(ols, depo)
    ores = O.advect(ols, p, square_etch())
    O.finalize_stencil_llf(ols)
    ctx = Context(0, 0)
    ctx.set_grid(g)
    ctx.set_level_set_count(len(ls))
    for i, d in enumerate(ls):
        ctx.upload(i, d)
    ctx.set_velocity(square_etch().descriptor())
    ctx.prepare_stencil_llf(depo)
    gres = ctx.advect(p)
    ctx.finalize_stencil_llf()
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps
