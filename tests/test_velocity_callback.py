"""Host velocity callbacks (VelocityField with user code, lsVelocityField.hpp:
17-30): the oracle and the CUDA path ask the callback with the coordinate,
material, normal and point id the reference passes (lsWENO.hpp:132-137,
lsLocalLaxFriedrichs.hpp:194-216, lsAdvect.hpp:150-173)."""
import numpy as np
import pytest

from parity_cases import compare, params, run_gpu, run_oracle, sphere_case, trench_case
from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
from viennals_b200.velocity import FunctorVelocity, VelocityField


class PolyCallback(FunctorVelocity):
    """The functor's polynomial, asked through the host callback."""

    def descriptor(self):
        return None


def poly(cls=PolyCallback):
    v = cls(1)
    v.set_rate(0, 1.0)
    v.set_square(0, 0, 2.3, 0.5)
    v.set_linear(0, 2, 0.3, -0.2)
    v.set_vector(0, (0.05, 0.0, -0.02))
    return v


class FieldOfEverything(VelocityField):
    """A velocity that depends on every argument of the callback (vectorised:
    the same elementwise float64 operations for one point or many)."""

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        m = materials.astype(np.float64)
        pid = (point_ids % np.uint64(7)).astype(np.float64)
        scalar_out[:] = (0.6 + 0.1 * coords[:, 0] - 0.05 * coords[:, 2] * normals[:, 2]
                         + 1e-3 * pid - 0.8 * m * (1.0 + 0.3 * normals[:, 2]))
        vector_out[:, 0] = 0.02 * coords[:, 1]
        vector_out[:, 1] = 0.0
        vector_out[:, 2] = -0.01 * m


class Recorder(VelocityField):
    def __init__(self):
        self.rows = []

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        for i in range(len(materials)):
            self.rows.append((tuple(coords[i]), int(materials[i]), int(point_ids[i])))
        scalar_out[:] = 1.0
        vector_out[:] = 0.0


class Failing(VelocityField):
    def batch(self, *a):
        raise RuntimeError("no velocity here")


SCHEMES = [S.ENGQUIST_OSHER_1ST_ORDER, S.WENO_5TH_ORDER, S.LOCAL_LAX_FRIEDRICHS_1ST_ORDER,
           S.LAX_FRIEDRICHS_2ND_ORDER, S.LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER]


@pytest.mark.parametrize("spatial", SCHEMES)
def test_oracle_callback_equals_functor(spatial):
    g, ls = sphere_case(3.0, 0.5)
    p = params(spatial, TS.RUNGE_KUTTA_2ND_ORDER, 0.0, single_step=1)
    a, ra = run_oracle(g, ls, poly(FunctorVelocity), p)
    b, rb = run_oracle(g, ls, poly(), p)
    ia, va = a[0].points(0)
    ib, vb = b[0].points(0)
    assert np.array_equal(ia, ib)
    assert np.array_equal(va, vb)
    assert ra.current_time_step == rb.current_time_step


def test_oracle_point_ids_are_hrle_ranks():
    g, ls = sphere_case(3.0, 0.5)
    rec = Recorder()
    run_oracle(g, ls, rec, params(S.WENO_5TH_ORDER, TS.FORWARD_EULER, 0.0, single_step=1))
    assert rec.rows
    by_id = {}
    for c, m, pid in rec.rows:
        assert m == 0
        by_id.setdefault(pid, set()).add(c)
    assert all(len(v) == 1 for v in by_id.values())  # one point per id
    ids = sorted(by_id)
    keys = [next(iter(by_id[i])) for i in ids]
    # HRLE order: z slowest, x fastest
    zyx = [(c[2], c[1], c[0]) for c in keys]
    assert zyx == sorted(zyx)


def test_oracle_callback_failure_is_an_error():
    from oracle import oracle as O

    g, ls = sphere_case(3.0, 0.5)
    with pytest.raises(RuntimeError, match="callback"):
        run_oracle(g, ls, Failing(), params(S.ENGQUIST_OSHER_1ST_ORDER, TS.FORWARD_EULER, 0.0,
                                               single_step=1))
    assert O is not None


@pytest.mark.gpu
@pytest.mark.parametrize("spatial", SCHEMES + [S.WENO_3RD_ORDER, S.LOCAL_LAX_FRIEDRICHS_2ND_ORDER])
def test_gpu_callback_matches_oracle(spatial):
    g, ls = sphere_case(4.0, 0.25)
    vel = FieldOfEverything()
    p = params(spatial, TS.RUNGE_KUTTA_3RD_ORDER, 0.0, single_step=1)
    ols, ores = run_oracle(g, ls, vel, p)
    ctx, gres = run_gpu(g, ls, vel, p)
    compare(ols, ctx)
    assert gres.current_time_step == ores.current_time_step
    assert gres.point_updates == ores.point_updates


@pytest.mark.gpu
@pytest.mark.parametrize("spatial,temporal", [(S.LOCAL_LAX_FRIEDRICHS_2ND_ORDER, TS.RUNGE_KUTTA_3RD_ORDER),
                                              (S.ENGQUIST_OSHER_1ST_ORDER, TS.FORWARD_EULER)])
def test_gpu_callback_two_materials(spatial, temporal):
    g, ls, _, p = trench_case(spatial, temporal, 0.15)
    vel = FieldOfEverything()
    ols, ores = run_oracle(g, ls, vel, p)
    ctx, gres = run_gpu(g, ls, vel, p)
    compare(ols, ctx)
    assert gres.number_of_time_steps == ores.number_of_time_steps
    assert gres.advected_time == ores.advected_time


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_callback_equals_functor(precision):
    g, ls = sphere_case(4.0, 0.25)
    p = params(S.WENO_5TH_ORDER, TS.RUNGE_KUTTA_3RD_ORDER, 0.5)
    if precision == 0:
        cb, fn = poly(), poly(FunctorVelocity)
    else:  # FP32: the functor's float arithmetic differs from a double callback
        cb, fn = PolyCallback(1).set_rate(0, 0.7), FunctorVelocity(1).set_rate(0, 0.7)
    a, ra = run_gpu(g, ls, fn, p, precision)
    b, rb = run_gpu(g, ls, cb, p, precision)
    ia, va, _ = a.download(0)
    ib, vb, _ = b.download(0)
    assert np.array_equal(ia, ib)
    assert np.array_equal(va, vb)
    assert ra.number_of_time_steps == rb.number_of_time_steps


@pytest.mark.gpu
def test_gpu_callback_point_ids_match_oracle():
    g, ls = sphere_case(3.0, 0.5)
    p = params(S.WENO_5TH_ORDER, TS.FORWARD_EULER, 0.0, single_step=1)
    ro, rg = Recorder(), Recorder()
    run_oracle(g, ls, ro, p)
    run_gpu(g, ls, rg, p)
    assert sorted(ro.rows) == sorted(rg.rows)


@pytest.mark.gpu
def test_gpu_callback_failure_is_an_error():
    from viennals_b200._abi import ERR_CALLBACK

    g, ls = sphere_case(3.0, 0.5)
    with pytest.raises(RuntimeError) as e:
        run_gpu(g, ls, Failing(), params(S.ENGQUIST_OSHER_1ST_ORDER, TS.FORWARD_EULER, 0.0,
                                         single_step=1))
    assert "callback" in str(e.value)
    assert ERR_CALLBACK == -7
