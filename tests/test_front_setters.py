"""Host logic of the Python front (viennals_b200.advect.Advect): the setters
and getters of lsAdvect.hpp:856-969 land in the C ABI's parameter block, and
the reference's error cases are reported before any device work."""
import pytest

from viennals_b200 import AdvectParams
from viennals_b200.advect import Advect


def test_defaults_and_getters():
    a = Advect()
    d = AdvectParams.defaults()
    for name, _ in AdvectParams._fields_:
        assert getattr(a.params, name) == getattr(d, name), name
    assert a.getCurrentTimeStep() == -1.0
    assert a.getTimeStepRatio() == pytest.approx(0.4999)
    assert a.getCalculateNormalVectors() is True
    assert a.getNumberOfTimeSteps() == 0
    assert a.getAdvectedTime() == 0.0


def test_setters_fill_the_parameter_block():
    a = Advect()
    a.setAdvectionTime(2.5)
    a.setSingleStep(True)
    a.setTimeStepRatio(0.3)
    a.setCalculateNormalVectors(False)
    a.setIgnoreVoids(True)
    a.setAdaptiveTimeStepping(True, 7)
    a.setSaveAdvectionVelocities(True)
    a.setSpatialScheme(11)
    a.setTemporalScheme(2)
    a.setDissipationAlpha(0.7)
    a.setCheckDissipation(False)
    a.setUpdatePointData(False)
    a.setMaxDissipation(3.0)
    p = a.params
    assert (p.advection_time, p.single_step, p.time_step_ratio) == (2.5, 1, 0.3)
    assert (p.calculate_normal_vectors, p.ignore_voids) == (0, 1)
    assert (p.adaptive_time_stepping, p.adaptive_subdivisions) == (1, 7)
    assert (p.save_advection_velocities, p.spatial_scheme, p.temporal_scheme) == (1, 11, 2)
    assert (p.dissipation_alpha, p.check_dissipation, p.update_point_data) == (0.7, 0, 0)
    assert p.max_dissipation == 3.0
    assert a.getTimeStepRatio() == 0.3 and a.getCalculateNormalVectors() is False
    a.setIntegrationScheme(4)  # the deprecated name
    assert p.spatial_scheme == 4
    with pytest.raises(ValueError):
        a.setSpatialScheme(12)


def test_velocity_update_callback_is_kept():
    a = Advect()
    calls = []
    a.setVelocityUpdateCallback(calls.append)
    assert a.velocityUpdateCallback is not None


def test_errors_before_device_work():
    with pytest.raises(RuntimeError, match="No level sets passed to Advect"):
        Advect().apply()
    with pytest.raises(RuntimeError, match="No level sets passed to Advect"):
        Advect().prepareLS()
    from viennals_b200 import BoundaryConditionEnum as BC, Grid
    from viennals_b200.geometry import make_sphere

    g = Grid([-2, 2, -2, 2, -2, 2], [BC.INFINITE_BOUNDARY] * 3, 0.5)
    a = Advect(make_sphere(g, [0, 0, 0], 1.0))
    with pytest.raises(RuntimeError, match="No velocity field passed to Advect"):
        a.apply()
    assert a.ctx is None
