"""B200-native level-set advection (drop-in for viennals::Advect<T,3>)."""
from ._abi import (AdvectParams, AdvectResult, BoundaryConditionEnum, Precision,
                   SpatialSchemeEnum, TemporalSchemeEnum, VelocityDesc)
from .domain import Domain, Grid
from .velocity import FunctorVelocity, VelocityField, constant_scalar, constant_vector
from .advect import FinalizeStencilLocalLaxFriedrichs, PrepareStencilLocalLaxFriedrichs  # noqa: E402
