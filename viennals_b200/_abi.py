"""ctypes mirror of include/vlsg.h (the C ABI of libvlsgpu.so).

The enums keep the numeric values of the reference's SpatialSchemeEnum /
TemporalSchemeEnum (include/viennals/lsAdvectIntegrationSchemes.hpp:10-35)
and of viennahrle::BoundaryType (python/viennals/_core.pyi:25-30).
"""
import ctypes
import enum

MAX_LEVEL_SETS = 8
MAX_MATERIALS = 16

OK = 0
ERR_ARGUMENT = -1
ERR_CUDA = -2
ERR_CAPACITY = -3
ERR_STATE = -4
ERR_NUMERIC = -5
ERR_DEVICE_CHECK = -6
ERR_CALLBACK = -7


class SpatialSchemeEnum(enum.IntEnum):
    ENGQUIST_OSHER_1ST_ORDER = 0
    ENGQUIST_OSHER_2ND_ORDER = 1
    LAX_FRIEDRICHS_1ST_ORDER = 2
    LAX_FRIEDRICHS_2ND_ORDER = 3
    LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER = 4
    LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 5
    LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER = 6
    LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 7
    LOCAL_LAX_FRIEDRICHS_2ND_ORDER = 8
    STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 9
    WENO_3RD_ORDER = 10
    WENO_5TH_ORDER = 11


class TemporalSchemeEnum(enum.IntEnum):
    FORWARD_EULER = 0
    RUNGE_KUTTA_2ND_ORDER = 1
    RUNGE_KUTTA_3RD_ORDER = 2


class BoundaryConditionEnum(enum.IntEnum):
    REFLECTIVE_BOUNDARY = 0
    INFINITE_BOUNDARY = 1
    PERIODIC_BOUNDARY = 2
    POS_INFINITE_BOUNDARY = 3
    NEG_INFINITE_BOUNDARY = 4


class Precision(enum.IntEnum):
    FP64 = 0
    FP32 = 1


class AdvectParams(ctypes.Structure):
    _fields_ = [
        ("spatial_scheme", ctypes.c_int32),
        ("temporal_scheme", ctypes.c_int32),
        ("time_step_ratio", ctypes.c_double),
        ("dissipation_alpha", ctypes.c_double),
        ("advection_time", ctypes.c_double),
        ("single_step", ctypes.c_int32),
        ("calculate_normal_vectors", ctypes.c_int32),
        ("ignore_voids", ctypes.c_int32),
        ("adaptive_time_stepping", ctypes.c_int32),
        ("adaptive_subdivisions", ctypes.c_uint32),
        ("check_dissipation", ctypes.c_int32),
        ("save_advection_velocities", ctypes.c_int32),
        ("update_point_data", ctypes.c_int32),
        ("max_steps", ctypes.c_uint32),
        ("max_dissipation", ctypes.c_double),
        ("track_point_data", ctypes.c_int32),
        ("fp32_compensation", ctypes.c_int32),
    ]

    @classmethod
    def defaults(cls):
        """Reference defaults, lsAdvect.hpp:64-79."""
        p = cls()
        p.spatial_scheme = SpatialSchemeEnum.ENGQUIST_OSHER_1ST_ORDER
        p.temporal_scheme = TemporalSchemeEnum.FORWARD_EULER
        p.time_step_ratio = 0.4999
        p.dissipation_alpha = 1.0
        p.advection_time = 0.0
        p.single_step = 0
        p.calculate_normal_vectors = 1
        p.ignore_voids = 0
        p.adaptive_time_stepping = 0
        p.adaptive_subdivisions = 20
        p.check_dissipation = 1
        p.save_advection_velocities = 0
        p.update_point_data = 1
        p.max_steps = 0
        p.max_dissipation = 0.0  # no limit
        p.track_point_data = 0
        p.fp32_compensation = 0
        return p


class AdvectResult(ctypes.Structure):
    _fields_ = [
        ("advected_time", ctypes.c_double),
        ("current_time_step", ctypes.c_double),
        ("number_of_time_steps", ctypes.c_uint32),
        ("number_of_stages", ctypes.c_uint32),
        ("point_updates", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64),
    ]


_Mat3 = (ctypes.c_double * 3) * MAX_MATERIALS


class VelocityDesc(ctypes.Structure):
    _fields_ = [
        ("n_materials", ctypes.c_int32),
        ("rate", ctypes.c_double * MAX_MATERIALS),
        ("lin_pos", _Mat3),
        ("lin_neg", _Mat3),
        ("abs_pos", _Mat3),
        ("abs_neg", _Mat3),
        ("sq_pos", _Mat3),
        ("sq_neg", _Mat3),
        ("vec", _Mat3),
        ("alpha", _Mat3),
    ]


class KernelStat(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
        ("algorithmic_bytes", ctypes.c_double),
    ]


class CompareResult(ctypes.Structure):
    """vlsg_compare_result (vlsg.h)."""
    _fields_ = [
        ("points_a", ctypes.c_int64), ("points_b", ctypes.c_int64),
        ("common_points", ctypes.c_int64),
        ("defined_only_a", ctypes.c_int64), ("defined_only_b", ctypes.c_int64),
        ("active_a", ctypes.c_int64), ("active_b", ctypes.c_int64),
        ("active_only_a", ctypes.c_int64), ("active_only_b", ctypes.c_int64),
        ("max_abs_diff", ctypes.c_double), ("rms_abs_diff", ctypes.c_double),
        ("inside_cells_a", ctypes.c_int64), ("inside_cells_b", ctypes.c_int64),
        ("nodes_a", ctypes.c_int64), ("nodes_b", ctypes.c_int64),
        ("chamfer_ab", ctypes.c_double), ("chamfer_ba", ctypes.c_double),
        ("chamfer_mean", ctypes.c_double), ("chamfer_rms", ctypes.c_double),
        ("chamfer_max", ctypes.c_double),
        ("chamfer_unresolved", ctypes.c_int64),
        ("diff_above", ctypes.c_int64 * 4),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["diff_above"] = list(self.diff_above)
        return d


ALPHA_CALLBACK = ctypes.CFUNCTYPE(
    ctypes.c_int,
    ctypes.c_void_p,
    ctypes.c_int64,
    ctypes.POINTER(ctypes.c_int32),
    ctypes.POINTER(ctypes.c_int32),
    ctypes.POINTER(ctypes.c_double),
    ctypes.POINTER(ctypes.c_double),
)

class LevelSetView(ctypes.Structure):
    """vlsg_levelset_view: a level set as the velocity-update callback sees it."""
    _fields_ = [
        ("n_points", ctypes.c_int64),
        ("indices", ctypes.POINTER(ctypes.c_int32)),
        ("values", ctypes.POINTER(ctypes.c_double)),
        ("n_runs", ctypes.c_int64),
        ("run_start", ctypes.POINTER(ctypes.c_int32)),
        ("run_sign", ctypes.POINTER(ctypes.c_int8)),
        ("width", ctypes.c_int32),
    ]


UPDATE_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(LevelSetView))
# vlsg_reduce_cb: (user, double *values, n, op) -> int
REDUCE_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                   ctypes.c_int32, ctypes.c_int32)
REDUCE_MIN = 0
REDUCE_MAX = 1

VELOCITY_CALLBACK = ctypes.CFUNCTYPE(
    ctypes.c_int,
    ctypes.c_void_p,
    ctypes.c_int64,
    ctypes.POINTER(ctypes.c_double),
    ctypes.POINTER(ctypes.c_int32),
    ctypes.POINTER(ctypes.c_double),
    ctypes.POINTER(ctypes.c_uint64),
    ctypes.POINTER(ctypes.c_double),
    ctypes.POINTER(ctypes.c_double),
)


class BatchDomain(ctypes.Structure):
    """vlsg_batch_domain: one domain of the batching form."""
    _fields_ = [
        ("grid_min", ctypes.POINTER(ctypes.c_int64)),
        ("grid_max", ctypes.POINTER(ctypes.c_int64)),
        ("boundary", ctypes.POINTER(ctypes.c_int32)),
        ("grid_delta", ctypes.c_double),
        ("n_points", ctypes.c_int64),
        ("indices", ctypes.POINTER(ctypes.c_int32)),
        ("values", ctypes.POINTER(ctypes.c_double)),
        ("n_runs", ctypes.c_int64),
        ("run_start", ctypes.POINTER(ctypes.c_int32)),
        ("run_sign", ctypes.POINTER(ctypes.c_int8)),
        ("width", ctypes.c_int32),
        ("velocity", ctypes.POINTER(VelocityDesc)),
    ]
