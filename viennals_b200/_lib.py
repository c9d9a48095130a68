"""Loader of the in-tree libvlsgpu.so (no CPU fallback: it fails loudly)."""
import ctypes
import os

from ._abi import (ALPHA_CALLBACK, REDUCE_CALLBACK, UPDATE_CALLBACK, VELOCITY_CALLBACK, AdvectParams,
                   AdvectResult, BatchDomain, CompareResult, KernelStat, VelocityDesc)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvlsgpu.so")

_lib = None


def load(build_if_missing=True):
    """Return the ctypes handle of libvlsgpu.so, building it if needed."""
    global _lib
    if _lib is not None:
        return _lib
    from .build import build, needs_build
    if needs_build():
        if not build_if_missing:
            raise RuntimeError(f"libvlsgpu.so missing or stale at {LIB_PATH}; run viennals_b200/build.py")
        build()
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    i32, i64 = ctypes.c_int32, ctypes.c_int64
    L.vlsg_version.restype = ctypes.c_int
    L.vlsg_last_error.restype = ctypes.c_char_p
    L.vlsg_last_error.argtypes = [vp]
    L.vlsg_create.argtypes = [P(vp), i32, i32]
    L.vlsg_destroy.argtypes = [vp]
    L.vlsg_set_stream.argtypes = [vp, vp]
    L.vlsg_get_stream.argtypes = [vp, P(vp)]
    L.vlsg_default_params.argtypes = [P(AdvectParams)]
    L.vlsg_default_params.restype = None
    L.vlsg_set_grid.argtypes = [vp, i32, P(i64), P(i64), P(i32), ctypes.c_double]
    L.vlsg_set_level_set_count.argtypes = [vp, i32]
    L.vlsg_upload_levelset.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_double), i64,
                                       P(i32), P(ctypes.c_int8), i32]
    L.vlsg_count_points.argtypes = [vp, i32, P(i64)]
    L.vlsg_download_levelset.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_double), P(i32)]
    L.vlsg_get_values.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_double)]
    L.vlsg_set_owned_region.argtypes = [vp, i32, i64, i64]
    L.vlsg_set_reduction_callback.argtypes = [vp, REDUCE_CALLBACK, vp]
    L.vlsg_download_point_data.argtypes = [vp, i32, i64, P(i64), P(ctypes.c_double),
                                           P(ctypes.c_double), P(i32)]
    L.vlsg_download_runs.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_int8), P(i64)]
    L.vlsg_compare.argtypes = [vp, i32, vp, i32, P(CompareResult)]
    L.vlsg_advect_batch.argtypes = [P(vp), i32, P(AdvectParams), P(AdvectResult), i32]
    L.vlsg_batch_set_domains.argtypes = [vp, i32, P(BatchDomain)]
    L.vlsg_batch_advect.argtypes = [vp, P(AdvectParams), P(AdvectResult)]
    L.vlsg_batch_count_points.argtypes = [vp, i32, P(i64)]
    L.vlsg_batch_download.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_double), P(i32)]
    L.vlsg_batch_get_values.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_double)]
    L.vlsg_batch_download_runs.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_int8), P(i64)]
    L.vlsg_get_values_noalloc.argtypes = [vp, i32, i64, P(i32), P(ctypes.c_double)]
    L.vlsg_set_velocity_functor.argtypes = [vp, P(VelocityDesc)]
    L.vlsg_set_velocity_callback.argtypes = [vp, VELOCITY_CALLBACK, vp]
    L.vlsg_set_dissipation_alpha_callback.argtypes = [vp, ALPHA_CALLBACK, vp]
    L.vlsg_set_velocity_update_callback.argtypes = [vp, UPDATE_CALLBACK, vp]
    L.vlsg_prepare_stencil_llf.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]
    L.vlsg_finalize_stencil_llf.argtypes = [vp]
    L.vlsg_prepare_ls.argtypes = [vp, i32]
    L.vlsg_advect.argtypes = [vp, P(AdvectParams), P(AdvectResult)]
    L.vlsg_set_profiling.argtypes = [vp, i32]
    L.vlsg_get_kernel_stats.argtypes = [vp, i32, P(KernelStat), P(i32)]
    _lib = L
    return _lib


EXPORTED = [
    "vlsg_version", "vlsg_last_error", "vlsg_create", "vlsg_destroy",
    "vlsg_default_params", "vlsg_set_stream", "vlsg_get_stream",
    "vlsg_set_grid", "vlsg_set_level_set_count",
    "vlsg_upload_levelset", "vlsg_count_points", "vlsg_download_levelset", "vlsg_download_runs",
    "vlsg_get_values", "vlsg_get_values_noalloc", "vlsg_download_point_data",
    "vlsg_set_velocity_functor", "vlsg_set_velocity_callback",
    "vlsg_set_dissipation_alpha_callback", "vlsg_prepare_stencil_llf", "vlsg_finalize_stencil_llf",
    "vlsg_prepare_ls",
    "vlsg_set_velocity_update_callback", "vlsg_advect", "vlsg_advect_batch",
    "vlsg_set_profiling", "vlsg_get_kernel_stats", "vlsg_compare",
    "vlsg_set_owned_region", "vlsg_set_reduction_callback",
    "vlsg_batch_set_domains", "vlsg_batch_advect", "vlsg_batch_count_points",
    "vlsg_batch_download", "vlsg_batch_get_values", "vlsg_batch_download_runs",
]
