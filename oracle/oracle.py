"""ctypes wrapper of the oracle (oracle/libvlso.so).

TEST INFRASTRUCTURE ONLY: the FP64 CPU restatement of ViennaLS 5.8.3's
advection path that checks the CUDA library.  Only tests/, the smoke() of
__graft_entry__ and the CPU-baseline leg of bench.py import this module.
"""
import ctypes
import os
import subprocess

import numpy as np

from viennals_b200._abi import (ALPHA_CALLBACK, REDUCE_CALLBACK, UPDATE_CALLBACK, VELOCITY_CALLBACK,
                                AdvectParams, AdvectResult, VelocityDesc)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libvlso.so")
SOURCES = ["vlso_api.cpp", "vlso_core.hpp", "vlso_advect.hpp", "vlso_metrics.hpp"]


def build(force=False):
    """Compile the oracle with g++ (-ffp-contract=off keeps FP64 bit-exact)."""
    newest = max(os.path.getmtime(os.path.join(HERE, s)) for s in SOURCES)
    newest = max(newest, os.path.getmtime(os.path.join(HERE, "..", "include", "vlsg.h")))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC",
           "-shared", os.path.join(HERE, "vlso_api.cpp"), "-o", LIB]
    subprocess.check_call(cmd)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, i64, i32, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
        P = ctypes.POINTER
        L.vlso_ls_new.restype = vp
        L.vlso_ls_new.argtypes = [i32, P(i64), P(i64), P(ctypes.c_int32), dbl]
        L.vlso_ls_free.argtypes = [vp]
        L.vlso_ls_copy.restype = vp
        L.vlso_ls_copy.argtypes = [vp]
        L.vlso_ls_set.argtypes = [vp, i64, P(ctypes.c_int32), P(dbl), i64,
                                  P(ctypes.c_int32), P(ctypes.c_int8), i32]
        L.vlso_ls_get.restype = i64
        L.vlso_ls_get.argtypes = [vp, i32, P(ctypes.c_int32), P(dbl)]
        L.vlso_ls_width.argtypes = [vp]
        L.vlso_set_shard.argtypes = [i32, i64, i64, REDUCE_CALLBACK, vp]
        L.vlso_set_shard.restype = None
        L.vlso_point_data.restype = i64
        L.vlso_point_data.argtypes = [vp, P(i64), P(dbl), P(dbl)]
        L.vlso_void_markers.restype = i64
        L.vlso_void_markers.argtypes = [vp, P(ctypes.c_uint8)]
        L.vlso_ls_set_width.argtypes = [vp, i32]
        L.vlso_ls_far_queries.restype = i64
        L.vlso_ls_far_queries.argtypes = [vp]
        L.vlso_ls_values_at.argtypes = [vp, i64, P(ctypes.c_int32), P(dbl)]
        L.vlso_expand.argtypes = [vp, i32]
        L.vlso_reduce.argtypes = [vp, i32]
        L.vlso_prune.argtypes = [vp, i32]
        L.vlso_rebuild.argtypes = [vp, dbl, i32]
        L.vlso_boolean.argtypes = [vp, vp, i32]
        L.vlso_check.restype = i64
        L.vlso_check.argtypes = [vp]
        L.vlso_chamfer.argtypes = [vp, vp, P(dbl), P(i64)]
        L.vlso_surface_nodes.restype = i64
        L.vlso_surface_nodes.argtypes = [vp, P(dbl), i64]
        L.vlso_advect.argtypes = [P(vp), i32, P(AdvectParams), P(VelocityDesc),
                                  P(AdvectResult)]
        L.vlso_advect_cb.argtypes = [P(vp), i32, P(AdvectParams), VELOCITY_CALLBACK, vp,
                                     ALPHA_CALLBACK, vp, P(AdvectResult)]
        L.vlso_advect_ex.argtypes = [P(vp), i32, P(AdvectParams), P(VelocityDesc), VELOCITY_CALLBACK,
                                     vp, ALPHA_CALLBACK, vp, UPDATE_CALLBACK, vp, P(AdvectResult)]
        L.vlso_prepare_stencil_llf.argtypes = [P(vp), i32, P(ctypes.c_int32), i32]
        L.vlso_finalize_stencil_llf.argtypes = [P(vp), i32]
        L.vlso_last_error.restype = ctypes.c_char_p
        L.vlso_set_threads.argtypes = [i32]
        L.vlso_get_threads.restype = i32
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().vlso_last_error().decode())


_shard_cb = None


def set_shard(axis=-1, lo=0, hi=0, reduce=None):
    """Owned z-slab and cross-shard reduction of the following advections:
    reduce(values (numpy array, changed in place), op) with op 0 = min,
    1 = max."""
    global _shard_cb
    if reduce is None:
        _shard_cb = REDUCE_CALLBACK()
    else:
        def cb(user, values, n, op):
            try:
                arr = np.ctypeslib.as_array(values, shape=(n,))
                reduce(arr, int(op))
                return 0
            except Exception:  # noqa: BLE001 -- reported to the C side as a failure
                return 1
        _shard_cb = REDUCE_CALLBACK(cb)
    lib().vlso_set_shard(int(axis), int(lo), int(hi), _shard_cb, None)


def set_threads(n):
    lib().vlso_set_threads(int(n))


class OracleLS:
    """One level set held by the oracle."""

    def __init__(self, grid, domain=None, _handle=None):
        self.grid = grid
        L = lib()
        if _handle is not None:
            self.h = _handle
        else:
            D = grid.dim
            gmin = np.array(grid.min, np.int64)
            gmax = np.array(grid.max, np.int64)
            bc = np.array(grid.bc, np.int32)
            self.h = L.vlso_ls_new(D, _ptr(gmin, ctypes.c_int64), _ptr(gmax, ctypes.c_int64),
                                   _ptr(bc, ctypes.c_int32), grid.delta)
        if domain is not None:
            self.set(domain)

    def __del__(self):
        try:
            if self.h:
                lib().vlso_ls_free(self.h)
        except Exception:
            pass

    def copy(self):
        return OracleLS(self.grid, _handle=lib().vlso_ls_copy(self.h))

    def set(self, dom):
        idx = np.ascontiguousarray(dom.idx, np.int32)
        val = np.ascontiguousarray(dom.values, np.float64)
        rs = np.ascontiguousarray(dom.run_start, np.int32)
        sg = np.ascontiguousarray(dom.run_sign, np.int8)
        _check(lib().vlso_ls_set(self.h, len(val), _ptr(idx, ctypes.c_int32),
                                 _ptr(val, ctypes.c_double), len(sg),
                                 _ptr(rs, ctypes.c_int32), _ptr(sg, ctypes.c_int8),
                                 int(dom.width)))

    def points(self, which=0):
        """(idx, values) of the defined points (which=0) or the whole map."""
        L = lib()
        n = L.vlso_ls_get(self.h, which, None, None)
        idx = np.zeros((n, self.grid.dim), np.int32)
        val = np.zeros(n)
        L.vlso_ls_get(self.h, which, _ptr(idx, ctypes.c_int32), _ptr(val, ctypes.c_double))
        return idx, val

    def values_at(self, idx):
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.zeros(len(idx))
        _check(lib().vlso_ls_values_at(self.h, len(idx), _ptr(idx, ctypes.c_int32),
                                       _ptr(out, ctypes.c_double)))
        return out

    def point_data(self):
        """(source, velocity, dissipation) of the defined points in the order
        of points(0), or None when the level set carries no point data."""
        L = lib()
        n = L.vlso_point_data(self.h, None, None, None)
        if n < 0:
            return None
        src = np.zeros(n, np.int64)
        vel = np.zeros(n)
        diss = np.zeros(n)
        L.vlso_point_data(self.h, _ptr(src, ctypes.c_int64), _ptr(vel, ctypes.c_double),
                          _ptr(diss, ctypes.c_double))
        return src, vel, diss

    def void_markers(self):
        """MarkVoidPoints (default options) markers of the defined points, in
        the order of points(0)."""
        L = lib()
        n = L.vlso_void_markers(self.h, None)
        out = np.zeros(n, np.uint8)
        L.vlso_void_markers(self.h, _ptr(out, ctypes.c_uint8))
        return out.astype(bool)

    @property
    def width(self):
        return lib().vlso_ls_width(self.h)

    @property
    def far_queries(self):
        return lib().vlso_ls_far_queries(self.h)

    def expand(self, w):
        _check(lib().vlso_expand(self.h, int(w)))

    def reduce(self, w):
        _check(lib().vlso_reduce(self.h, int(w)))

    def prune(self, remove_stray_zeros=False):
        _check(lib().vlso_prune(self.h, int(remove_stray_zeros)))

    def rebuild(self, cutoff=1.0, width=2):
        _check(lib().vlso_rebuild(self.h, float(cutoff), int(width)))

    def boolean(self, other, op):
        _check(lib().vlso_boolean(self.h, other.h, int(op)))

    def check(self):
        return lib().vlso_check(self.h)

    def surface_nodes(self):
        n = lib().vlso_surface_nodes(self.h, None, 0)
        out = np.zeros((n, self.grid.dim))
        lib().vlso_surface_nodes(self.h, _ptr(out, ctypes.c_double), n)
        return out


def chamfer(target, sample):
    """forward, backward, chamfer, rms, max (lsCompareChamfer.hpp:104-242)."""
    out = np.zeros(5)
    cnt = np.zeros(2, np.int64)
    _check(lib().vlso_chamfer(target.h, sample.h, _ptr(out, ctypes.c_double),
                              _ptr(cnt, ctypes.c_int64)))
    return dict(forward=out[0], backward=out[1], chamfer=out[2], rms=out[3],
                max=out[4], n_target=int(cnt[0]), n_sample=int(cnt[1]))


def advect(level_sets, params, velocity, update=None):
    """Advect::apply on the oracle; level_sets bottom..top (modified).
    `update`: a velocity-update callback fn(Domain) (points only)."""
    arr = (ctypes.c_void_p * len(level_sets))(*[ls.h for ls in level_sets])
    res = AdvectResult()
    desc = velocity.descriptor() if hasattr(velocity, "descriptor") else velocity
    if update is not None:
        from viennals_b200.advect import update_callback
        ucb = update_callback(update)
        if desc is None:
            vcb, acb, dptr = velocity.c_callback(), velocity.c_alpha_callback(), None
        else:
            vcb, acb, dptr = VELOCITY_CALLBACK(), ALPHA_CALLBACK(), ctypes.byref(desc)
        _check(lib().vlso_advect_ex(arr, len(level_sets), ctypes.byref(params), dptr, vcb, None,
                                    acb, None, ucb, None, ctypes.byref(res)))
        return res
    if desc is None:  # a host velocity field: one callback per point
        _check(lib().vlso_advect_cb(arr, len(level_sets), ctypes.byref(params),
                                    velocity.c_callback(), None, velocity.c_alpha_callback(),
                                    None, ctypes.byref(res)))
        return res
    _check(lib().vlso_advect(arr, len(level_sets), ctypes.byref(params),
                             ctypes.byref(desc), ctypes.byref(res)))
    return res


def prepare_stencil_llf(level_sets, is_depo):
    """PrepareStencilLocalLaxFriedrichs on the oracle (top level set replaced)."""
    arr = (ctypes.c_void_p * len(level_sets))(*[ls.h for ls in level_sets])
    d = np.asarray([1 if x else 0 for x in is_depo], dtype=np.int32)
    _check(lib().vlso_prepare_stencil_llf(arr, len(level_sets), _ptr(d, ctypes.c_int32), len(d)))


def finalize_stencil_llf(level_sets):
    """FinalizeStencilLocalLaxFriedrichs on the oracle."""
    arr = (ctypes.c_void_p * len(level_sets))(*[ls.h for ls in level_sets])
    _check(lib().vlso_finalize_stencil_llf(arr, len(level_sets)))
