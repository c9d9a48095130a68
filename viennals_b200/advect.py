"""`Advect` -- the drop-in front of viennals::Advect<T,D> (D = 3, or 2) over libvlsgpu.

Same setters, getters and semantics as the reference (lsAdvect.hpp:836-1043,
bound to Python at python/pyWrap.hpp:324-401): level sets are inserted bottom
to top, the last one is advected and must wrap the others, and apply()
writes the results back into the same Domain objects.  Errors that the
reference logs and returns on raise RuntimeError here.
"""
import ctypes

import numpy as np

from . import _lib
from ._abi import (AdvectParams, AdvectResult, KernelStat, Precision,
                   SpatialSchemeEnum, TemporalSchemeEnum)
from .domain import Domain, make_runs, make_runs_2d


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _as3(a):
    """Index rows of a D = 2 domain with a zero third component (the library's
    layout for D = 2); 3-column rows as they are."""
    a = np.asarray(a)
    if a.ndim == 2 and a.shape[1] == 2:
        return np.concatenate([a, np.zeros((len(a), 1), a.dtype)], 1)
    return a


class Context:
    """One libvlsgpu context (device, precision, CUDA stream)."""

    def __init__(self, device=0, precision=Precision.FP64):
        self.lib = _lib.load()
        self.h = ctypes.c_void_p()
        self._check(self.lib.vlsg_create(ctypes.byref(self.h), int(device), int(precision)), None)
        self.precision = Precision(precision)

    def _check(self, rc, h="self"):
        if rc != 0:
            msg = self.lib.vlsg_last_error(self.h if h == "self" else None)
            raise RuntimeError(f"vlsg error {rc}: {msg.decode() if msg else ''}")

    def close(self):
        if self.h:
            self.lib.vlsg_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------
    def set_stream(self, stream_ptr):
        """Run the context's kernels on an external cudaStream_t (int handle)."""
        self._check(self.lib.vlsg_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self.lib.vlsg_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def set_grid(self, grid):
        """vlsg_set_grid; a D = 2 grid (grid.dim 2) takes 2D domains, whose
        indices go to the library with a zero third component and come back
        without it."""
        self._grid = grid
        self._dim = grid.dim
        gmin = np.array(grid.min[:3], np.int64)
        gmax = np.array(grid.max[:3], np.int64)
        bc = np.array(grid.bc[:3], np.int32)
        self._check(self.lib.vlsg_set_grid(self.h, grid.dim, _p(gmin, ctypes.c_int64),
                                           _p(gmax, ctypes.c_int64), _p(bc, ctypes.c_int32),
                                           float(grid.delta)))

    def set_level_set_count(self, n):
        self._check(self.lib.vlsg_set_level_set_count(self.h, int(n)))

    def upload(self, slot, dom):
        idx = np.ascontiguousarray(_as3(dom.idx), np.int32)
        val = np.ascontiguousarray(dom.values, np.float64)
        rs = np.ascontiguousarray(_as3(dom.run_start), np.int32)
        sg = np.ascontiguousarray(dom.run_sign, np.int8)
        self._check(self.lib.vlsg_upload_levelset(
            self.h, int(slot), len(val), _p(idx, ctypes.c_int32), _p(val, ctypes.c_double),
            len(sg), _p(rs, ctypes.c_int32), _p(sg, ctypes.c_int8), int(dom.width)))

    def count(self, slot):
        n = ctypes.c_int64()
        self._check(self.lib.vlsg_count_points(self.h, int(slot), ctypes.byref(n)))
        return n.value

    def download(self, slot, idx_out=None, val_out=None):
        """(idx, values, width) of the defined points in HRLE order.  With
        idx_out ((M,3) int32) and val_out ((M,) float64) of capacity M >= n
        (e.g. pinned host memory), the points land there and views of their
        first n rows are returned."""
        n = self.count(slot)
        planar = getattr(self, "_dim", 3) == 2
        if (not planar and idx_out is not None and val_out is not None and len(idx_out) >= n
                and len(val_out) >= n):
            idx, val = idx_out[:n], val_out[:n]
        else:
            idx = np.empty((n, 3), np.int32)
            val = np.empty(n)
        w = ctypes.c_int32()
        self._check(self.lib.vlsg_download_levelset(self.h, int(slot), n, _p(idx, ctypes.c_int32),
                                                    _p(val, ctypes.c_double), ctypes.byref(w)))
        if planar:
            idx = np.ascontiguousarray(idx[:, :2])
        return idx, val, w.value

    def set_owned_region(self, axis, lo=0, hi=0):
        """vlsg_set_owned_region: only points with index[axis] in [lo, hi)
        count towards the time step, the alphas and the point updates (axis 2;
        -1 owns everything)."""
        self._check(self.lib.vlsg_set_owned_region(self.h, int(axis), int(lo), int(hi)))

    def set_reduction_callback(self, fn):
        """vlsg_set_reduction_callback: fn(values, op) replaces the numpy array
        `values` by its reduction over all shards (op 0 = min, 1 = max).  None
        clears it."""
        from ._abi import REDUCE_CALLBACK

        if fn is None:
            self._reduce_cb = REDUCE_CALLBACK()
        else:
            def cb(user, values, n, op):
                try:
                    arr = np.ctypeslib.as_array(values, shape=(n,))
                    fn(arr, int(op))
                    return 0
                except Exception:  # noqa: BLE001 -- reported as VLSG_ERR_CALLBACK
                    return 1
            self._reduce_cb = REDUCE_CALLBACK(cb)
        self._check(self.lib.vlsg_set_reduction_callback(self.h, self._reduce_cb, None))

    def download_point_data(self, slot):
        """vlsg_download_point_data: (source, velocity, dissipation) of the
        defined points in download order, or None when the level set carries
        no point data."""
        n = self.count(slot)
        src = np.empty(n, np.int64)
        vel = np.empty(n)
        diss = np.empty(n)
        has = ctypes.c_int32()
        self._check(self.lib.vlsg_download_point_data(
            self.h, int(slot), n, _p(src, ctypes.c_int64), _p(vel, ctypes.c_double),
            _p(diss, ctypes.c_double), ctypes.byref(has)))
        return (src, vel, diss) if has.value else None

    def values_at(self, slot, idx):
        idx = np.ascontiguousarray(_as3(idx), np.int32)
        out = np.zeros(len(idx))
        self._check(self.lib.vlsg_get_values(self.h, int(slot), len(idx), _p(idx, ctypes.c_int32),
                                             _p(out, ctypes.c_double)))
        return out

    def compare(self, slot, other, other_slot=0):
        """vlsg_compare of this context's level set (a) against another
        context's (b) on the same device; a dict of vlsg_compare_result."""
        from ._abi import CompareResult
        r = CompareResult()
        self._check(self.lib.vlsg_compare(self.h, int(slot), other.h, int(other_slot), ctypes.byref(r)))
        return r.as_dict()

    def prepare_stencil_llf(self, is_depo):
        """vlsg_prepare_stencil_llf: the top level set becomes the wrapping
        STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER advects."""
        d = (ctypes.c_int32 * max(1, len(is_depo)))(*[1 if x else 0 for x in is_depo])
        self._check(self.lib.vlsg_prepare_stencil_llf(self.h, d, len(is_depo)))

    def finalize_stencil_llf(self):
        self._check(self.lib.vlsg_finalize_stencil_llf(self.h))

    def prepare_ls(self, spatial_scheme):
        """vlsg_prepare_ls: Expand the top level set to the scheme's width."""
        self._check(self.lib.vlsg_prepare_ls(self.h, int(spatial_scheme)))

    def set_velocity(self, desc):
        self._check(self.lib.vlsg_set_velocity_functor(self.h, ctypes.byref(desc)))

    def set_velocity_update_callback(self, fn):
        """setVelocityUpdateCallback: fn(Domain) between RK stages (None clears)."""
        from ._abi import UPDATE_CALLBACK
        self._update_cb = update_callback(fn, getattr(self, "_grid", None)) if fn is not None else None
        self._check(self.lib.vlsg_set_velocity_update_callback(
            self.h, self._update_cb if fn is not None else UPDATE_CALLBACK(), None))

    def set_velocity_callback(self, field):
        """Host callback mode: `field` is a VelocityField (its c_callback())."""
        self._velocity_field = field  # keeps the function pointers alive
        self._check(self.lib.vlsg_set_velocity_callback(self.h, field.c_callback(), None))
        self._check(self.lib.vlsg_set_dissipation_alpha_callback(self.h, field.c_alpha_callback(),
                                                                 None))

    def advect(self, params):
        res = AdvectResult()
        self._check(self.lib.vlsg_advect(self.h, ctypes.byref(params), ctypes.byref(res)))
        return res

    def set_profiling(self, on):
        self._check(self.lib.vlsg_set_profiling(self.h, int(bool(on))))

    def kernel_stats(self):
        cnt = ctypes.c_int32()
        self._check(self.lib.vlsg_get_kernel_stats(self.h, 0, None, ctypes.byref(cnt)))
        arr = (KernelStat * max(1, cnt.value))()
        self._check(self.lib.vlsg_get_kernel_stats(self.h, cnt.value, arr, ctypes.byref(cnt)))
        return [dict(name=arr[i].name.decode(), launches=arr[i].launches,
                     device_ms=arr[i].device_ms, bytes=arr[i].algorithmic_bytes)
                for i in range(cnt.value)]

    def download_runs(self, slot, start_out=None, sign_out=None):
        """(run_start (K,3) int32, run_sign (K,) int8) of the undefined runs in
        HRLE order, built on the device (vlsg_download_runs); optional output
        buffers as for download().  A D = 2 context returns (K,2) starts."""
        if getattr(self, "_dim", 3) == 2:
            starts, signs = self._runs(slot, None, None)
            return np.ascontiguousarray(starts[:, :2]), signs
        return self._runs(slot, start_out, sign_out)

    def _runs(self, slot, start_out, sign_out):
        n = ctypes.c_int64()
        cap = 0
        if start_out is not None and sign_out is not None:
            cap = min(len(start_out), len(sign_out))
            rc = self.lib.vlsg_download_runs(self.h, int(slot), cap, _p(start_out, ctypes.c_int32),
                                             _p(sign_out, ctypes.c_int8), ctypes.byref(n))
            if rc == 0:
                return start_out[:n.value], sign_out[:n.value]
            if rc != -3:
                self._check(rc)
        else:
            rc = self.lib.vlsg_download_runs(self.h, int(slot), 0, None, None, ctypes.byref(n))
            if rc not in (0, -3):
                self._check(rc)
        starts = np.empty((n.value, 3), np.int32)
        signs = np.empty(n.value, np.int8)
        self._check(self.lib.vlsg_download_runs(self.h, int(slot), n.value, _p(starts, ctypes.c_int32),
                                                _p(signs, ctypes.c_int8), ctypes.byref(n)))
        return starts, signs

    def download_domain(self, slot, grid, out=None):
        """Domain with the defined points and the undefined runs, both in HRLE
        order from the device.  `out` may be a Domain whose arrays serve as
        output buffers (capacity permitting)."""
        if out is not None:
            idx, val, w = self.download(slot, out.idx, out.values)
            rs, sg = self.download_runs(slot, out.run_start, out.run_sign)
        else:
            idx, val, w = self.download(slot)
            rs, sg = self.download_runs(slot)
        return Domain(grid, idx, val, rs, sg, width=w)

    def download_domain_host_runs(self, slot, grid):
        """Same as download_domain with the runs rebuilt on the host from
        point queries (the reference layout the device builder follows)."""
        idx, val, w = self.download(slot)
        if getattr(self, "_dim", 3) == 2:
            lo = idx.min(0) - 1 if len(idx) else np.zeros(2, np.int64)
            hi = idx.max(0) + 1 if len(idx) else np.zeros(2, np.int64)

            def sign2(x, y):
                q = np.stack([np.asarray(x), np.asarray(y)], 1).astype(np.int32)
                return np.where(self.values_at(slot, q) < 0, -1, 1)

            rs, sg = make_runs_2d(idx, sign2, lo, hi)
            return Domain(grid, idx, val, rs, sg, width=w)
        if len(idx):
            lo = idx.min(0) - 1
            hi = idx.max(0) + 1
        else:
            lo = np.zeros(3, np.int64)
            hi = np.zeros(3, np.int64)

        def sign_fn(x, y, z):
            q = np.stack([np.asarray(x), np.asarray(y), np.asarray(z)], 1).astype(np.int32)
            v = self.values_at(slot, q)
            return np.where(v < 0, -1, 1)

        rs, sg = make_runs(idx, sign_fn, lo, hi)
        return Domain(grid, idx, val, rs, sg, width=w)


def advect_batch(contexts, params, threads=0):
    """vlsg_advect_batch over a list of Contexts; returns their results."""
    n = len(contexts)
    handles = (ctypes.c_void_p * n)(*[c.h.value for c in contexts])
    results = (AdvectResult * n)()
    lib = _lib.load()
    rc = lib.vlsg_advect_batch(handles, n, ctypes.byref(params), results, int(threads))
    if rc != 0:
        for c in contexts:
            msg = lib.vlsg_last_error(c.h)
            if msg:
                raise RuntimeError(f"vlsg error {rc}: {msg.decode()}")
        raise RuntimeError(f"vlsg error {rc}")
    return list(results)


class BatchContext(Context):
    """The batching form: many independent domains advanced together in one
    context (vlsg_batch_set_domains / vlsg_batch_advect): every pass of a
    time step is one kernel launch over all domains, each domain with its own
    gridDelta, velocity functor and time step."""

    def set_domains(self, items):
        """items: (grid, domain, velocity) triples -- a Grid periodic in x and y
        (extents multiples of 8 points) and infinite in z, its Domain, and a
        FunctorVelocity."""
        from ._abi import BatchDomain, VelocityDesc

        self._grids = []
        keep = []
        arr = (BatchDomain * len(items))()
        for k, (grid, dom, vel) in enumerate(items):
            if grid.dim != 3:
                raise RuntimeError("batching form: three-dimensional domains only")
            gmin = np.array(grid.min[:3], np.int64)
            gmax = np.array(grid.max[:3], np.int64)
            bc = np.array(grid.bc[:3], np.int32)
            idx = np.ascontiguousarray(dom.idx, np.int32)
            val = np.ascontiguousarray(dom.values, np.float64)
            rs = np.ascontiguousarray(dom.run_start, np.int32)
            sg = np.ascontiguousarray(dom.run_sign, np.int8)
            desc = vel.descriptor()
            if not isinstance(desc, VelocityDesc):
                raise RuntimeError("batching form: device velocity functors only")
            keep += [gmin, gmax, bc, idx, val, rs, sg, desc]
            arr[k] = BatchDomain(_p(gmin, ctypes.c_int64), _p(gmax, ctypes.c_int64),
                                 _p(bc, ctypes.c_int32), float(grid.delta), len(val),
                                 _p(idx, ctypes.c_int32), _p(val, ctypes.c_double), len(sg),
                                 _p(rs, ctypes.c_int32), _p(sg, ctypes.c_int8), int(dom.width),
                                 ctypes.pointer(desc))
            self._grids.append(grid)
        self._check(self.lib.vlsg_batch_set_domains(self.h, len(items), arr))
        del keep

    def advect(self, params):
        n = len(self._grids)
        results = (AdvectResult * n)()
        self._check(self.lib.vlsg_batch_advect(self.h, ctypes.byref(params), results))
        return list(results)

    def count(self, domain):
        n = ctypes.c_int64()
        self._check(self.lib.vlsg_batch_count_points(self.h, int(domain), ctypes.byref(n)))
        return n.value

    def download(self, domain, idx_out=None, val_out=None):
        """(idx, values, width) of domain `domain`'s defined points in HRLE
        order, in its own indices."""
        n = self.count(domain)
        idx = np.empty((n, 3), np.int32)
        val = np.empty(n)
        w = ctypes.c_int32()
        self._check(self.lib.vlsg_batch_download(self.h, int(domain), n, _p(idx, ctypes.c_int32),
                                                 _p(val, ctypes.c_double), ctypes.byref(w)))
        return idx, val, w.value

    def values_at(self, domain, idx):
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.zeros(len(idx))
        self._check(self.lib.vlsg_batch_get_values(self.h, int(domain), len(idx),
                                                   _p(idx, ctypes.c_int32), _p(out, ctypes.c_double)))
        return out

    def download_runs(self, domain):
        n = ctypes.c_int64()
        rc = self.lib.vlsg_batch_download_runs(self.h, int(domain), 0, None, None, ctypes.byref(n))
        if rc not in (0, -3):  # -3: the count, with capacity 0
            self._check(rc)
        rs = np.empty((n.value, 3), np.int32)
        sg = np.empty(n.value, np.int8)
        self._check(self.lib.vlsg_batch_download_runs(self.h, int(domain), n.value,
                                                      _p(rs, ctypes.c_int32), _p(sg, ctypes.c_int8),
                                                      ctypes.byref(n)))
        return rs, sg

    def download_domain(self, domain, grid=None, out=None):
        """Domain `domain`: its points and its undefined runs."""
        idx, val, w = self.download(domain)
        rs, sg = self.download_runs(domain)
        return Domain(grid or self._grids[domain], idx, val, rs, sg, width=w)


class Advect:
    """Mirror of viennals::Advect<T,D> running on the GPU (D from the level
    sets' grid: 3, or 2 held as one plane)."""

    velocityLabel = "AdvectionVelocities"
    dissipationLabel = "Dissipation"

    def __init__(self, levelSets=None, velocities=None, precision=Precision.FP64, device=0):
        if isinstance(levelSets, Domain):
            levelSets = [levelSets]
        self.levelSets = list(levelSets) if levelSets else []
        self.velocities = velocities
        self.params = AdvectParams.defaults()
        self.precision = Precision(precision)
        self.device = device
        self.ctx = None
        self.result = AdvectResult()
        self.result.current_time_step = -1.0
        self._resident = None  # (ids, fingerprints) of the level sets on the device

    # setters, lsAdvect.hpp:856-969 ---------------------------------------
    def insertNextLevelSet(self, ls):
        self.levelSets.append(ls)

    def clearLevelSets(self):
        self.levelSets = []

    def setVelocityField(self, v):
        self.velocities = v

    def setAdvectionTime(self, t):
        self.params.advection_time = float(t)

    def setSingleStep(self, b):
        self.params.single_step = int(bool(b))

    def setTimeStepRatio(self, cfl):
        self.params.time_step_ratio = float(cfl)

    def setCalculateNormalVectors(self, b):
        self.params.calculate_normal_vectors = int(bool(b))

    def setIgnoreVoids(self, b):
        self.params.ignore_voids = int(bool(b))

    def setAdaptiveTimeStepping(self, b=True, subdivisions=20):
        self.params.adaptive_time_stepping = int(bool(b))
        self.params.adaptive_subdivisions = max(1, int(subdivisions))

    def setSaveAdvectionVelocities(self, b):
        self.params.save_advection_velocities = int(bool(b))

    def setSpatialScheme(self, s):
        self.params.spatial_scheme = int(SpatialSchemeEnum(s))

    setIntegrationScheme = setSpatialScheme  # deprecated name, lsAdvect.hpp:940-946

    def setTemporalScheme(self, s):
        self.params.temporal_scheme = int(TemporalSchemeEnum(s))

    def setDissipationAlpha(self, a):
        self.params.dissipation_alpha = float(a)

    def setCheckDissipation(self, b):
        self.params.check_dissipation = int(bool(b))

    def setUpdatePointData(self, b):
        self.params.update_point_data = int(bool(b))

    def setVelocityUpdateCallback(self, callback):
        """setVelocityUpdateCallback (lsAdvect.hpp:966-969): callback(Domain)
        with the top level set between the RK2/RK3 stages."""
        self.velocityUpdateCallback = callback

    def setMaxDissipation(self, d):
        """StencilLocalLaxFriedrichsScalar.setMaxDissipation (a class-wide
        static in the reference, per Advect object here)."""
        self.params.max_dissipation = float(d)

    # getters, lsAdvect.hpp:920-932 ---------------------------------------
    def getAdvectedTime(self):
        return self.result.advected_time

    def getCurrentTimeStep(self):
        return self.result.current_time_step

    def getNumberOfTimeSteps(self):
        return self.result.number_of_time_steps

    def getTimeStepRatio(self):
        return self.params.time_step_ratio

    def getCalculateNormalVectors(self):
        return bool(self.params.calculate_normal_vectors)

    # ---------------------------------------------------------------------
    @staticmethod
    def _fingerprint(d):
        return (d.n_points, d.width, hash(d.idx.tobytes()), hash(d.values.tobytes()))

    def _sync_to_device(self, need_velocity=True):
        if not self.levelSets:
            raise RuntimeError("No level sets passed to Advect. Not advecting.")
        if self.velocities is None and need_velocity:
            raise RuntimeError("No velocity field passed to Advect. Not advecting.")
        if self.ctx is None:
            self.ctx = Context(self.device, self.precision)
        key = [id(d) for d in self.levelSets]
        fps = [self._fingerprint(d) for d in self.levelSets]
        if self._resident is None or self._resident != (key, fps):
            grid = self.levelSets[-1].grid
            self.ctx.set_grid(grid)
            self.ctx.set_level_set_count(len(self.levelSets))
            for i, d in enumerate(self.levelSets):
                self.ctx.upload(i, d)
        if self.velocities is not None:
            desc = self.velocities.descriptor()
            if desc is not None:
                self.ctx.set_velocity(desc)
            else:
                self.ctx.set_velocity_callback(self.velocities)
        self.ctx.set_velocity_update_callback(getattr(self, "velocityUpdateCallback", None))

    def _write_back(self, which):
        for i in which:
            d = self.levelSets[i]
            nd = self.ctx.download_domain(i, d.grid)
            d.idx, d.values, d.run_start, d.run_sign, d.width = (
                nd.idx, nd.values, nd.run_start, nd.run_sign, nd.width)
        self._resident = ([id(d) for d in self.levelSets],
                          [self._fingerprint(d) for d in self.levelSets])

    def prepareLS(self):
        """Advect::prepareLS, lsAdvect.hpp:972-1015: the top level set expanded
        to the width the spatial scheme reads, written back."""
        if not self.levelSets:
            raise RuntimeError("No level sets passed to Advect.")
        self._sync_to_device(need_velocity=False)
        self.ctx.prepare_ls(self.params.spatial_scheme)
        self._write_back([len(self.levelSets) - 1])

    def apply(self):
        """Advect::apply, lsAdvect.hpp:1017-1043; results written back.  The top
        level set's point data (Domain.point_data) is carried along as the
        reference's passes translate it; with setSaveAdvectionVelocities it
        gains the "AdvectionVelocities" and "Dissipation" arrays of the last
        value update (lsAdvect.hpp:780-796); with setUpdatePointData(False) it
        is dropped (rebuildLS keeps none, lsAdvect.hpp:418-423)."""
        top = self.levelSets[-1] if self.levelSets else None
        save = bool(self.params.save_advection_velocities)
        track = save or bool(top is not None and top.point_data)
        self.params.track_point_data = int(track)
        self._sync_to_device()
        self.result = self.ctx.advect(self.params)
        old = dict(top.point_data) if top is not None else {}
        self._write_back(range(len(self.levelSets)))
        if track:
            top.point_data = self._translate_point_data(old, save)
        return self.result

    def _translate_point_data(self, old, save):
        pd = self.ctx.download_point_data(len(self.levelSets) - 1)
        if pd is None:
            return {}
        src, vel, diss = pd
        ok = src >= 0
        new = {}
        for label, arr in old.items():
            if save and label in (self.velocityLabel, self.dissipationLabel):
                continue  # replaced by this advection's values
            arr = np.asarray(arr)
            out = np.zeros((len(src),) + arr.shape[1:], arr.dtype)
            out[ok] = arr[src[ok]]
            new[label] = out
        if save:
            new[self.velocityLabel] = vel
            new[self.dissipationLabel] = diss
        return new


def update_callback(fn, grid=None):
    """vlsg_update_cb around fn(Domain): the Domain holds copies of the top
    level set's points and runs (HRLE order); an exception in fn makes the
    call return 1 (VLSG_ERR_CALLBACK)."""
    from ._abi import UPDATE_CALLBACK

    def trampoline(user, view):
        try:
            v = view.contents
            n, m = int(v.n_points), int(v.n_runs)
            a = np.ctypeslib.as_array
            d = Domain.__new__(Domain)
            d.grid = grid
            d.idx = a(v.indices, (n, 3)).copy() if n else np.zeros((0, 3), np.int32)
            d.values = a(v.values, (n,)).copy() if n else np.zeros(0)
            d.run_start = a(v.run_start, (m, 3)).copy() if m else np.zeros((0, 3), np.int32)
            d.run_sign = a(v.run_sign, (m,)).copy() if m else np.zeros(0, np.int8)
            d.width = int(v.width)
            if grid is not None and grid.dim == 2:  # the library's third index is 0
                d.idx = np.ascontiguousarray(d.idx[:, :2])
                d.run_start = np.ascontiguousarray(d.run_start[:, :2])
            fn(d)
            return 0
        except Exception:  # reported through the library's status
            return 1
    return UPDATE_CALLBACK(trampoline)


def _stencil_helper(levelSets, fn, device, precision):
    ctx = Context(device, precision)
    try:
        ctx.set_grid(levelSets[-1].grid)
        ctx.set_level_set_count(len(levelSets))
        for i, d in enumerate(levelSets):
            ctx.upload(i, d)
        fn(ctx)
        nd = ctx.download_domain(len(levelSets) - 1, levelSets[-1].grid)
        top = levelSets[-1]
        top.idx, top.values, top.run_start, top.run_sign, top.width = (
            nd.idx, nd.values, nd.run_start, nd.run_sign, nd.width)
    finally:
        ctx.close()


def PrepareStencilLocalLaxFriedrichs(levelSets, isDepo, device=0, precision=Precision.FP64):
    """viennals::PrepareStencilLocalLaxFriedrichs
    (lsStencilLocalLaxFriedrichsScalar.hpp:423-477) on the GPU: the last
    Domain is replaced by the layer wrapping the Stencil LLF scheme advects."""
    _stencil_helper(levelSets, lambda c: c.prepare_stencil_llf(list(isDepo)), device, precision)


def FinalizeStencilLocalLaxFriedrichs(levelSets, device=0, precision=Precision.FP64):
    """viennals::FinalizeStencilLocalLaxFriedrichs (:480-492) on the GPU."""
    _stencil_helper(levelSets, lambda c: c.finalize_stencil_llf(), device, precision)
