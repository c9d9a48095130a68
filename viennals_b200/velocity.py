"""Velocity fields: the device functor of vlsg.h and host callbacks.

`VelocityField` mirrors viennals::VelocityField<T> (lsVelocityField.hpp:11-41).
A `FunctorVelocity` (coefficients only) runs entirely on the GPU
(vlsg_set_velocity_functor); any other subclass overrides getScalarVelocity /
getVectorVelocity (one point at a time, as the reference calls them) or
`batch` (numpy arrays of queries) and is called back from the host with
batches of points (vlsg_set_velocity_callback).
"""
import ctypes

import numpy as np

from ._abi import ALPHA_CALLBACK, MAX_MATERIALS, VELOCITY_CALLBACK, VelocityDesc


class VelocityField:
    """Base class with the reference's defaults (zero velocity)."""

    def getScalarVelocity(self, coordinate, material, normalVector, pointId):
        return 0.0

    def getVectorVelocity(self, coordinate, material, normalVector, pointId):
        return (0.0, 0.0, 0.0)

    def getDissipationAlpha(self, direction, material, centralDifferences):
        return 0.0

    def descriptor(self):
        """Return a VelocityDesc when the field is a device functor, else None."""
        return None

    def batch(self, coords, materials, normals, point_ids, scalar_out, vector_out):
        """Velocities of n queries: coords (n, 3), materials (n,), normals
        (n, 3), point_ids (n,) in; scalar_out (n,) and vector_out (n, 3) out.
        The default asks getScalarVelocity / getVectorVelocity per query."""
        for i in range(len(materials)):
            c = (float(coords[i, 0]), float(coords[i, 1]), float(coords[i, 2]))
            n = (float(normals[i, 0]), float(normals[i, 1]), float(normals[i, 2]))
            m, pid = int(materials[i]), int(point_ids[i])
            scalar_out[i] = self.getScalarVelocity(c, m, n, pid)
            vector_out[i, :] = self.getVectorVelocity(c, m, n, pid)

    def c_callback(self):
        """The vlsg_velocity_cb function pointer of this field (kept alive by
        the field).  An exception in `batch` makes the call return 1, which
        the library reports as VLSG_ERR_CALLBACK."""
        cb = getattr(self, "_c_callback", None)
        if cb is None:
            def trampoline(user, n, coords, materials, normals, point_ids, s_out, v_out):
                try:
                    n = int(n)
                    if n <= 0:
                        return 0
                    a = np.ctypeslib.as_array
                    self.batch(a(coords, (n, 3)), a(materials, (n,)), a(normals, (n, 3)),
                               a(point_ids, (n,)), a(s_out, (n,)), a(v_out, (n, 3)))
                    return 0
                except Exception as e:  # reported through the library's status
                    self.last_callback_error = repr(e)
                    return 1
            cb = VELOCITY_CALLBACK(trampoline)
            self._c_callback = cb
        return cb

    def alpha_batch(self, directions, materials, central_differences, alpha_out):
        """getDissipationAlpha of n queries: directions (n,), materials (n,),
        central_differences (n, 3) in; alpha_out (n,) out."""
        for i in range(len(materials)):
            cd = (float(central_differences[i, 0]), float(central_differences[i, 1]),
                  float(central_differences[i, 2]))
            alpha_out[i] = self.getDissipationAlpha(int(directions[i]), int(materials[i]), cd)

    def c_alpha_callback(self):
        """The vlsg_alpha_cb function pointer of this field."""
        cb = getattr(self, "_c_alpha_callback", None)
        if cb is None:
            def trampoline(user, n, directions, materials, cd, out):
                try:
                    n = int(n)
                    if n <= 0:
                        return 0
                    a = np.ctypeslib.as_array
                    self.alpha_batch(a(directions, (n,)), a(materials, (n,)), a(cd, (n, 3)),
                                     a(out, (n,)))
                    return 0
                except Exception as e:  # reported through the library's status
                    self.last_callback_error = repr(e)
                    return 1
            cb = ALPHA_CALLBACK(trampoline)
            self._c_alpha_callback = cb
        return cb


class FunctorVelocity(VelocityField):
    """Per-material polynomial in the unit normal, evaluated on the device.

    For material m (clamped to the last entry) and normal n:
        scalar = rate[m] + sum_k c_lin[m][k](n_k) * n_k
                         + sum_k c_abs[m][k](n_k) * |n_k|
                         + sum_k c_sq [m][k](n_k) * n_k^2
    where each c(n_k) takes its `pos` coefficient for n_k > 0 and its `neg`
    one otherwise; zero coefficients are skipped.  vector = vec[m].
    """

    def __init__(self, n_materials=1):
        if not 1 <= n_materials <= MAX_MATERIALS:
            raise ValueError("n_materials out of range")
        self.n = n_materials
        z3 = lambda: [[0.0, 0.0, 0.0] for _ in range(n_materials)]
        self.rate = [0.0] * n_materials
        self.lin_pos, self.lin_neg = z3(), z3()
        self.abs_pos, self.abs_neg = z3(), z3()
        self.sq_pos, self.sq_neg = z3(), z3()
        self.vec = z3()
        self.alpha = z3()

    # convenience builders -------------------------------------------------
    def set_rate(self, material, rate):
        self.rate[material] = float(rate)
        return self

    def set_linear(self, material, axis, coeff, coeff_neg=None):
        self.lin_pos[material][axis] = float(coeff)
        self.lin_neg[material][axis] = float(coeff if coeff_neg is None else coeff_neg)
        return self

    def set_abs(self, material, axis, coeff_pos, coeff_neg=None):
        self.abs_pos[material][axis] = float(coeff_pos)
        self.abs_neg[material][axis] = float(coeff_pos if coeff_neg is None else coeff_neg)
        return self

    def set_square(self, material, axis, coeff_pos, coeff_neg=None):
        self.sq_pos[material][axis] = float(coeff_pos)
        self.sq_neg[material][axis] = float(coeff_pos if coeff_neg is None else coeff_neg)
        return self

    def set_dissipation_alpha(self, material, direction, alpha):
        """getDissipationAlpha(direction, material, .) = alpha (constant)."""
        self.alpha[material][direction] = float(alpha)
        return self

    def set_vector(self, material, v):
        self.vec[material] = [float(v[0]), float(v[1]), float(v[2])]
        return self

    def _m(self, material):
        return min(max(material, 0), self.n - 1)

    def getScalarVelocity(self, coordinate, material, normalVector, pointId):
        m = self._m(material)
        s = self.rate[m]
        n = normalVector
        for tab_pos, tab_neg, f in (
            (self.lin_pos, self.lin_neg, lambda x: x),
            (self.abs_pos, self.abs_neg, abs),
            (self.sq_pos, self.sq_neg, lambda x: x * x),
        ):
            for k in range(3):
                c = tab_pos[m][k] if n[k] > 0 else tab_neg[m][k]
                if c != 0:
                    s = s + c * f(n[k])
        return s

    def getVectorVelocity(self, coordinate, material, normalVector, pointId):
        return tuple(self.vec[self._m(material)])

    def getDissipationAlpha(self, direction, material, centralDifferences):
        return self.alpha[self._m(material)][direction]

    def descriptor(self):
        d = VelocityDesc()
        d.n_materials = self.n
        for m in range(self.n):
            d.rate[m] = self.rate[m]
            for k in range(3):
                d.lin_pos[m][k] = self.lin_pos[m][k]
                d.lin_neg[m][k] = self.lin_neg[m][k]
                d.abs_pos[m][k] = self.abs_pos[m][k]
                d.abs_neg[m][k] = self.abs_neg[m][k]
                d.sq_pos[m][k] = self.sq_pos[m][k]
                d.sq_neg[m][k] = self.sq_neg[m][k]
                d.vec[m][k] = self.vec[m][k]
                d.alpha[m][k] = self.alpha[m][k]
        return d


def constant_scalar(v, n_materials=1):
    f = FunctorVelocity(n_materials)
    for m in range(n_materials):
        f.set_rate(m, v)
    return f


def constant_vector(vec, n_materials=1):
    f = FunctorVelocity(n_materials)
    for m in range(n_materials):
        f.set_vector(m, vec)
    return f
