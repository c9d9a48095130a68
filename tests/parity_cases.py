"""Parity cases shared by the GPU tests and smoke(): inputs, parameters and
the comparison of the CUDA path with the oracle."""
import numpy as np

from viennals_b200 import AdvectParams, BoundaryConditionEnum as BC, Grid
from viennals_b200.geometry import make_sphere, trench_etch_level_sets
from viennals_b200.velocity import FunctorVelocity, constant_scalar, constant_vector


def egg_velocity():
    """Advection.cpp:25-44: 1 + (n_x > 0 ? 2.3 : 0.5) * n_x^2."""
    v = FunctorVelocity(1)
    v.set_rate(0, 1.0)
    v.set_square(0, 0, 2.3, 0.5)
    return v


def sphere_case(radius=5.0, delta=0.25, origin=(0.0, 0.0, 0.0)):
    g = Grid([-10, 10, -10, 10, -10, 10], [BC.INFINITE_BOUNDARY] * 3, delta)
    return g, [make_sphere(g, list(origin), radius)]


def params(spatial=0, temporal=0, time=0.0, cfl=0.4999, **kw):
    p = AdvectParams.defaults()
    p.spatial_scheme = spatial
    p.temporal_scheme = temporal
    p.advection_time = time
    p.time_step_ratio = cfl
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def sphere_growth_eo1():
    """Sphere R 5 at gridDelta 0.25, v = +1, EO1, FE, CFL 0.5, t = 2."""
    g, ls = sphere_case(5.0, 0.25)
    return g, ls, constant_scalar(1.0), params(0, 0, 2.0, cfl=0.5)


def trench_case(scheme=8, temporal=2, time=0.2, opening=1.6):
    g = Grid([-2.4, 2.4, -2.4, 2.4, -1.6, 1.6],
             [BC.PERIODIC_BOUNDARY, BC.PERIODIC_BOUNDARY, BC.INFINITE_BOUNDARY], 0.1)
    m, t = trench_etch_level_sets(g, 0.5, opening)
    v = FunctorVelocity(2)
    v.set_rate(1, -1.0)
    v.set_linear(1, 2, -0.3)
    return g, [m, t], v, params(scheme, temporal, time)


def run_oracle(grid, level_sets, velocity, p):
    from oracle import oracle as O

    ols = [O.OracleLS(grid, d) for d in level_sets]
    res = O.advect(ols, p, velocity)
    return ols, res


def run_gpu(grid, level_sets, velocity, p, precision=0, profile=False):
    from viennals_b200.advect import Context

    ctx = Context(0, precision)
    ctx.set_grid(grid)
    ctx.set_level_set_count(len(level_sets))
    for i, d in enumerate(level_sets):
        ctx.upload(i, d)
    desc = velocity.descriptor()
    if desc is None:  # a host velocity field: callback mode
        ctx.set_velocity_callback(velocity)
    else:
        ctx.set_velocity(desc)
    if profile:
        ctx.set_profiling(True)
    res = ctx.advect(p)
    return ctx, res


def compare(ols, ctx, exact=True, atol=0.0):
    """Defined points identical (indices), values bit-identical (or within
    atol), signs of the oracle's undefined shell identical."""
    report = []
    for i, o in enumerate(ols):
        oi, ov = o.points(0)
        gi, gv, _ = ctx.download(i)
        if oi.shape != gi.shape or not np.array_equal(oi, gi):
            so = set(map(tuple, oi.tolist()))
            sg = set(map(tuple, gi.tolist()))
            raise AssertionError(
                f"level set {i}: active/defined point sets differ: oracle {len(so)}, gpu {len(sg)}, "
                f"only oracle {len(so - sg)}, only gpu {len(sg - so)}; e.g. {sorted(so ^ sg)[:5]}")
        if exact:
            bad = np.nonzero(ov.view(np.int64) != gv.view(np.int64))[0]
            if len(bad):
                raise AssertionError(
                    f"level set {i}: {len(bad)} values differ bitwise, max |d| = "
                    f"{np.max(np.abs(ov[bad] - gv[bad])):.3e} at {oi[bad[0]].tolist()}")
        else:
            d = np.max(np.abs(ov - gv)) if len(ov) else 0.0
            if d > atol:
                raise AssertionError(f"level set {i}: max |dphi| {d} > {atol}")
        mi, mv = o.points(1)
        und = ~(np.abs(mv) < 1e300)
        if und.any():
            dv = ctx.values_at(i, mi[und])
            if not np.array_equal(np.sign(dv), np.sign(mv[und])) or np.any(np.abs(dv) < 1e300):
                raise AssertionError(f"level set {i}: undefined shell signs differ")
        report.append((len(oi), int(und.sum())))
    return report
