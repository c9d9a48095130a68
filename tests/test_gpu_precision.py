"""The precision form on the perturbed-sphere workload at a reduced radius:
radius 16 at gridDelta 0.05 (320 cells, about 2.7M band points), radius
modulated by seeded real spherical harmonics l <= 8 with coefficients
~ N(0, 0.02 R), v = 1 + 0.3 n_z, WENO5 + RK3, CFL 0.4, 50 time steps.  The
FP32 path (phi stored in FP32, stencils in FP32, FP64 time step, advected
time, value update and stage combination, rounded to FP32 or kept with a
compensation term) against the FP64 path,
which the parity tests hold bit-identical to the FP64 oracle.

Bound (in grid units, i.e. max |dphi| / gridDelta): <= 1e-3, and the same
active points (defined, |phi| <= 0.5) after the last step."""
import pytest

pytestmark = pytest.mark.gpu

STEPS = 50


def _context(grid, dom, vel, precision):
    from viennals_b200.advect import Context

    c = Context(0, precision)
    c.set_grid(grid)
    c.set_level_set_count(1)
    c.upload(0, dom)
    c.set_velocity(vel.descriptor())
    return c


@pytest.mark.parametrize("compensation", [0, 1], ids=["rounded", "compensated"])
def test_precision_form_radius_16_fifty_rk3_steps(compensation):
    from viennals_b200 import AdvectParams
    from viennals_b200.synth import perturbed_sphere, precision_velocity

    grid, dom = perturbed_sphere(radius=16.0, grid_delta=0.05, seed=1234, device="cuda")
    vel = precision_velocity()
    p = AdvectParams.defaults()
    p.spatial_scheme = 11  # WENO_5TH_ORDER
    p.temporal_scheme = 2  # RUNGE_KUTTA_3RD_ORDER
    p.time_step_ratio = 0.4
    p.advection_time = 0.0  # one step per call
    p.fp32_compensation = compensation
    c32, c64 = _context(grid, dom, vel, 1), _context(grid, dom, vel, 0)
    t32 = t64 = 0.0
    for _ in range(STEPS):
        r32, r64 = c32.advect(p), c64.advect(p)
        t32 += r32.advected_time
        t64 += r64.advected_time
    r = c32.compare(0, c64, 0)
    print(f"\nR 16, {STEPS} RK3 steps: max |dphi| {r['max_abs_diff']:.3e} (grid units), "
          f"above 1e-6/1e-5/1e-4/1e-3: {r['diff_above']}, active {r['active_a']}/"
          f"{r['active_b']}, defined-only {r['defined_only_a']}/{r['defined_only_b']}, "
          f"time {t32:.9f}/{t64:.9f}")
    assert r["common_points"] > 2_000_000
    assert r["max_abs_diff"] <= 1e-3
    assert r["active_only_a"] == 0 and r["active_only_b"] == 0
    assert r["active_a"] == r["active_b"]
    # advected time: FP64 CFL reduction over FP32 rates
    assert abs(t32 - t64) <= 1e-6 * t64
    assert abs(r["inside_cells_a"] - r["inside_cells_b"]) <= 1e-6 * r["inside_cells_b"]
