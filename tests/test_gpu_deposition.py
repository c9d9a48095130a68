"""The stacked-deposition workload: three stacked level sets over a periodic
hole array (substrate with holes of radius 0.5 and depth 2.0 at pitch 1.28,
two slabs on the flat top; gridDelta 0.02), velocities 1.0 / 0.6 / 0.0 plus
0.2 |n_z| per material, WENO5 + RK3, 20 time steps, FP32 against the FP64
GPU path (the oracle is too slow at this size).  The hole axes lie on grid
points, so cells at exactly the hole radius hold values of order 1e-9.  The
lateral extent is
1024 x 1024 cells (16 x 16 holes, about 12M points per level set at width
2); the 4096^2 extent holds about 200M points per level set because the
hole walls dominate, beyond one GPU for both precisions and three level
sets with their RK copies."""
import pytest


def advect_steps(grid, doms, vel, p, precision, steps):
    from viennals_b200.advect import Context

    ctx = Context(0, precision)
    ctx.set_grid(grid)
    ctx.set_level_set_count(len(doms))
    for i, d in enumerate(doms):
        ctx.upload(i, d)
    ctx.set_velocity(vel.descriptor())
    t = 0.0
    updates = 0
    for _ in range(steps):
        r = ctx.advect(p)
        t += r.advected_time
        updates += r.point_updates
    return ctx, t, updates


@pytest.mark.gpu
def test_deposition_hole_stack_fp32_vs_fp64():
    from parity_cases import params
    from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
    from viennals_b200.synth import hole_stack

    grid, doms, vel = hole_stack(lateral_cells=1024, device="cuda")
    p = params(S.WENO_5TH_ORDER, TS.RUNGE_KUTTA_3RD_ORDER, 1.0, cfl=0.4, single_step=1)
    c64, t64, u64 = advect_steps(grid, doms, vel, p, 0, 20)
    c32, t32, u32 = advect_steps(grid, doms, vel, p, 1, 20)
    print(f"\ndeposition (1024^2): points {[d.n_points for d in doms]}, time fp64 {t64:.6f} "
          f"fp32 {t32:.6f}, point updates {u64} / {u32}")
    assert abs(t32 - t64) <= 1e-4 * t64
    for i in range(3):
        r = c32.compare(i, c64, i)
        print(f"level set {i}: common {r['common_points']}, max |dphi| {r['max_abs_diff']:.3e}, "
              f"rms {r['rms_abs_diff']:.3e}, active {r['active_a']}/{r['active_b']} "
              f"(differ {r['active_only_a'] + r['active_only_b']}), above 1e-3 "
              f"{r['diff_above'][3]}, inside {r['inside_cells_a']}/{r['inside_cells_b']}, "
              f"chamfer rms {r['chamfer_rms']:.3e}")
        # the bound max |dphi| <= 1e-3 (grid units), identical point and active
        # sets, volume and surface distance
        assert r["defined_only_a"] + r["defined_only_b"] == 0
        assert r["active_only_a"] + r["active_only_b"] == 0
        assert r["max_abs_diff"] <= 1e-3
        assert abs(r["inside_cells_a"] - r["inside_cells_b"]) <= 1e-6 * r["inside_cells_b"]
        assert r["chamfer_rms"] <= 1e-5


@pytest.mark.gpu
def test_deposition_hole_stack_2048_fp32_tiles():
    """FP32 at 2048^2 lateral cells (32 x 32 holes, four times the area of
    the FP64 comparison above; the full 4096^2 extent is bench.py's
    --deposition-tiles 4 run).  The input is the 1024^2 workload tiled 2 x 2
    (the hole period divides 1024 cells), so after 20 steps every 1024^2
    tile of the 2048^2 run must equal the 1024^2 run bit for bit: nothing in
    a step depends on where a point lies."""
    import time

    import numpy as np

    from parity_cases import params
    from viennals_b200 import SpatialSchemeEnum as S, TemporalSchemeEnum as TS
    from viennals_b200.domain import lex_order
    from viennals_b200.synth import tiled_hole_stack

    p = params(S.WENO_5TH_ORDER, TS.RUNGE_KUTTA_3RD_ORDER, 1.0, cfl=0.4, single_step=1)
    grid_l, doms_l, vel, grid_s, doms_s = tiled_hole_stack(2, 1024, device="cuda")
    n = 1024
    small, t_s, _ = advect_steps(grid_s, doms_s, vel, p, 1, 20)
    small_pts = [small.download(i)[:2] for i in range(3)]
    small.close()
    t0 = time.perf_counter()
    large, t_l, upd = advect_steps(grid_l, doms_l, vel, p, 1, 20)
    secs = time.perf_counter() - t0
    assert t_l == t_s
    for i in range(3):
        idx, val, _ = large.download(i)
        si, sv = small_pts[i]
        assert len(idx) == 4 * len(si)
        for a in range(2):
            for b in range(2):
                m = ((idx[:, 0] >= n * a - n) & (idx[:, 0] < n * a) &
                     (idx[:, 1] >= n * b - n) & (idx[:, 1] < n * b))
                ti = idx[m].copy()
                ti[:, 0] -= n * a - n // 2
                ti[:, 1] -= n * b - n // 2
                o = lex_order(ti)
                assert np.array_equal(ti[o], si)
                assert np.array_equal(val[m][o].view(np.int64), sv.view(np.int64))
    print(f"\ndeposition FP32 2048^2: points {[d.n_points for d in doms_l]}, "
          f"{upd} point updates in {secs:.1f} s (20 RK3 steps, host loop included)")
    large.close()
