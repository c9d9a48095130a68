"""Benchmark: narrow-band point-updates/s of the level-set advection step.

Workload (one "step" = one RK3 time step, Advect::apply with
advectionTime = 0, over the whole band): the precision form -- a sphere of
radius 40 at gridDelta 0.05 whose radius is modulated by seeded real
spherical harmonics (l <= 8, coefficients ~ N(0, 0.02 R)), velocity
1 + 0.3 n_z, WENO5 + RK3, CFL 0.4, phi stored in FP32 with FP64 time step,
advected time and stage combination.  Inputs are synthetic (seeded), built
on the GPU before the timed region.

value : point-updates/s with the level set resident in HBM (K steps of the
        C ABI's vlsg_advect, timed with CUDA events on the library stream).
e2e   : the same metric through the C ABI with host buffers: every step
        uploads the level set from host memory, advects one step and
        downloads the result.
Multi-GPU (torchrun): replicas -- every rank advects its own copy of the
domain; value = all ranks' point updates / max-over-ranks time.

--impl reference times the CPU restatement of the reference's algorithm
(oracle/, FP64, OpenMP on all host cores) on a bounded sample of the same
workload, since the reference itself cannot be built on this image.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "band point-updates/s WENO5-RK3 FP32 vs FP64 on 1 B200 at stated err; % HBM peak"
UNIT = "point-updates/s"
HBM_PEAK_FALLBACK = 6650.0


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region is short (~0.1 s): start it once nvidia-smi
            # reports, and count only the samples taken from then on
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.005)
            self.samples = []
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        mx = max((float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def reduce_over_ranks(ms, updates, device):
    """Timed-region milliseconds (max over ranks) and point updates (sum over
    ranks) through the initialised process group."""
    import torch

    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    u = torch.tensor([float(updates)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(u)
    return float(t.item()), float(u.item())


def build_workload(args, device):
    from viennals_b200.synth import perturbed_sphere, precision_velocity

    grid, dom = perturbed_sphere(radius=args.radius, grid_delta=args.grid_delta,
                                 seed=args.seed, device=device)
    return grid, dom, precision_velocity()


def params_for(args):
    from viennals_b200 import AdvectParams

    p = AdvectParams.defaults()
    p.spatial_scheme = 11  # WENO_5TH_ORDER
    p.temporal_scheme = 2  # RUNGE_KUTTA_3RD_ORDER
    p.time_step_ratio = 0.4
    p.advection_time = 0.0  # one step per call
    return p


def run_ours(args, rank, world):
    import numpy as np
    import torch

    from viennals_b200.advect import Context
    from viennals_b200._abi import Precision

    dev = torch.device("cuda", args.local_rank)
    torch.cuda.set_device(dev)
    t0 = time.time()
    grid, dom, vel = build_workload(args, f"cuda:{args.local_rank}")
    gen_s = time.time() - t0
    prec = Precision.FP32 if args.precision == "fp32" else Precision.FP64
    stream = torch.cuda.Stream(device=dev)
    ctx = Context(args.local_rank, prec)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_grid(grid)
    ctx.set_level_set_count(1)
    ctx.upload(0, dom)
    ctx.set_velocity(vel.descriptor())
    p = params_for(args)
    for _ in range(args.warmup):
        ctx.advect(p)
    dist = world > 1
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    updates = 0
    launches = 0
    with ClockSampler(args.local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            r = ctx.advect(p)
            updates += r.point_updates
            launches += r.kernel_launches
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        torch.distributed.barrier()
        ms, total_updates = reduce_over_ranks(ms, updates, dev)
        # what follows (profiling step, e2e, precision report, CPU baseline)
        # runs on rank 0 alone and needs no collective: the other ranks leave
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    else:
        total_updates = float(updates)
    value = total_updates / (ms / 1e3)
    out = {"ms": ms, "updates": updates, "value": value, "launches": launches,
           "clocks": clk.summary(), "gen_s": gen_s, "n_points": int(dom.n_points)}

    if rank == 0:
        # per-kernel device times of one more step (events around every
        # launch) -> dominant kernel and its roofline
        ctx.set_profiling(True)
        r = ctx.advect(p)
        stats = ctx.kernel_stats()
        ctx.set_profiling(False)
        out["kernels"] = stats
        out["profile_updates"] = r.point_updates
        # e2e through the C ABI with host buffers: every step uploads the level
        # set from pinned host memory, advects it one step and downloads the
        # result (points and runs) into pinned host memory
        from viennals_b200.domain import Domain

        n_e2e = max(1, min(args.steps, args.e2e_steps))
        host_dom = ctx.download_domain(0, grid)

        def pinned(a, rows):
            t = torch.empty((rows,) + a.shape[1:], dtype=torch.from_numpy(a[:0]).dtype,
                            pin_memory=True)
            arr = t.numpy()
            arr[:len(a)] = a
            return arr, t

        np_, nr_ = len(host_dom.values), len(host_dom.run_sign)
        cp, cr = np_ * 3 // 2 + 4096, nr_ * 3 // 2 + 4096
        (bi, t1), (bv, t2) = pinned(host_dom.idx, cp), pinned(host_dom.values, cp)
        (bs, t3), (bg, t4) = pinned(host_dom.run_start, cr), pinned(host_dom.run_sign, cr)
        out_dom = Domain(grid, bi, bv, bs, bg, width=host_dom.width)
        cur = Domain(grid, bi[:np_], bv[:np_], bs[:nr_], bg[:nr_], width=host_dom.width)
        ctx2 = Context(args.local_rank, prec)
        ctx2.set_stream(stream.cuda_stream)
        ctx2.set_grid(grid)
        ctx2.set_level_set_count(1)
        ctx2.set_velocity(vel.descriptor())
        # untimed warm-up steps (the first ones size the context's buffers)
        for _ in range(max(1, args.warmup)):
            ctx2.upload(0, cur)
            ctx2.advect(p)
            cur = ctx2.download_domain(0, grid, out=out_dom)
        torch.cuda.synchronize()
        e2e_updates = 0
        h2d = d2h = 0
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            h2d += cur.idx.nbytes + cur.values.nbytes + cur.run_start.nbytes + cur.run_sign.nbytes
            ctx2.upload(0, cur)
            r2 = ctx2.advect(p)
            e2e_updates += r2.point_updates
            cur = ctx2.download_domain(0, grid, out=out_dom)
            d2h += cur.idx.nbytes + cur.values.nbytes + cur.run_start.nbytes + cur.run_sign.nbytes
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out["e2e"] = {"value": e2e_updates / wall, "unit": UNIT,
                      "h2d_bytes_per_step": int(h2d // n_e2e), "d2h_bytes_per_step": int(d2h // n_e2e),
                      "steps": n_e2e, "wall_s_per_step": wall / n_e2e,
                      "warmup": max(1, args.warmup), "host_memory": "pinned",
                      "timing": "host wall clock around upload + advect + download"}
        del t1, t2, t3, t4
        ctx2.close()
    ctx.close()
    if rank == 0 and args.err_steps > 0:
        out["precision_report"] = precision_report(args, grid, dom, vel, p, stream)
    if rank == 0 and args.batch_domains > 0:
        try:
            out["batching"] = batching_report(args, f"cuda:{args.local_rank}")
        except Exception as e:  # noqa: BLE001 -- reported in the line, the bench goes on
            out["batching"] = {"error": str(e)[:300]}
    return out


def precision_report(args, grid, dom, vel, p, stream):
    """The FP32 path against the FP64 path on the same input after
    `err_steps` RK3 steps (the precision form runs 50): both timed with CUDA
    events on the same stream, compared on the device (vlsg_compare).  The
    FP64 path is the one the parity tests hold bit-identical to the FP64
    oracle."""
    import torch

    from viennals_b200.advect import Context
    from viennals_b200._abi import Precision

    res = {}

    def run(prec, compensation=0, dom_in=None):
        p.fp32_compensation = compensation
        c = Context(args.local_rank, prec)
        c.set_stream(stream.cuda_stream)
        c.set_grid(grid)
        c.set_level_set_count(1)
        c.upload(0, dom if dom_in is None else dom_in)
        c.set_velocity(vel.descriptor())
        c.count(0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        upd = 0
        e0.record(stream)
        for _ in range(args.err_steps):
            upd += c.advect(p).point_updates
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        return c, {"point_updates_per_s": upd / (ms / 1e3), "ms_per_step": ms / args.err_steps}

    # each path timed alone on the device; the FP32 result crosses to the
    # host and back (exact: FP32 values are doubles on the way) so that both
    # results are resident for the comparison
    c32, res["fp32"] = run(Precision.FP32)
    out32 = c32.download_domain(0, grid)
    c32.close()
    c32c, res["fp32c"] = run(Precision.FP32, 1)
    out32c = c32c.download_domain(0, grid)
    c32c.close()
    p.fp32_compensation = 0
    c64, res["fp64"] = run(Precision.FP64)

    def against64(dom):
        c = Context(args.local_rank, Precision.FP64)  # the FP32 result, exactly
        c.set_grid(grid)
        c.set_level_set_count(1)
        c.upload(0, dom)
        r = c.compare(0, c64, 0)
        c.close()
        return r

    r = against64(out32)
    rc = against64(out32c)
    # the reference algorithm's own sensitivity: the FP64 path started from
    # the input rounded to FP32 (one rounding of each value, no FP32
    # arithmetic), against the FP64 path from the exact input
    import numpy as np

    from viennals_b200.domain import Domain

    rounded = Domain(grid, dom.idx, dom.values.astype(np.float32).astype(np.float64),
                     dom.run_start, dom.run_sign, width=dom.width)
    c64r, _ = run(Precision.FP64, dom_in=rounded)
    rr = c64r.compare(0, c64, 0)
    c64r.close()
    c64.close()
    gd = float(grid.delta)
    vol64, vol32 = r["inside_cells_b"], r["inside_cells_a"]
    comp = {
        "fp32_point_updates_per_s": res["fp32c"]["point_updates_per_s"],
        "fp32_ms_per_step": res["fp32c"]["ms_per_step"],
        "max_abs_dphi_over_gridDelta": rc["max_abs_diff"],
        "rms_abs_dphi_over_gridDelta": rc["rms_abs_diff"],
        "points_with_abs_dphi_above": dict(zip(["1e-6", "1e-5", "1e-4", "1e-3"], rc["diff_above"])),
        "active_set_differences": rc["active_only_a"] + rc["active_only_b"],
        "defined_set_differences": rc["defined_only_a"] + rc["defined_only_b"],
        "chamfer_rms": rc["chamfer_rms"] * gd, "chamfer_max": rc["chamfer_max"] * gd,
    }
    return {
        "steps": args.err_steps, "against": "FP64 GPU path (bit-identical to the FP64 oracle "
        "in the parity tests)",
        "fp32_point_updates_per_s": res["fp32"]["point_updates_per_s"],
        "fp64_point_updates_per_s": res["fp64"]["point_updates_per_s"],
        "fp32_ms_per_step": res["fp32"]["ms_per_step"], "fp64_ms_per_step": res["fp64"]["ms_per_step"],
        "fp32_over_fp64": res["fp32"]["point_updates_per_s"] / res["fp64"]["point_updates_per_s"],
        "max_abs_dphi_over_gridDelta": r["max_abs_diff"], "rms_abs_dphi_over_gridDelta": r["rms_abs_diff"],
        "points_with_abs_dphi_above": dict(zip(["1e-6", "1e-5", "1e-4", "1e-3"], r["diff_above"])),
        "common_points": r["common_points"],
        "active_points_fp32": r["active_a"], "active_points_fp64": r["active_b"],
        "active_set_differences": r["active_only_a"] + r["active_only_b"],
        "defined_set_differences": r["defined_only_a"] + r["defined_only_b"],
        "inside_cells_fp32": vol32, "inside_cells_fp64": vol64,
        "rel_volume_error": (vol32 - vol64) / vol64 if vol64 else None,
        "chamfer_rms": r["chamfer_rms"] * gd, "chamfer_max": r["chamfer_max"] * gd,
        "chamfer_mean": r["chamfer_mean"] * gd, "chamfer_unit": "length (gridDelta x grid units)",
        "surface_nodes_fp32": r["nodes_a"], "surface_nodes_fp64": r["nodes_b"],
        "compensated": comp,
        "fp64_from_fp32_rounded_input": {
            "what": "FP64 path from the input values rounded to FP32 once, against the FP64 "
                    "path from the exact input (no FP32 arithmetic anywhere)",
            "max_abs_dphi_over_gridDelta": rr["max_abs_diff"],
            "rms_abs_dphi_over_gridDelta": rr["rms_abs_diff"],
            "points_with_abs_dphi_above": dict(zip(["1e-6", "1e-5", "1e-4", "1e-3"], rr["diff_above"])),
            "active_set_differences": rr["active_only_a"] + rr["active_only_b"],
            "defined_set_differences": rr["defined_only_a"] + rr["defined_only_b"],
            "chamfer_rms": rr["chamfer_rms"] * gd, "chamfer_max": rr["chamfer_max"] * gd,
        },
    }


def batching_report(args, device):
    """The batching form: `args.batch_domains` seeded plane domains with a
    trench or a hole (bands of 1e4..2e6 points, log-uniform), LLF 1st order,
    RK2, FP32, per-domain rates in [0.2, 1.5]; one RK2 step of every domain
    advanced three ways: one context after another (loop), vlsg_advect_batch
    (host threads, one stream per context) and the batch context (every pass
    one launch over all domains, per-domain time steps on the device, the
    step replayed from a CUDA graph).  Each way is warmed by two steps and
    the third is timed by the host clock around it; all three must end
    identical."""
    import numpy as np
    import torch

    from viennals_b200 import AdvectParams
    from viennals_b200._abi import Precision
    from viennals_b200.advect import BatchContext, Context, advect_batch
    from viennals_b200.synth import batch_domains

    t0 = time.time()
    doms = batch_domains(args.batch_domains, seed=7, device=device)
    gen_s = time.time() - t0
    p = AdvectParams.defaults()
    p.spatial_scheme = 7  # LOCAL_LAX_FRIEDRICHS_1ST_ORDER
    p.temporal_scheme = 1  # RUNGE_KUTTA_2ND_ORDER
    p.advection_time = 0.0

    def contexts():
        out = []
        for grid, dom, vel in doms:
            c = Context(args.local_rank, Precision.FP32)
            c.set_grid(grid)
            c.set_level_set_count(1)
            c.upload(0, dom)
            c.set_velocity(vel.descriptor())
            out.append(c)
        return out

    def run(mode):
        # one set of contexts at a time: 256 contexts hold tens of GB
        if mode == "batch":
            b = BatchContext(args.local_rank, Precision.FP32)
            b.set_domains(doms)
            cs = None
            step = lambda: b.advect(p)  # noqa: E731
        else:
            cs = contexts()
            step = ((lambda: advect_batch(cs, p, threads=args.batch_threads)) if mode == "threads"
                    else (lambda: [c.advect(p) for c in cs]))
        try:
            step()  # sizes the buffers
            step()  # the batch context captures its step into a CUDA graph here
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = step()
            torch.cuda.synchronize()
            secs = time.perf_counter() - t0
            upd = sum(r.point_updates for r in res)
            launches = (res[0].kernel_launches if mode == "batch"
                        else sum(r.kernel_launches for r in res))
            got = ([b.download(d)[:2] for d in range(len(doms))] if mode == "batch"
                   else [c.download(0)[:2] for c in cs])
        finally:
            if cs:
                for c in cs:
                    c.close()
            else:
                b.close()
            torch.cuda.empty_cache()
        return upd, secs, got, launches

    upd_loop, loop_s, got_loop, l_loop = run("loop")
    upd_thr, thr_s, got_thr, l_thr = run("threads")
    upd_b, b_s, got_b, l_b = run("batch")

    def same(a, b):
        return all(x[0].shape == y[0].shape and bool((x[0] == y[0]).all()) and
                   bool((x[1].view(np.int64) == y[1].view(np.int64)).all()) for x, y in zip(a, b))

    pts = [d.n_points for _, d, _ in doms]
    return {"domains": len(doms), "band_points_total": int(sum(pts)),
            "band_points_min": int(min(pts)), "band_points_max": int(max(pts)),
            "scheme": "LLF1 + RK2, FP32, one step per domain",
            "loop_ms": loop_s * 1e3, "threads_ms": thr_s * 1e3, "batch_ms": b_s * 1e3,
            "threads": args.batch_threads,
            "loop_point_updates_per_s": upd_loop / loop_s,
            "threads_point_updates_per_s": upd_thr / thr_s,
            "batch_point_updates_per_s": upd_b / b_s,
            "batch_over_loop": loop_s / b_s, "threads_over_loop": loop_s / thr_s,
            "kernel_launches": {"loop": l_loop, "threads": l_thr, "batch": l_b},
            "identical": bool(upd_loop == upd_thr == upd_b and same(got_loop, got_thr)
                              and same(got_loop, got_b)),
            "generation_s": gen_s, "timing": "host clock around one step of every domain"}


def deposition_report(args):
    """Config 5, the stacked deposition over a periodic hole array: (1024 x
    tiles)^2 lateral cells at gridDelta 0.02 (tiles 4: the stated 4096^2,
    64 x 64 holes of radius 0.5 and depth 2.0), three level sets, rates
    1.0 / 0.6 / 0.0 + 0.2 |n_z|, WENO5 + RK3, CFL 0.4, 20 steps, FP32.  The
    input is the 1024^2 workload tiled (synth.tiled_hole_stack), so every
    1024^2 tile of the result must equal the FP32 1024^2 run bit for bit
    (checked on the four corner tiles).  The 20 steps are timed with CUDA
    events on the context's stream."""
    import numpy as np
    import torch

    from viennals_b200 import AdvectParams
    from viennals_b200._abi import Precision
    from viennals_b200.advect import Context
    from viennals_b200.domain import lex_order
    from viennals_b200.synth import tiled_hole_stack

    dev = f"cuda:{args.local_rank}"
    t0 = time.time()
    grid, doms, vel, grid_s, doms_s = tiled_hole_stack(args.deposition_tiles, 1024, device=dev)
    gen_s = time.time() - t0
    p = AdvectParams.defaults()
    p.spatial_scheme = 11  # WENO_5TH_ORDER
    p.temporal_scheme = 2  # RUNGE_KUTTA_3RD_ORDER
    p.time_step_ratio = 0.4
    p.advection_time = 1.0
    p.single_step = 1
    steps = 20

    def run(g, ds, timed):
        stream = torch.cuda.Stream(device=dev)
        c = Context(args.local_rank, Precision.FP32)
        c.set_stream(stream.cuda_stream)
        c.set_grid(g)
        c.set_level_set_count(len(ds))
        for i, d in enumerate(ds):
            c.upload(i, d)
        c.set_velocity(vel.descriptor())
        c.count(len(ds) - 1)  # builds the layout before the timed region
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        upd = 0
        t = 0.0
        e0.record(stream)
        for _ in range(steps):
            r = c.advect(p)
            upd += r.point_updates
            t += r.advected_time
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        used = torch.cuda.mem_get_info()[1] - min(free0, torch.cuda.mem_get_info()[0])
        out = [c.download(i)[:2] for i in range(len(ds))]
        c.close()
        return out, {"ms": ms, "updates": upd, "time": t, "device_bytes_used": int(used)}

    big, rb = run(grid, doms, True)
    small, rs = run(grid_s, doms_s, False)
    n, tiles = 1024, args.deposition_tiles
    half_big = tiles * n // 2
    same = rb["time"] == rs["time"]
    for (bi, bv), (si, sv) in zip(big, small):
        same &= len(bi) == tiles * tiles * len(si)
        for a, b in ((0, 0), (0, tiles - 1), (tiles - 1, 0), (tiles - 1, tiles - 1)):
            x0, y0 = -half_big + n * a, -half_big + n * b
            m = (bi[:, 0] >= x0) & (bi[:, 0] < x0 + n) & (bi[:, 1] >= y0) & (bi[:, 1] < y0 + n)
            ti = bi[m].astype(np.int64)
            ti[:, 0] -= x0 + n // 2
            ti[:, 1] -= y0 + n // 2
            o = lex_order(ti)
            same &= bool(np.array_equal(ti[o], si)) and bool(
                np.array_equal(bv[m][o].view(np.int64), sv.view(np.int64)))
    return {"workload": f"stacked deposition over a periodic hole array, {tiles * n}^2 lateral "
                        f"cells at gridDelta 0.02 ({tiles * 16} x {tiles * 16} holes, r 0.5, depth "
                        f"2.0), 3 level sets, rates 1.0/0.6/0.0 + 0.2|n_z|, WENO5 + RK3, CFL 0.4, "
                        f"FP32, {steps} steps",
            "band_points_per_level_set": [int(d.n_points) for d in doms],
            "point_updates": int(rb["updates"]), "ms": rb["ms"],
            "point_updates_per_s": rb["updates"] / (rb["ms"] / 1e3),
            "advected_time": rb["time"], "device_bytes_used": rb["device_bytes_used"],
            "tiles_equal_the_1024_run": bool(same), "generation_s": gen_s,
            "timing": "CUDA events around the 20 vlsg_advect calls on the context stream"}


def cpu_baseline(args, sample_radius, steps=1, threads=None):
    """The oracle (FP64 restatement, OpenMP) on a bounded sample: the same
    workload at a smaller radius, `steps` RK3 steps each timed on its own.
    value = the median of the per-step point-updates/s."""
    from oracle import oracle as O
    from viennals_b200.synth import perturbed_sphere, precision_velocity

    cores = threads or os.cpu_count() or 1
    O.set_threads(cores)
    grid, dom = perturbed_sphere(radius=sample_radius, grid_delta=args.grid_delta,
                                 seed=args.seed, device="cuda" if _has_cuda() else "cpu")
    ls = O.OracleLS(grid, dom)
    p = params_for(args)
    runs = []
    for _ in range(steps):
        t0 = time.perf_counter()
        r = O.advect([ls], p, precision_velocity())
        runs.append(r.point_updates / (time.perf_counter() - t0))
    runs_sorted = sorted(runs)
    return {"value": runs_sorted[len(runs) // 2], "unit": UNIT, "cores": cores, "kind": "port",
            "runs": runs, "band_points": int(dom.n_points), "radius": sample_radius,
            "sample": (f"perturbed sphere R={sample_radius} at gridDelta {args.grid_delta} "
                       f"({dom.n_points} band points), WENO5+RK3 CFL 0.4, v=1+0.3 n_z, "
                       f"median of {steps} single-step run(s) on {cores} host thread(s), FP64 "
                       f"oracle restatement (the reference cannot be built here)")}


def cpu_baseline_line(args, steps):
    """All host threads on the R `cpu_sample_radius` sample (median of
    `steps` runs) and one thread on the smaller R `cpu_single_radius` sample."""
    cb = cpu_baseline(args, args.cpu_sample_radius, steps=steps)
    one = cpu_baseline(args, args.cpu_single_radius, steps=1, threads=1)
    out = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    out["runs"] = cb["runs"]
    out["single_thread"] = {k: one[k] for k in ("value", "unit", "cores", "sample")}
    return out, cb


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# DRAM traffic per launch of the dominant kernel from one ncu capture of the
# default workload (its summary sits under profiles/ with the command).
TRAFFIC_PROFILE = {"expand": "expand_pass_dram_fp32_sphere_r40.md"}
PROFILES_DIR = os.path.join(ROOT, "profiles")


def default_workload(args):
    return (args.radius == 40.0 and args.grid_delta == 0.05 and args.seed == 1234
            and args.precision == "fp32")


# The sources of the kernel the traffic figure belongs to: a figure captured
# from other sources is stale and not quoted.
TRAFFIC_SOURCES = ["viennals_b200/csrc/vlsg_frontier.cuh", "viennals_b200/csrc/vlsg_passes.cuh",
                   "viennals_b200/csrc/vlsg_common.cuh"]


def kernel_sources_hash():
    import hashlib

    h = hashlib.sha256()
    for f in TRAFFIC_SOURCES:
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def profiled_traffic(kernel, with_stamp=False):
    """DRAM bytes per launch from the committed ncu summary of `kernel`, with
    the commit it was captured at; None when the summary's kernel sources
    differ from the current ones."""
    name = TRAFFIC_PROFILE.get(kernel)
    if not name:
        return (None, None) if with_stamp else None
    vals = {}
    try:
        with open(os.path.join(PROFILES_DIR, name)) as f:
            for line in f:
                for key in ("traffic_bytes_per_launch", "kernel_sources_sha256", "captured_at_commit"):
                    if line.startswith(key + ":"):
                        vals[key] = line.split(":", 1)[1].strip()
    except OSError:
        return (None, None) if with_stamp else None
    t = vals.get("traffic_bytes_per_launch")
    if t is None or vals.get("kernel_sources_sha256") != kernel_sources_hash():
        return (None, None) if with_stamp else None
    return (float(t), vals.get("captured_at_commit")) if with_stamp else float(t)


def roofline(out, peaks, args=None):
    """Dominant kernel: device time share; achieved = its algorithmic bytes /
    its average launch time.  traffic = ncu DRAM bytes per launch of that
    kernel on the default workload (null for other workloads)."""
    ks = out.get("kernels") or []
    if not ks:
        return None
    top = max(ks, key=lambda k: k["device_ms"])
    hbm = peaks.get("hbm_gbs") if peaks else None
    src = "measured" if hbm else "fallback"
    hbm = hbm or HBM_PEAK_FALLBACK
    per_launch_ms = top["device_ms"] / max(1, top["launches"])
    bytes_per_launch = top["bytes"] / max(1, top["launches"])
    achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9 if per_launch_ms > 0 else 0.0
    total = sum(k["device_ms"] for k in ks)
    traffic, stamp = (profiled_traffic(top["name"], with_stamp=True)
                      if args and default_workload(args) else (None, None))
    return {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": hbm,
            "peak_source": src, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, mean per launch, "
                               f"captured at commit {stamp}" if traffic is not None else
                               "no ncu capture of the current kernel sources for this workload"),
            "share": top["device_ms"] / total if total else None,
            "launch_ms": per_launch_ms}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--radius", type=float, default=40.0)
    ap.add_argument("--grid-delta", type=float, default=0.05)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-sample-radius", type=float, default=8.0)
    ap.add_argument("--cpu-single-radius", type=float, default=4.0,
                    help="sample radius of the single-thread CPU figure")
    ap.add_argument("--cpu-runs", type=int, default=5,
                    help="single-step oracle runs behind the cpu_baseline median")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-domains", type=int, default=256,
                    help="domains of the batching-form report (0: skip)")
    ap.add_argument("--batch-threads", type=int, default=16)
    ap.add_argument("--deposition-tiles", type=int, default=0,
                    help="run only the deposition workload at (1024 x tiles)^2 lateral cells")
    ap.add_argument("--err-steps", type=int, default=50,
                    help="RK3 steps of the FP32-vs-FP64 precision report (0: skip)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    args.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = {"workload": f"perturbed sphere R={args.radius} gridDelta={args.grid_delta} "
                       f"(seed {args.seed}), WENO5+RK3, CFL 0.4, v=1+0.3 n_z",
           "precision": args.precision, "step": "one RK3 time step (3 FE stages + 2 combines)",
           "l2": "inputs larger than L2 (band ~17M points, ~1.3 GB of values per buffer at R 40)", "parallelism": f"replicas x{world}"}

    if args.deposition_tiles > 0:
        print(json.dumps({"metric": "deposition point-updates/s (FP32)",
                          "deposition": deposition_report(args)}))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        # K single-step runs of the oracle on all host threads (median), plus
        # one single-thread run on a smaller sample
        cbl, cb = cpu_baseline_line(args, max(1, args.steps))
        ref_cfg = dict(cfg)
        ref_cfg["workload"] = (f"perturbed sphere R={cb['radius']} gridDelta={args.grid_delta} "
                               f"(seed {args.seed}, {cb['band_points']} band points), WENO5+RK3, "
                               f"CFL 0.4, v=1+0.3 n_z")
        ref_cfg["sample_of"] = cfg["workload"]
        ref_cfg["precision"] = "fp64"
        ref_cfg["l2"] = "CPU run (no GPU)"
        ref_cfg["timing"] = f"median of {max(1, args.steps)} single-step runs"
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "config": ref_cfg,
                "cpu_baseline": cbl,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        torch.cuda.set_device(args.local_rank)
        # collectives: barriers and reductions around the timed region only
        torch.distributed.init_process_group(
            "nccl", timeout=__import__("datetime").timedelta(seconds=120))
    out = run_ours(args, rank, world)
    if rank != 0:
        return
    peaks = measured_peaks()
    line = {"metric": METRIC, "value": out["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["ms"] / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic", "config": cfg, "gpu_launches": out["launches"],
            "clocks": out["clocks"], "e2e": out.get("e2e"),
            "roofline": roofline(out, peaks, args), "band_points": out["n_points"],
            "precision_report": out.get("precision_report"),
            "batching": out.get("batching"),
            "kernels": out.get("kernels")}
    if not args.no_cpu_baseline:
        line["cpu_baseline"], _ = cpu_baseline_line(args, args.cpu_runs)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
