"""Host logic of bench.py on CPU: the roofline entry, the committed traffic
figure it quotes, and the reference arm's JSON line (the oracle on a small
sample of the workload)."""
import json
import os
import subprocess
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _args(**kw):
    a = types.SimpleNamespace(radius=40.0, grid_delta=0.05, seed=1234, precision="fp32")
    a.__dict__.update(kw)
    return a


def test_roofline_picks_the_dominant_kernel():
    out = {"kernels": [
        {"name": "expand", "launches": 19, "device_ms": 8.3, "bytes": 13.3e9},
        {"name": "rates", "launches": 3, "device_ms": 2.8, "bytes": 0.67e9},
    ]}
    r = bench.roofline(out, {"hbm_gbs": 6456.5}, _args())
    assert r["kernel"] == "expand" and r["bound"] == "hbm" and r["unit"] == "GB/s"
    per_launch_s = 8.3 / 19 / 1e3
    assert abs(r["achieved"] - 13.3e9 / 19 / per_launch_s / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / 6456.5) < 1e-12
    assert r["peak_source"] == "measured"
    assert r["traffic"] == bench.profiled_traffic("expand")
    assert (r["traffic"] is None) == ("captured at" not in r["traffic_source"])
    assert abs(r["share"] - 8.3 / 11.1) < 1e-12
    # other workloads quote no traffic; no peaks file -> the fallback peak
    r2 = bench.roofline(out, None, _args(radius=24.0))
    assert r2["traffic"] is None and r2["peak_source"] == "fallback"
    assert bench.roofline({"kernels": []}, None) is None


def test_profiled_traffic_is_the_committed_figure(tmp_path, monkeypatch):
    # the committed summary, when it was captured from the current sources
    t = bench.profiled_traffic("expand")
    assert t is None or 4e8 < t < 1.2e9  # bytes per Expand launch at R 40
    assert bench.profiled_traffic("rates") is None
    # a summary is quoted with its commit only while the kernel sources match
    name = bench.TRAFFIC_PROFILE["expand"]
    monkeypatch.setattr(bench, "PROFILES_DIR", str(tmp_path))
    (tmp_path / name).write_text("traffic_bytes_per_launch: 7.5e8\n"
                                 f"kernel_sources_sha256: {bench.kernel_sources_hash()}\n"
                                 "captured_at_commit: abc123\n")
    assert bench.profiled_traffic("expand", with_stamp=True) == (7.5e8, "abc123")
    (tmp_path / name).write_text("traffic_bytes_per_launch: 7.5e8\n"
                                 "kernel_sources_sha256: 0000000000000000\n")
    assert bench.profiled_traffic("expand") is None


def test_reference_arm_line():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "3", "--warmup", "0", "--cpu-sample-radius", "2.0",
                        "--cpu-single-radius", "1.5"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == bench.UNIT
    assert line["metric"] == bench.METRIC and line["higher_is_better"] is True
    assert line["value"] > 0 and line["value"] == line["cpu_baseline"]["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT,
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the labels name what ran: the sample's radius and band, FP64, a median
    cfg, cb = line["config"], line["cpu_baseline"]
    assert "R=2.0" in cfg["workload"] and "band points" in cfg["workload"]
    assert "R=40.0" in cfg["sample_of"] and cfg["precision"] == "fp64"
    assert line["dtype"] == "f64" and "median of 3" in cfg["timing"]
    assert len(cb["runs"]) == 3 and cb["value"] == sorted(cb["runs"])[1]
    assert cb["single_thread"]["cores"] == 1 and cb["single_thread"]["value"] > 0
