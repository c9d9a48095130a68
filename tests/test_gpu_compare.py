"""vlsg_compare (the device comparison used for the FP32-vs-FP64 precision
report) against the same figures computed with numpy / scipy from the
downloaded points."""
import numpy as np
import pytest

from parity_cases import egg_velocity, params, run_gpu, sphere_case

pytestmark = pytest.mark.gpu


def _keys(idx):
    off = 1 << 20
    i = idx.astype(np.int64) + off
    return (i[:, 2] << 42) | (i[:, 1] << 21) | i[:, 0]


def _nodes(idx, val):
    """Edge zero-crossing nodes (grid units), the rule of kSurfaceNodes."""
    k = _keys(idx)
    out = []
    for d in range(3):
        nb = idx.copy()
        nb[:, d] += 1
        kn = _keys(nb)
        j = np.searchsorted(k, kn)
        j = np.minimum(j, len(k) - 1)
        found = k[j] == kn
        d0, d1 = val, val[j]
        cross = found & ((d0 >= 0) != (d1 >= 0))
        c = idx[cross].astype(np.float64)
        a, b = d0[cross], d1[cross]
        base = c[:, d]
        cc = np.where(a == -b, base + 0.5,
                      np.where(np.abs(a) <= np.abs(b), base + a / (a - b), base + 1 - b / (b - a)))
        cc = np.minimum(np.maximum(cc, base + 1e-12), base + 1 - 1e-12)
        c[:, d] = cc
        out.append(c)
    return np.concatenate(out)


def _reference(ia, va, ib, vb):
    from scipy.spatial import cKDTree

    ka, kb = _keys(ia), _keys(ib)
    common, pa, pb = np.intersect1d(ka, kb, assume_unique=True, return_indices=True)
    diff = np.abs(va[pa] - vb[pb])
    act_a, act_b = np.abs(va) <= 0.5, np.abs(vb) <= 0.5
    both_a = np.zeros(len(ka), bool)
    both_a[pa] = act_b[pb]
    both_b = np.zeros(len(kb), bool)
    both_b[pb] = act_a[pa]
    na, nb = _nodes(ia, va), _nodes(ib, vb)
    dab = cKDTree(nb).query(na)[0]
    dba = cKDTree(na).query(nb)[0]
    return {
        "common_points": len(common), "defined_only_a": len(ka) - len(common),
        "defined_only_b": len(kb) - len(common), "active_a": int(act_a.sum()),
        "active_b": int(act_b.sum()), "active_only_a": int((act_a & ~both_a).sum()),
        "active_only_b": int((act_b & ~both_b).sum()), "max_abs_diff": float(diff.max()),
        "rms_abs_diff": float(np.sqrt(np.mean(diff ** 2))), "nodes_a": len(na), "nodes_b": len(nb),
        "chamfer_ab": float(dab.mean()), "chamfer_ba": float(dba.mean()),
        "chamfer_max": float(max(dab.max(), dba.max())),
        "chamfer_rms": float(np.sqrt((np.sum(dab ** 2) + np.sum(dba ** 2)) / (len(dab) + len(dba)))),
        "diff_above": [int((diff > t).sum()) for t in (1e-6, 1e-5, 1e-4, 1e-3)],
    }


def test_compare_fp32_against_fp64_matches_numpy():
    g, lss = sphere_case(4.0, 0.3)
    p = params(11, 2, 0.6, cfl=0.4)
    c64, _ = run_gpu(g, lss, egg_velocity(), p, precision=0)
    c32, _ = run_gpu(g, lss, egg_velocity(), p, precision=1)
    got = c32.compare(0, c64, 0)
    ia, va, _ = c32.download(0)
    ib, vb, _ = c64.download(0)
    ref = _reference(ia, va, ib, vb)
    for k in ("common_points", "defined_only_a", "defined_only_b", "active_a", "active_b",
              "active_only_a", "active_only_b", "nodes_a", "nodes_b", "diff_above"):
        assert got[k] == ref[k], k
    assert got["points_a"] == len(va) and got["points_b"] == len(vb)
    assert got["max_abs_diff"] == ref["max_abs_diff"]
    for k in ("rms_abs_diff", "chamfer_ab", "chamfer_ba", "chamfer_max", "chamfer_rms"):
        assert got[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-12), k
    assert got["chamfer_unresolved"] == 0
    # the FP32 path stays close to the FP64 one
    assert got["max_abs_diff"] < 1e-3
    assert abs(got["inside_cells_a"] - got["inside_cells_b"]) <= 0.001 * got["inside_cells_b"]


def test_compare_identical_and_volume():
    g, lss = sphere_case(5.0, 0.25)
    a, _ = run_gpu(g, lss, egg_velocity(), params(0, 0, 0.25))
    b, _ = run_gpu(g, lss, egg_velocity(), params(0, 0, 0.25))
    r = a.compare(0, b, 0)
    assert r["defined_only_a"] == 0 and r["defined_only_b"] == 0
    assert r["active_only_a"] == 0 and r["active_only_b"] == 0
    assert r["max_abs_diff"] == 0.0 and r["chamfer_max"] == 0.0
    assert r["inside_cells_a"] == r["inside_cells_b"]
    # the uploaded sphere: about 4/3 pi R^3 cells (R = 20 cells)
    from viennals_b200.advect import Context

    c = Context()
    c.set_grid(g)
    c.set_level_set_count(1)
    c.upload(0, lss[0])
    v = c.compare(0, c, 0)["inside_cells_a"]
    assert abs(v - 4.0 / 3.0 * np.pi * 20 ** 3) < 0.03 * 4.0 / 3.0 * np.pi * 20 ** 3
