"""vlsg_get_values_noalloc (the query entry point that allocates no device
memory) against vlsg_get_values, through the C ABI, on two calls in a row.

Both entry points run the same query kernel, so the values must be
bit-identical (the tolerance of every FP64 parity test here is zero)."""
import ctypes

import numpy as np
import pytest

from parity_cases import egg_velocity, params, sphere_case

VLSG_ERR_CAPACITY = -3
VLSG_ERR_STATE = -4
MAX_QUERIES = 65536  # VLSG_NOALLOC_MAX_QUERIES


def _query(ctx, fn, idx):
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.empty(len(idx), dtype=np.float64)
    rc = fn(ctx.h, 0, len(idx), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return rc, out


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def _queries(ctx, n, seed):
    """Half defined points of the band, half random indices around it and far
    outside it (undefined regions of both signs, outside the brick box)."""
    band, _, _ = ctx.download(0)
    rng = np.random.default_rng(seed)
    nb = min(len(band), n // 2)
    pick = band[rng.choice(len(band), nb, replace=False)]
    rnd = rng.integers(-120, 121, size=(n - nb, 3), dtype=np.int32)
    q = np.concatenate([pick, rnd])
    return q[rng.permutation(len(q))]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_get_values_twice(precision):
    from viennals_b200.advect import Context

    g, lss = sphere_case(5.0, 0.25)
    ctx = Context(0, precision)
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, lss[0])
    ctx.set_velocity(egg_velocity().descriptor())
    ctx.advect(params(11, 2, 0.5))
    L = ctx.lib
    # two calls in a row, different sizes and contents; the second fills the
    # staging array to its maximum
    for n, seed in ((20000, 1), (MAX_QUERIES, 2)):
        q = _queries(ctx, n, seed)
        rc_ref, ref = _query(ctx, L.vlsg_get_values, q)
        assert rc_ref == 0, L.vlsg_last_error(ctx.h)
        free_before = _free_bytes()
        rc, got = _query(ctx, L.vlsg_get_values_noalloc, q)
        assert rc == 0, L.vlsg_last_error(ctx.h)
        # the staging array was placed at set-up: the call takes no memory
        assert _free_bytes() == free_before
        assert np.array_equal(got, ref)
        assert np.array_equal(np.signbit(got), np.signbit(ref))
        assert np.isfinite(got).all()
        assert (np.abs(got) < 1).sum() > 0 and (got == np.finfo(np.float64).max).sum() > 0


@pytest.mark.gpu
def test_noalloc_rejects_oversize_and_unbuilt():
    from viennals_b200.advect import Context

    g, lss = sphere_case(3.0, 0.5)
    ctx = Context(0, 0)
    ctx.set_grid(g)
    ctx.set_level_set_count(1)
    ctx.upload(0, lss[0])
    L = ctx.lib
    q = np.zeros((4, 3), dtype=np.int32)
    rc, _ = _query(ctx, L.vlsg_get_values_noalloc, q)
    assert rc == VLSG_ERR_STATE
    assert b"not on the device" in L.vlsg_last_error(ctx.h)
    n_points = ctx.count(0)  # moves the level set to the device
    assert n_points > 0
    big = np.zeros((MAX_QUERIES + 1, 3), dtype=np.int32)
    rc, _ = _query(ctx, L.vlsg_get_values_noalloc, big)
    assert rc == VLSG_ERR_CAPACITY
    assert b"maximum of 65536" in L.vlsg_last_error(ctx.h)
    rc, got = _query(ctx, L.vlsg_get_values_noalloc, q)
    assert rc == 0
    rc_ref, ref = _query(ctx, L.vlsg_get_values, q)
    assert rc_ref == 0 and np.array_equal(got, ref)
