"""Identities the engine relies on to skip work, checked with the oracle (the
reference's Expand and Prune rules restated on the CPU).

* Expand: while the defined values stay within half the width reached, each
  cycle depends only on the width it starts from, so expanding to an
  intermediate width and then on gives the direct result.  The engine takes
  the RK copy of the top level set at that intermediate width during the
  first stage's Expand instead of expanding the copy separately.
* Prune: after a Prune with stray-zero removal that met no defined value
  +-0, a Prune without it changes nothing.  The engine then only copies the
  masks in the second pass of the pair.
"""
import numpy as np
import pytest

from viennals_b200 import BoundaryConditionEnum as BC, Grid
from viennals_b200.geometry import sdf_levelset


def _oracle():
    from oracle import oracle as O

    return O


def _grid():
    return Grid([-5, 5, -5, 5, -5, 5], [BC.INFINITE_BOUNDARY] * 3, 0.15)


def _sphere(g, half):
    return sdf_levelset(g, lambda x, y, z: np.sqrt(x * x + y * y + z * z) - 1.5,
                        [-22] * 3, [22] * 3, half_width=half)


def _same(a, b):
    ia, va = a.points()
    ib, vb = b.points()
    assert np.array_equal(ia, ib)
    assert np.array_equal(va.view(np.int64), vb.view(np.int64))  # bit for bit, signs of zero too


@pytest.mark.parametrize("half,mid,final", [(1.0, 4, 7), (1.0, 3, 7), (1.0, 3, 4), (1.5, 4, 9),
                                            (1.0, 4, 11), (1.5, 4, 8)])
def test_expand_in_two_legs_equals_direct(half, mid, final):
    O = _oracle()
    g = _grid()
    s = O.OracleLS(g, _sphere(g, half))
    direct = s.copy()
    direct.expand(final)
    split = s.copy()
    split.expand(mid)
    assert split.width == mid
    split.expand(final)
    assert direct.width == split.width == final
    _same(direct, split)


def _noisy_band(g, seed, zeros):
    dom = _sphere(g, 2.0)  # width 4, like the stage combination's input
    rng = np.random.default_rng(seed)
    v = dom.values + rng.uniform(-0.3, 0.3, len(dom.values))
    flip = rng.random(len(v)) < 0.05  # isolated cells of the other sign
    v[flip] = -v[flip]
    v[np.abs(v) < 1e-9] = 1e-3
    if zeros:
        v[rng.random(len(v)) < 0.02] = 0.0
    dom.values = v
    return dom


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_second_prune_is_identity_without_zeros(seed):
    O = _oracle()
    g = _grid()
    dom = _noisy_band(g, seed, zeros=False)
    assert not np.any(dom.values == 0.0)
    first = O.OracleLS(g, dom)
    first.prune(True)
    second = first.copy()
    second.prune(False)
    _same(first, second)


def test_prune_pair_with_zeros_needs_both_passes():
    # With zeros the identity fails: a zero neighbour keeps a cell in the
    # first pass only, and a stray zero can take a neighbour's value.  The
    # engine runs the second pass in full then.
    O = _oracle()
    g = _grid()
    dom = _noisy_band(g, 4, zeros=True)
    assert np.any(dom.values == 0.0)
    first = O.OracleLS(g, dom)
    first.prune(True)
    second = first.copy()
    second.prune(False)
    assert len(second.points()[1]) < len(first.points()[1])
