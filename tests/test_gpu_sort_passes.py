"""The sort's low digits after a shallow tree.

When the last tree was no deeper than level 22, the next sort skips its two
lowest 8-bit digits (quadrant levels 24..31); no deeper than 26, its lowest
one (levels 28..31).  A fix-up kernel then sorts each run of keys equal in
the sorted digits by the full key.  That gives the
order of the full sort exactly.  A run longer than 1024 bodies instead
replays the iteration with every digit.  Both paths must leave the body
order bit-exact with the oracle's (the reference's in-order tree sort).

Two anchor bodies pin the root box to [-1024, 1024]^2, so a level-24 cell is
2048 / 2^24 wide and the cell [0, w)^2 can hold a whole cluster: its bodies
share 24 quadrant digits but, spaced wider than a level-32 cell, no 64-bit
key.
"""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu

W24 = 2048.0 / 2 ** 24   # level-24 cell width
SPACING = 1.6e-6          # > a level-32 cell (2048 / 2^32 = 4.8e-7)


def _anchored(g, seed):
    from oracle import oracle as O
    xy = O.random_positions(g.n, 2000, 2000, seed)
    xy[0] = (-1024.0, -1024.0)
    xy[1] = (1024.0, 1024.0)
    return xy


def _cluster(xy, first, count, cols):
    """count bodies from index `first` on a grid inside the level-24 cell
    [0, W24)^2, centred in it."""
    xy = xy.copy()
    rows = (count + cols - 1) // cols
    x0 = W24 / 2 - SPACING * (cols - 1) / 2
    y0 = W24 / 2 - SPACING * (rows - 1) / 2
    for j in range(count):
        xy[first + j] = (x0 + SPACING * (j % cols), y0 + SPACING * (j // cols))
    return xy


def _engine_after_shallow_step(g, seed):
    from gpugraphlayout_b200 import Engine
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0)
    e.set_positions(_anchored(g, seed))
    e.step(1)
    assert 0 < e.stats()["max_level"] <= 22  # the next sort skips two digits
    assert e.stats()["sort_passes"] == 8
    return e


def test_short_low_digit_runs_are_fixed_exactly(ba3k):
    from oracle import oracle as O
    g = ba3k
    e = _engine_after_shallow_step(g, 31)
    xy = _anchored(g, 32)
    for c in range(12):  # twelve runs of 8 bodies, each in its own level-24 cell
        xy = _cluster(xy, 2 + 8 * c, 8, 4)
        xy[2 + 8 * c: 10 + 8 * c, 0] += c * W24
    e.set_positions(xy)
    e.step(1)
    assert e.stats()["max_level"] >= 24
    t = O.Tree(xy, g.mass)
    assert np.array_equal(e.sort_order(), t.sort().astype(np.uint32))
    tot, ga = e.forces()
    ref, ovf, _ = t.repulsion(10.0)
    if not ovf:
        assert rel_rmse(tot - ga, ref) <= 1e-4


def test_a_run_too_long_for_the_fix_up_replays_with_every_digit(ba3k):
    from oracle import oracle as O
    g = ba3k
    e = _engine_after_shallow_step(g, 33)
    xy = _cluster(_anchored(g, 34), 2, 1100, 34)
    e.set_positions(xy)
    e.step(1)
    st = e.stats()
    assert st["device_error"] == 0
    assert st["perturb_rounds"] >= 1  # the replay with the full sort
    assert np.array_equal(e.sort_order(), O.Tree(xy, g.mass).sort().astype(np.uint32))
    # and the layout goes on from there
    e.step(3)
    assert np.isfinite(e.get_positions()).all()


def test_seven_passes_after_a_tree_of_depth_26(ba3k):
    """A pair sharing 26 quadrant digits makes the tree 26 deep: the next
    sort skips one digit (levels 28..31), and clusters sharing 28 digits are
    put in order by the fix-up."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    w26, w28 = 2048.0 / 2 ** 26, 2048.0 / 2 ** 28
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0)
    xy = _anchored(g, 35)
    xy[2] = (0.25 * w26, 0.25 * w26)
    xy[3] = (0.75 * w26, 0.75 * w26)
    e.set_positions(xy)
    e.step(1)
    assert e.stats()["max_level"] == 26
    xy = _anchored(g, 36)
    for c in range(10):  # ten 2 x 2 clusters, each centred in its own level-28 cell
        for j in range(4):
            xy[2 + 4 * c + j] = ((c + 0.5) * w28 + SPACING * (j % 2 - 0.5),
                                 0.5 * w28 + SPACING * (j // 2 - 0.5))
    e.set_positions(xy)
    e.step(1)
    assert e.stats()["sort_passes"] == 7
    assert np.array_equal(e.sort_order(), O.Tree(xy, g.mass).sort().astype(np.uint32))
