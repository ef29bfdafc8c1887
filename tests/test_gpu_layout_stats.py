"""Final layouts against the oracle by edge-length and stress statistics.

ForceAtlas2 iterates chaotically: two runs whose forces differ by float
rounding drift apart position by position, so a layout after many steps is
judged by what it looks like, not by its coordinates.  Both runs start from
the same positions and take the same number of steps; the engine's layout
must have the oracle's edge-length distribution and the oracle's stress
against graph distances.  The bars come from the oracle itself on this graph:
layouts from two different random starts differ by 0.03 % in mean edge
length, 0.1 % in its coefficient of variation and 2 % in stress, while a 10 %
change of the repulsion strength moves the mean edge length by 5 %.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_MEAN = 0.01   # mean edge length
TOL_CV = 0.02     # coefficient of variation of the edge lengths
TOL_STRESS = 0.05


def _edge_lengths(xy, g):
    from gpugraphlayout_b200.layout_stats import edge_lengths
    return edge_lengths(xy, g.sources, g.targets)


def _stress(xy, g, n_src=24, seed=0):
    from gpugraphlayout_b200.layout_stats import stress
    return stress(xy, g.sources, g.targets, n_src, seed)


@pytest.mark.parametrize("sg,k_r", [(False, 80.0), (True, 10.0)])
def test_layout_statistics_match_oracle(ba3k, sg, k_r):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 1234)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=sg, gravity=1.0, scale=k_r)
    e.set_positions(xy)
    fo = O.FA2(g, xy, k_r, 1.0, sg)
    e.step(60)
    fo.step(60)
    a, b = e.get_positions(), fo.positions
    la, lb = _edge_lengths(a, g), _edge_lengths(b, g)
    assert abs(la.mean() - lb.mean()) <= TOL_MEAN * lb.mean(), (la.mean(), lb.mean())
    cva, cvb = la.std() / la.mean(), lb.std() / lb.mean()
    assert abs(cva - cvb) <= TOL_CV * cvb, (cva, cvb)
    sa, sb = _stress(a, g), _stress(b, g)
    assert abs(sa - sb) <= TOL_STRESS * sb, (sa, sb)
