"""NaN and infinite positions are refused on the device, before any tree is
built from them.

The bounding-box pass that starts every iteration (and the displacement pass
that ends one) flags a non-finite position; every later kernel of the
iteration then returns at once, the step reports FA2_ERR_DEVICE_LIMIT with
bit 16 in fa2_stats.device_error, and fa2_set_positions with finite
positions clears it.  The tree walk's acceptance vote is written so that a
NaN distance accepts, so a walk never runs past the tree even if such a
position reached it.  The reference has no such check: its kernels build a
tree and walk it from whatever the positions hold."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_NON_FINITE = 16
DEVICE_LIMIT = 5


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_step_refuses_non_finite_positions_and_recovers(ba3k, bad):
    from gpugraphlayout_b200 import Engine, Fa2Error
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 4)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0)
    broken = xy.copy()
    broken[1234, 1] = bad
    e.set_positions(broken)
    with pytest.raises(Fa2Error) as ex:
        e.step(3)
    assert ex.value.status == DEVICE_LIMIT
    assert e.stats()["device_error"] & ERR_NON_FINITE
    # finite positions again: the step runs and matches a fresh engine
    e.set_positions(xy)
    e.step(1)
    assert e.stats()["device_error"] == 0
    f = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0)
    f.set_positions(xy)
    f.step(1)
    assert np.array_equal(e.sort_order(), f.sort_order())


def test_quadrupole_walk_refuses_non_finite_positions(ba3k):
    from gpugraphlayout_b200 import Engine, Fa2Error
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 6)
    xy[[5, 900, 2999], 0] = np.nan
    e = Engine(g.n, g.sources, g.targets, scale=10.0, theta=1.5, multipole=2)
    e.set_positions(xy)
    with pytest.raises(Fa2Error):
        e.step(1)
    assert e.stats()["device_error"] & ERR_NON_FINITE


def test_batch_stops_only_the_graph_with_a_non_finite_position():
    from gpugraphlayout_b200 import BatchEngine, Fa2Error, synth
    from oracle import oracle as O
    graphs = []
    for i, n in enumerate((300, 800, 500)):
        s, t = synth.sbm_edges(n, 4, 0.05, 0.002, 40.0, seed=30 + i)
        graphs.append(O.Graph(s, t))
    xy = [O.random_positions(g.n, 2000, 2000, 40 + i) for i, g in enumerate(graphs)]
    b = BatchEngine([(g.n, g.sources, g.targets) for g in graphs], scale=2.0)
    broken = [a.copy() for a in xy]
    broken[1][17, 0] = np.inf
    b.set_positions(np.concatenate(broken))
    with pytest.raises(Fa2Error) as ex:
        b.step(2)
    assert ex.value.status == DEVICE_LIMIT
    moved = b.get_positions()
    n0, n1 = graphs[0].n, graphs[1].n
    assert not np.array_equal(moved[:n0], xy[0])           # graph 0 stepped
    assert np.array_equal(moved[n0:n0 + n1], broken[1])    # graph 1 did not
    assert not np.array_equal(moved[n0 + n1:], xy[2])      # graph 2 stepped
    b.set_positions(np.concatenate(xy))
    b.step(2)
    assert np.isfinite(b.get_positions()).all()

