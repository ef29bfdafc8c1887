"""Edge weight influence: fa2_graph_desc.weights with fa2_params.delta.

The reference declares ForceAtlas2::delta (src/RPForceAtlas2.hpp:49, 0 by
default, src/RPForceAtlas2.cpp:49) but its UGraph has no weights and its GPU
path never reads delta.  Here an edge of weight w attracts with w^delta times
the unweighted force, linear or linear-log, the rule F_a = w^delta d of the
ForceAtlas2 paper.  The oracle (orc_attraction_weighted) restates it per
edge; the engine sums the same terms per CSR row, so gravity + attraction
agree to float rounding (the 1e-5 bar of the unweighted parity tests).
"""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu

GA_TOL = 1e-5


def _weights(m, seed):
    return np.random.default_rng(seed).uniform(0.1, 10.0, m).astype(np.float32)


@pytest.mark.parametrize("linlog,delta", [(False, 1.0), (False, 0.5), (True, 1.0), (True, -1.5)])
def test_weighted_attraction_matches_oracle(ba3k, linlog, delta):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    w = _weights(g.m, 3)
    xy = O.random_positions(g.n, 2000, 2000, 6)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0, linlog=linlog,
               weights=w, delta=delta)
    e.set_positions(xy)
    e.step(1)
    _, ga = e.forces()
    ref = O.gravity_attraction(g, xy, 1.0, True, linlog=linlog, weights=w, delta=delta)
    assert rel_rmse(ga, ref) <= GA_TOL
    # and the weights did change the force
    plain = O.gravity_attraction(g, xy, 1.0, True, linlog=linlog)
    assert rel_rmse(ga, plain) > 100 * GA_TOL


def _positions_after(g, xy, steps, **kw):
    from gpugraphlayout_b200 import Engine
    e = Engine(g.n, g.sources, g.targets, strong_gravity=False, scale=10.0, **kw)
    e.set_positions(xy)
    e.step(steps)
    return e.get_positions()


def test_delta_zero_ignores_weights(ba3k):
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 7)
    plain = _positions_after(g, xy, 6)
    assert np.array_equal(_positions_after(g, xy, 6, weights=_weights(g.m, 4), delta=0.0), plain)


def test_unit_weights_equal_unweighted(ba3k):
    """1^delta = 1 exactly: the weighted kernel multiplies every pull by 1.0,
    which leaves the layout bit for bit the same."""
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 8)
    ones = np.ones(g.m, np.float32)
    for linlog in (False, True):
        plain = _positions_after(g, xy, 6, linlog=linlog)
        got = _positions_after(g, xy, 6, linlog=linlog, weights=ones, delta=1.7)
        assert np.array_equal(got, plain), linlog


def test_weighted_layout_follows_oracle(ba3k):
    """Ten steps with weights: the layout stays with the oracle's gravity +
    attraction at every step (checked on the positions before each step)."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    w = _weights(g.m, 5)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0, weights=w, delta=1.0)
    e.set_positions(O.random_positions(g.n, 2000, 2000, 9))
    for _ in range(10):
        before = e.get_positions()
        e.step(1)
        _, ga = e.forces()
        assert rel_rmse(ga, O.gravity_attraction(g, before, 1.0, True, weights=w,
                                                 delta=1.0)) <= GA_TOL
    assert np.isfinite(e.get_positions()).all()


@pytest.mark.parametrize("bad", [0.0, -1.0, np.nan, np.inf])
def test_bad_weights_are_refused(ba3k, bad):
    from gpugraphlayout_b200 import Engine, Fa2Error
    g = ba3k
    w = np.ones(g.m, np.float32)
    w[g.m // 2] = bad
    with pytest.raises(Fa2Error) as ex:
        Engine(g.n, g.sources, g.targets, weights=w, delta=1.0)
    assert ex.value.status == 1
    # with delta 0 the weights are not read
    Engine(g.n, g.sources, g.targets, weights=w, delta=0.0).close()


def test_bad_delta_is_refused(ba3k):
    from gpugraphlayout_b200 import Engine, Fa2Error
    g = ba3k
    w = np.full(g.m, 1e30, np.float32)
    with pytest.raises(Fa2Error):  # w^delta overflows float
        Engine(g.n, g.sources, g.targets, weights=w, delta=2.0)
    with pytest.raises(Fa2Error):
        Engine(g.n, g.sources, g.targets, weights=np.ones(g.m, np.float32), delta=np.nan)


def test_batch_refuses_weights_with_delta():
    import ctypes as C
    from gpugraphlayout_b200 import _native
    from gpugraphlayout_b200 import synth
    L = _native.lib()
    s, t = synth.ba_edges(200, 2, seed=1)
    s = np.ascontiguousarray(s, np.uint32)
    t = np.ascontiguousarray(t, np.uint32)
    w = np.ones(len(s), np.float32)
    descs = (_native.GraphDesc * 1)()
    descs[0] = _native.GraphDesc(int(max(s.max(), t.max()) + 1), len(s), s.ctypes.data,
                                 t.ctypes.data, w.ctypes.data)
    p = _native.Params()
    L.fa2_default_params(C.byref(p))
    p.delta = 1.0
    st = C.c_int(0)
    assert not L.fa2_batch_create(1, descs, C.byref(p), C.byref(st))
    assert st.value == 7  # FA2_ERR_UNSUPPORTED
    p.delta = 0.0
    b = L.fa2_batch_create(1, descs, C.byref(p), C.byref(st))
    assert b and st.value == 0
    L.fa2_batch_destroy(b)
