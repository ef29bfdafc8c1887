"""prevent_overlap on the GPU (fa2_set_prevent_overlap) against the oracle's
restatement of the ForceAtlas2 paper's rule, at the parity bars of the plain
path: bit-exact body order, gravity + attraction within 1e-5, total force
within 1e-4, positions within 1e-5 after one step."""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu


def _setup(n=3000, seed=0, size_hi=25.0):
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(n, 3, seed=seed)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 2000, 2000, 1234)
    sz = np.random.default_rng(seed + 1).uniform(0.0, size_hi, g.n).astype(np.float32)
    return g, xy, sz


@pytest.mark.parametrize("sg,k_r", [(True, 10.0), (False, 80.0)])
def test_one_step_matches_oracle(sg, k_r):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g, xy, sz = _setup()
    e = Engine(g.n, g.sources, g.targets, strong_gravity=sg, gravity=1.0, scale=k_r)
    e.set_positions(xy)
    e.set_prevent_overlap(sz)
    fo = O.FA2(g, xy, k_r, 1.0, sg, sizes=sz)
    e.step(1)
    fo.step(1)
    assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
    tot, ga = e.forces()
    assert rel_rmse(ga, fo.f_ga.reshape(-1, 2)) <= 1e-5
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) <= 1e-4
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-5


def test_overlapping_pairs_drop_over_the_iterations():
    """With sizes, nodes are pushed apart to their borders: after 200 steps
    far fewer edges join overlapping nodes than in the plain run."""
    from gpugraphlayout_b200 import Engine
    g, xy, sz = _setup(2000, seed=4, size_hi=40.0)
    counts = []
    for sizes in (None, sz):
        e = Engine(g.n, g.sources, g.targets, strong_gravity=False, gravity=1.0, scale=2.0)
        e.set_positions(xy)
        if sizes is not None:
            e.set_prevent_overlap(sizes)
        e.step(200)
        p = e.get_positions().astype(np.float64)
        d = np.sqrt(((p[g.sources] - p[g.targets]) ** 2).sum(1))
        counts.append(int((d < sz[g.sources] + sz[g.targets]).sum()))
    assert counts[1] < 0.5 * counts[0], counts


def test_combinations_it_does_not_offer_are_refused():
    from gpugraphlayout_b200 import Engine, Fa2Error, FarFieldMLP
    g, xy, sz = _setup(500)
    e = Engine(g.n, g.sources, g.targets, scale=1.0)
    e.set_positions(xy)
    e.set_prevent_overlap(sz)
    for call in (lambda: e.set_linlog(True), lambda: e.set_approximation(1.0, 2),
                 lambda: e.set_learned_correction(FarFieldMLP(seed=None)),
                 lambda: e.set_accuracy_guard(10, 64)):
        with pytest.raises(Fa2Error) as ex:
            call()
        assert ex.value.status == 7
    bad = sz.copy()
    bad[3] = -1.0
    with pytest.raises(Fa2Error):
        e.set_prevent_overlap(bad)
    e.set_prevent_overlap(None)
    e.set_linlog(True)  # allowed again
    e.step(1)
