"""The batched engine (fa2_batch_*) against the oracle, graph by graph.

Each graph of a batch gets the single-graph iteration: bit-exact body order,
gravity + attraction within 1e-5 and total force within 1e-4 relative RMSE
of the oracle (summation orders differ), positions after one step within
1e-5, over several steps within the single-graph engine's trajectory bar."""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu


def _graphs(sizes, seed=0):
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    out = []
    for i, n in enumerate(sizes):
        blocks = 2 + (i * 7) % 31
        s, t = synth.sbm_edges(n, min(blocks, max(2, n // 4)), 0.05, 0.002, 40.0, seed=seed + i)
        out.append(O.Graph(s, t))
    return out


def _batch(graphs, **kw):
    from gpugraphlayout_b200 import BatchEngine
    return BatchEngine([(g.n, g.sources, g.targets) for g in graphs], **kw)


def _positions(graphs, width=2000.0, seed=7):
    from oracle import oracle as O
    return [O.random_positions(g.n, width, width, seed + i) for i, g in enumerate(graphs)]


@pytest.mark.parametrize("sg,k_r,linlog", [(False, 2.0, False), (True, 10.0, False),
                                           (False, 2.0, True)])
def test_one_step_matches_oracle_per_graph(sg, k_r, linlog):
    from oracle import oracle as O
    graphs = _graphs([50, 3000, 120, 777, 1999, 64, 5000, 300])
    xys = _positions(graphs)
    b = _batch(graphs, strong_gravity=sg, gravity=1.0, scale=k_r, linlog=linlog)
    b.set_positions(np.concatenate(xys))
    b.step(1)
    tot, ga = b.forces()
    order = b.sort_order()
    pos = b.get_positions()
    gs, _ = b.speeds()
    for i, (g, xy) in enumerate(zip(graphs, xys)):
        fo = O.FA2(g, xy, k_r, 1.0, sg, linlog=linlog)
        fo.step(1)
        assert np.array_equal(b.part(order, i), fo.sortd.astype(np.uint32)), i
        assert rel_rmse(b.part(ga, i), fo.f_ga.reshape(-1, 2)) <= 1e-5, i
        assert rel_rmse(b.part(tot, i), fo.f_tot.reshape(-1, 2)) <= 1e-4, i
        assert rel_rmse(b.part(pos, i), fo.positions) <= 1e-5, i
        assert gs[i] == pytest.approx(fo.global_speed, rel=1e-4), i


def test_trajectory_tracks_the_single_graph_engine():
    """5 iterations of every graph in one launch against one Engine per graph
    (the bar of the single-graph trajectory test against the oracle: float
    sums in another order drift apart over the steps)."""
    from gpugraphlayout_b200 import Engine
    graphs = _graphs([200, 1500, 50, 4000])
    xys = _positions(graphs, seed=3)
    b = _batch(graphs, scale=2.0)
    b.set_positions(np.concatenate(xys))
    b.step(5)
    pos = b.get_positions()
    gs, se = b.speeds()
    for i, (g, xy) in enumerate(zip(graphs, xys)):
        e = Engine(g.n, g.sources, g.targets, scale=2.0)
        e.set_positions(xy)
        e.step(5)
        assert rel_rmse(b.part(pos, i), e.get_positions()) <= 1e-3, i
        st = e.stats()
        assert gs[i] == pytest.approx(st["global_speed"], rel=1e-3), i
        assert se[i] == pytest.approx(st["speed_efficiency"], rel=1e-3), i


def test_one_launch_of_many_iterations_equals_one_launch_per_iteration():
    """A CTA runs all iterations of a graph before taking the next: the same
    arithmetic, bit for bit, as one launch per iteration."""
    graphs = _graphs([300, 2000, 90])
    xys = _positions(graphs, seed=5)
    a = _batch(graphs, scale=2.0)
    a.set_positions(np.concatenate(xys))
    a.step(12)
    b = _batch(graphs, scale=2.0)
    b.set_positions(np.concatenate(xys))
    for _ in range(12):
        b.step(1)
    assert np.array_equal(a.get_positions(), b.get_positions())
    assert np.array_equal(a.speeds()[0], b.speeds()[0])


def test_coincident_bodies_replayed_like_oracle():
    from oracle import oracle as O
    graphs = _graphs([400, 90])
    xys = _positions(graphs, width=500.0, seed=4)
    xys[0][7] = xys[0][3]
    xys[0][11] = xys[0][3]
    xys[1][20] = xys[1][19]
    b = _batch(graphs, scale=1.0, strong_gravity=True)
    b.set_positions(np.concatenate(xys))
    b.step(1)
    tot, ga = b.forces()
    order = b.sort_order()
    for i, (g, xy) in enumerate(zip(graphs, xys)):
        fo = O.FA2(g, xy, 1.0, 1.0, True)
        fo.step(1)
        assert np.array_equal(b.part(order, i), fo.sortd.astype(np.uint32)), i
        assert rel_rmse(b.part(ga, i), fo.f_ga.reshape(-1, 2)) < 1e-5, i
        assert rel_rmse(b.part(tot, i), fo.f_tot.reshape(-1, 2)) < 1e-4, i


def test_batch_results_do_not_depend_on_the_other_graphs():
    """A graph laid out alone and inside a batch gives the same bits."""
    graphs = _graphs([1000, 300, 2500])
    xys = _positions(graphs, seed=11)
    b = _batch(graphs, scale=2.0)
    b.set_positions(np.concatenate(xys))
    b.step(5)
    solo = _batch(graphs[1:2], scale=2.0)
    solo.set_positions(xys[1])
    solo.step(5)
    assert np.array_equal(b.part(b.get_positions(), 1), solo.get_positions())


def test_results_do_not_depend_on_the_cta_sizes():
    """Graphs up to a size on 256- or 512-thread CTAs beside the rest on
    1024-thread CTAs: stable sort, exact integer sums, per-warp walks and
    fixed-order speed sums make every graph's steps bit-identical."""
    graphs = _graphs([50, 3000, 120, 777, 1999, 64, 5000, 300, 40, 2500])
    xy = np.concatenate(_positions(graphs))
    runs = []
    for split, threads, large in ((0, 256, 1024), (1000, 256, 1024), (3000, 512, 1024),
                                  (10000, 256, 1024), (0, 256, 512), (500, 256, 512)):
        b = _batch(graphs, scale=2.0)
        b.configure(split, threads, large)
        assert b.config() == {"split": split, "small_threads": threads, "large_threads": large}
        b.set_positions(xy)
        b.step(3)
        runs.append((b.get_positions(), b.sort_order(), b.speeds()))
    for pos, order, (gs, se) in runs[1:]:
        assert np.array_equal(pos, runs[0][0])
        assert np.array_equal(order, runs[0][1])
        assert np.array_equal(gs, runs[0][2][0]) and np.array_equal(se, runs[0][2][1])


def test_autotune_leaves_the_layout_state_as_it_was():
    from gpugraphlayout_b200 import Fa2Error
    graphs = _graphs([50, 3000, 120, 777, 1999, 64, 5000, 300])
    xy = np.concatenate(_positions(graphs))
    b = _batch(graphs, scale=2.0)
    b.set_positions(xy)
    b.step(2)
    before = (b.get_positions(), b.sort_order(), b.speeds())
    cfg = b.autotune(2)
    assert cfg["small_threads"] in (256, 512) and cfg["ms_per_iter"] > 0
    assert b.config() == {"split": cfg["split"], "small_threads": cfg["small_threads"],
                          "large_threads": cfg["large_threads"]}
    after = (b.get_positions(), b.sort_order(), b.speeds())
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
    assert np.array_equal(before[2][0], after[2][0])
    # and the steps that follow are those of an untuned batch
    ref = _batch(graphs, scale=2.0)
    ref.set_positions(xy)
    ref.step(4)
    b.step(2)
    assert np.array_equal(b.get_positions(), ref.get_positions())
    with pytest.raises(Fa2Error):
        b.configure(100, 128, 1024)
