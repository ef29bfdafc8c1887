"""Parity at the sizes of the benchmark workloads, through the C ABI.

The small-graph suites stop at a few thousand bodies.  The code paths that
only appear at scale are checked here against the oracle:

* R-MAT scale 16 (1,048,576 draws: N = 46,716, E = 909,538), the graph the
  far-field correction trains on: three steps.
* R-MAT scale 20 (16,777,216 draws: N = 646,567, E = 15,702,443), the bench
  graph with the bench's positions: the 127-or-more-tile radix sort, the
  632-tile tree-count look-back, and at the second step the 6-pass sort with
  the fix-up pass (the first tree is no deeper than level 22).
* A batch whose largest graphs have 12,000-20,000 nodes (the top of the
  batched workload's size range, on 1024-thread CTAs).

Bars, as in the small-graph suites: the body sort order is bit-exact (the
reference's sortd at the first step, the reference tree of the engine's own
positions at later steps); gravity + attraction within 1e-5 and the total
force within 1e-4 relative RMSE of the oracle; the global speed within 1e-4
after one step.  At scale 20 the repulsion's relative RMSE against the exact
FP64 pairwise sum on 4,096 sampled bodies must not exceed the reference
walk's own error at the same positions (+1e-4).
"""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GA_TOL = 1e-5
TOT_TOL = 1e-4
K_R, K_G = 10.0, 1.0
WIDTH = 2.0e4

_graphs = {}


def _rmat(scale, draws):
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    if scale not in _graphs:
        s, t = synth.rmat_edges(scale, draws, seed=0)
        _graphs[scale] = O.Graph(s, t)
    return _graphs[scale]


def _engine(g, xy):
    from gpugraphlayout_b200 import Engine
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, gravity=K_G, scale=K_R)
    e.set_positions(xy)
    return e


def _check_step_against_tree(e, g, before, it):
    """The step just taken against the oracle's tree of the positions it
    started from: sort order, gravity + attraction, total force."""
    from oracle import oracle as O
    tree = O.Tree(before, g.mass)
    assert np.array_equal(e.sort_order(), tree.sort().astype(np.uint32)), it
    tot, ga = e.forces()
    ga_ref = O.gravity_attraction(g, before, K_G, True)
    assert rel_rmse(ga, ga_ref) <= GA_TOL, it
    rep_ref, ovf, _ = tree.repulsion(K_R)
    assert not ovf
    assert rel_rmse(tot, ga_ref + rep_ref) <= TOT_TOL, it
    return tree, tot, ga, rep_ref


def test_rmat16_three_steps_match_oracle():
    from oracle import oracle as O
    g = _rmat(16, 1 << 20)
    assert (g.n, g.m) == (46_716, 909_538)
    xy = O.random_positions(g.n, WIDTH, WIDTH, 1234)
    e = _engine(g, xy)
    fo = O.FA2(g, xy, K_R, K_G, True)
    for it in range(3):
        before = e.get_positions()
        e.step(1)
        fo.step(1)
        _check_step_against_tree(e, g, before, it)
        if it == 0:
            # the same step of the oracle's iteration
            assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
            tot, ga = e.forces()
            assert rel_rmse(ga, fo.f_ga.reshape(-1, 2)) <= GA_TOL
            assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) <= TOT_TOL
            assert e.stats()["global_speed"] == pytest.approx(fo.global_speed, rel=1e-4)
            assert rel_rmse(e.get_positions(), fo.positions) <= 1e-5
    # float sums in another order drift apart slowly over the steps
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-3
    assert e.stats()["global_speed"] == pytest.approx(fo.global_speed, rel=1e-3)


def test_rmat20_bench_graph_matches_oracle():
    from oracle import oracle as O
    g = _rmat(20, 1 << 24)
    assert (g.n, g.m) == (646_567, 15_702_443)
    xy = O.random_positions(g.n, WIDTH, WIDTH, 1234)
    e = _engine(g, xy)
    fo = O.FA2(g, xy, K_R, K_G, True)
    e.step(1)
    fo.step(1)
    st = e.stats()
    assert st["sort_passes"] == 8
    assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
    tot, ga = e.forces()
    assert rel_rmse(ga, fo.f_ga.reshape(-1, 2)) <= GA_TOL
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) <= TOT_TOL
    assert st["global_speed"] == pytest.approx(fo.global_speed, rel=1e-4)
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-5

    # second step: the first tree was shallow, so the sort skips its two low
    # digits and the fix-up pass orders the runs of equal high digits
    assert st["max_level"] <= 22
    before = e.get_positions()
    rng = np.random.default_rng(20)
    samples = np.sort(rng.choice(g.n, 4096, replace=False)).astype(np.int32)
    # the engine's FP64 kernel, at the positions the second step starts from
    exact_gpu = e.exact_repulsion(samples.astype(np.uint32))
    e.step(1)
    assert e.stats()["sort_passes"] == 6
    tree, tot, ga, rep_ref = _check_step_against_tree(e, g, before, 1)

    # accuracy against the exact FP64 sum at the same positions
    exact = O.exact_repulsion_f64(tree.xy.reshape(-1, 2), g.mass, K_R, samples)
    err_gpu = rel_rmse((tot - ga)[samples], exact)
    err_ref = rel_rmse(rep_ref[samples], exact)
    assert err_gpu <= err_ref + 1e-4, (err_gpu, err_ref)
    # the engine's own FP64 kernel gives the oracle's exact sum
    assert rel_rmse(exact_gpu, exact) <= 1e-12


def test_batch_with_graphs_at_the_top_of_the_size_range():
    """Graphs of 12,000-20,000 nodes beside small ones, each against the
    oracle: the large CTA class with slots sized for 20,000 nodes."""
    from gpugraphlayout_b200 import BatchEngine, synth
    from oracle import oracle as O
    sizes = [20000, 50, 12000, 3000, 16000, 777]
    graphs = []
    for i, n in enumerate(sizes):
        blocks = 2 + (i * 7) % 31
        s, t = synth.sbm_edges(n, min(blocks, max(2, n // 4)), 0.05, 0.002, 40.0, seed=40 + i)
        graphs.append(O.Graph(s, t))
    assert max(g.n for g in graphs) >= 19_000
    xys = [O.random_positions(g.n, 10000.0, 10000.0, 1234 + i) for i, g in enumerate(graphs)]
    b = BatchEngine([(g.n, g.sources, g.targets) for g in graphs], strong_gravity=False,
                    gravity=1.0, scale=2.0)
    b.configure(4096, 512, 1024)
    b.set_positions(np.concatenate(xys))
    b.step(1)
    tot, ga = b.forces()
    order = b.sort_order()
    pos = b.get_positions()
    gs, _ = b.speeds()
    for i, (g, xy) in enumerate(zip(graphs, xys)):
        fo = O.FA2(g, xy, 2.0, 1.0, False)
        fo.step(1)
        assert np.array_equal(b.part(order, i), fo.sortd.astype(np.uint32)), i
        assert rel_rmse(b.part(ga, i), fo.f_ga.reshape(-1, 2)) <= GA_TOL, i
        assert rel_rmse(b.part(tot, i), fo.f_tot.reshape(-1, 2)) <= TOT_TOL, i
        assert rel_rmse(b.part(pos, i), fo.positions) <= 1e-5, i
        assert gs[i] == pytest.approx(fo.global_speed, rel=1e-4), i
