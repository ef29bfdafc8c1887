"""Parity of the CUDA engine (through the C ABI) with the oracle.

Bit-exact: body sort order (the reference's sortd), mass/CSR-derived values.
Tolerances (float32 sums in a different order than the reference's atomics):
  * gravity + attraction: relative RMSE <= 1e-5 against the oracle;
  * total force: relative RMSE <= 1e-4 against the oracle's restatement of
    the reference GPU path (same tree, same warp-vote semantics);
  * repulsion against the FP64 exact pairwise sum: no worse than the
    reference GPU path's own error at theta = 1 (+1e-4 absolute slack).
"""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu

GA_TOL = 1e-5
TOT_TOL = 1e-4


def _engine(g, xy, k_r, k_g, sg):
    from gpugraphlayout_b200 import Engine
    e = Engine(g.n, g.sources, g.targets, strong_gravity=sg, gravity=k_g, scale=k_r)
    e.set_positions(xy)
    return e


@pytest.mark.parametrize("sg,k_r", [(True, 10.0), (False, 80.0)])
def test_one_step_matches_oracle(ba3k, sg, k_r):
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 1234)
    e = _engine(g, xy, k_r, 1.0, sg)
    fo = O.FA2(g, xy, k_r, 1.0, sg)
    e.step(1)
    fo.step(1)
    assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
    tot, ga = e.forces()
    assert rel_rmse(ga, fo.f_ga.reshape(-1, 2)) <= GA_TOL
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) <= TOT_TOL
    st = e.stats()
    assert st["global_speed"] == pytest.approx(fo.global_speed, rel=1e-4)
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-5


def test_trajectory_tracks_oracle(ba3k):
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 1234)
    e = _engine(g, xy, 10.0, 1.0, True)
    fo = O.FA2(g, xy, 10.0, 1.0, True)
    for it in range(5):
        before = e.get_positions()
        e.step(1)
        fo.step(1)
        # the sort order is a function of the positions the step started from
        expect = O.Tree(before, g.mass).sort().astype(np.uint32)
        assert np.array_equal(e.sort_order(), expect), it
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-3


def test_repulsion_error_vs_fp64(ba3k):
    """Repulsion error against the exact FP64 sum is that of the reference GPU path."""
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 7)
    e = _engine(g, xy, 10.0, 1.0, True)
    e.step(1)
    tot, ga = e.forces()
    rep_gpu = tot - ga
    t = O.Tree(xy, g.mass)
    rep_ref, ovf, _ = t.repulsion(10.0)
    assert not ovf
    samples = np.arange(g.n, dtype=np.int32)
    exact = O.exact_repulsion_f64(t.xy.reshape(-1, 2), g.mass, 10.0, samples)
    err_gpu = rel_rmse(rep_gpu, exact)
    err_ref = rel_rmse(rep_ref, exact)
    assert err_gpu <= err_ref + 1e-4, (err_gpu, err_ref)
    assert err_gpu < 0.05


def test_walk_visits_match_oracle(ba3k):
    """Node tests of the warp walk (every accept or open, times the group's
    lanes) against the oracle's restatement of the reference walk on the same
    positions: the same tree and the same vote decide every step, so the counts
    agree up to the rare test that float rounding of a cell centre flips."""
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 99)
    e = _engine(g, xy, 10.0, 1.0, True)
    e.step(1)
    st = e.stats()
    _, ovf, visits = O.Tree(xy, g.mass).repulsion(10.0)
    assert not ovf and visits > 0
    assert abs(st["visits"] - visits) <= 1e-3 * visits, (st["visits"], visits)
    assert 0 < st["interactions"] < st["visits"]


@pytest.mark.parametrize("sg,k_r", [(True, 10.0), (False, 80.0)])
def test_linlog_step_matches_oracle(ba3k, sg, k_r):
    """Linear-log attraction (the reference's CPU use_linlog rule, pinned
    against its own code on the CPU) on the GPU, at the tolerances of the
    linear form."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 1234)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=sg, gravity=1.0, scale=k_r, linlog=True)
    e.set_positions(xy)
    fo = O.FA2(g, xy, k_r, 1.0, sg, linlog=True)
    e.step(1)
    fo.step(1)
    assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
    tot, ga = e.forces()
    assert rel_rmse(ga, fo.f_ga.reshape(-1, 2)) <= GA_TOL
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) <= TOT_TOL
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-5


def test_linlog_switches_between_steps(ba3k):
    """fa2_set_linlog between steps: linear, then linear-log, then linear."""
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 5)
    e = _engine(g, xy, 10.0, 1.0, True)
    fo = O.FA2(g, xy, 10.0, 1.0, True)
    for linlog in (False, True, False):
        e.set_linlog(linlog)
        fo.s.linlog = int(linlog)
        before = e.get_positions()
        e.step(1)
        fo.step(1)
        _, ga = e.forces()
        ga_ref = O.gravity_attraction(g, before, 1.0, True, linlog=linlog)
        assert rel_rmse(ga, ga_ref) <= GA_TOL, linlog
    assert rel_rmse(e.get_positions(), fo.positions) <= 1e-3
