"""The quadrupole far-field option (fa2_set_approximation) against the oracle.

multipole 2 adds to every accepted cell the quadrupole term conj(a2 / w^3) of
its far field, a2 = sum m (z - Z)^2 over the cell's bodies about its centre of
mass.  The oracle computes a2 in double precision bottom-up and adds the term
inside its restatement of the reference walk; the engine sums a2 in double
and adds the term in float.  Same tree, same votes: the forces agree to float
rounding (relative RMSE 1e-4, the bar of the monopole parity tests) and the
node visits to 0.1 %.

The point of the option is accuracy per visit: at theta 1.5 the quadrupole
walk is more accurate than the reference's monopole walk at theta 1 while
visiting far fewer nodes.  Errors are measured against the exact all-pairs sum
in double precision (the oracle's on the CPU; the engine's own FP64 kernel is
checked against it to 1e-12).
"""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _rep(e, xy):
    e.set_positions(xy)
    e.step(1)
    tot, ga = e.forces()
    return tot - ga, e.stats()["visits"]


@pytest.mark.parametrize("theta", [1.0, 1.5])
def test_quadrupole_walk_matches_oracle(ba3k, theta):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 5)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0, theta=theta,
               multipole=2)
    rep, visits = _rep(e, xy)
    ref, ovf, ref_visits = O.Tree(xy, g.mass).repulsion(10.0, itolsq=1.0 / theta ** 2,
                                                         multipole=2)
    assert not ovf
    assert rel_rmse(rep, ref) <= TOL
    assert abs(visits - ref_visits) <= 1e-3 * ref_visits, (visits, ref_visits)
    # and it is not the monopole walk
    mono, _, _ = O.Tree(xy, g.mass).repulsion(10.0, itolsq=1.0 / theta ** 2)
    assert rel_rmse(rep, mono) > 3 * TOL


def _relaxed(g, steps=150):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    e = Engine(g.n, g.sources, g.targets, strong_gravity=False, scale=10.0)
    e.set_positions(O.random_positions(g.n, 2000, 2000, 17))
    e.step(steps)
    return e.get_positions()


@pytest.mark.parametrize("layout", ["random", "relaxed"])
def test_quadrupole_at_theta_1_5_beats_monopole_at_theta_1(ba3k, layout):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 5) if layout == "random" else _relaxed(g)
    exact = O.exact_repulsion_f64(xy, g.mass, 10.0, np.arange(g.n, dtype=np.int32))
    e = Engine(g.n, g.sources, g.targets, strong_gravity=False, scale=10.0)
    mono, v_mono = _rep(e, xy)
    e.set_approximation(1.5, 2)
    quad, v_quad = _rep(e, xy)
    err_mono, err_quad = rel_rmse(mono, exact), rel_rmse(quad, exact)
    assert err_quad < err_mono, (err_quad, err_mono)
    assert v_quad < 0.7 * v_mono, (v_quad, v_mono)


def test_set_approximation_switches_between_steps(ba3k):
    """Back to theta 1, multipole 1 after a quadrupole step gives the
    reference's forces again; bad arguments are refused."""
    from gpugraphlayout_b200 import Engine, Fa2Error
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 8)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0)
    e.set_approximation(1.2, 2)
    quad, _ = _rep(e, xy)
    e.set_approximation(1.0, 1)
    mono, _ = _rep(e, xy)
    ref, _, _ = O.Tree(xy, g.mass).repulsion(10.0)
    assert rel_rmse(mono, ref) <= TOL
    assert rel_rmse(quad, ref) > 3 * TOL
    for theta, mp in ((0.0, 1), (-1.0, 2), (1.0, 0), (1.0, 3)):
        with pytest.raises(Fa2Error):
            e.set_approximation(theta, mp)


def test_device_exact_repulsion_matches_oracle(ba3k):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 9)
    e = Engine(g.n, g.sources, g.targets, scale=10.0)
    e.set_positions(xy)
    samples = np.random.default_rng(0).choice(g.n, 257, replace=False).astype(np.int32)
    got = e.exact_repulsion(samples)
    ref = O.exact_repulsion_f64(xy, g.mass, 10.0, samples)
    assert rel_rmse(got, ref) <= 1e-12
    assert e.exact_repulsion(np.zeros(0, np.int32)).shape == (0, 2)


def test_quadrupole_layout_runs_many_steps(ba3k):
    """Fifty quadrupole steps in one call (one CUDA graph replayed): no device
    limit is hit and the layout stays finite."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    e = Engine(g.n, g.sources, g.targets, strong_gravity=False, scale=10.0, theta=1.5,
               multipole=2)
    e.set_positions(O.random_positions(g.n, 2000, 2000, 21))
    e.step(50)
    assert e.stats()["device_error"] == 0
    assert np.isfinite(e.get_positions()).all()


def _with_equal_key_runs(xy, n_runs=25, run=8):
    """Replaces n_runs * run bodies by tight clusters near the origin whose
    bodies share all 32 quadrant digits (runs of equal 64-bit keys)."""
    xy = xy.copy()
    k = 0
    for c in range(n_runs):
        for j in range(run):
            xy[k] = (1e-3 * (c + 1), 1e-3 + 1e-9 * j)
            k += 1
    return xy


def test_moment_scan_beside_the_tree_count_gives_the_same_forces(ba3k):
    """The moment scan runs on the second stream from a copy of the sort's
    order while the tree count reorders runs of equal keys; no cell boundary
    falls inside a run, so the forces equal those of the in-line scan bit for
    bit."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = _with_equal_key_runs(O.random_positions(g.n, 2000, 2000, 12))
    e = Engine(g.n, g.sources, g.targets, scale=10.0, theta=1.5, multipole=2)
    e.set_overlap(False)
    inline, _ = _rep(e, xy)
    assert e.stats()["max_level"] == 32
    e.set_overlap(True)
    beside, _ = _rep(e, xy)
    assert np.array_equal(inline, beside)
    assert np.isfinite(beside).all()


def test_quadrupole_replay_of_coincident_bodies_matches_oracle(ba3k):
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 13)
    xy[7] = xy[3]
    xy[11] = xy[3]
    xy[200] = xy[100]
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0, theta=1.2,
               multipole=2)
    rep, _ = _rep(e, xy)
    assert e.stats()["perturb_rounds"] >= 1
    t = O.Tree(xy, g.mass)  # scales the later coincident bodies as the engine does
    ref, ovf, _ = t.repulsion(10.0, itolsq=1.0 / 1.2 ** 2, multipole=2)
    assert not ovf
    assert np.array_equal(e.sort_order(), t.sort().astype(np.uint32))
    assert rel_rmse(rep, ref) <= TOL


def test_accuracy_guard_errors_match_the_oracle(ba3k):
    """With as many samples as bodies the guard compares every body: its two
    errors are the relative RMSEs of the step's repulsion and of the
    reference walk against the oracle's FP64 sum.  The quadrupole walk at
    theta 1.5 is the more accurate, so it is kept."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 14)
    exact = O.exact_repulsion_f64(xy, g.mass, 10.0, np.arange(g.n, dtype=np.int32))
    plain_engine = Engine(g.n, g.sources, g.targets, scale=10.0)
    plain, _ = _rep(plain_engine, xy)
    e = Engine(g.n, g.sources, g.targets, scale=10.0, theta=1.5, multipole=2)
    e.set_accuracy_guard(1, g.n)
    rep, _ = _rep(e, xy)
    gd = e.accuracy_guard()
    assert gd["checks"] == 1 and gd["fallbacks"] == 0
    assert gd["err_current"] == pytest.approx(rel_rmse(rep, exact), rel=1e-9)
    # the guard keeps the reference walk's sum itself; a step's repulsion is
    # read back as (gravity + attraction + repulsion) - (gravity + attraction),
    # rounded twice in float, which moves the error by about 1e-5 of itself
    assert gd["err_plain"] == pytest.approx(rel_rmse(plain, exact), rel=1e-4)
    assert gd["err_current"] < gd["err_plain"]


def test_accuracy_guard_falls_back_to_the_reference_walk(ba3k):
    """A monopole walk at theta 2.5 is less accurate than the reference's at
    theta 1: the first check switches the context to the reference walk, whose
    forces then equal a plain engine's bit for bit, and checks stop."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 15)
    e = Engine(g.n, g.sources, g.targets, scale=10.0)
    e.set_approximation(2.5, 1)
    e.set_accuracy_guard(2, 512)
    e.set_positions(xy)
    e.step(5)
    gd = e.accuracy_guard()
    assert gd["checks"] == 1 and gd["fallbacks"] == 1
    assert gd["err_current"] > gd["err_plain"] > 0
    after, _ = _rep(e, xy)
    plain, _ = _rep(Engine(g.n, g.sources, g.targets, scale=10.0), xy)
    assert np.array_equal(after, plain)
    e.step(4)
    assert e.accuracy_guard()["checks"] == 1
