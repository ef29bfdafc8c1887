"""Edge cases of the CUDA engine against the oracle, through the C ABI.

* coincident bodies: the replay path scales later bodies by .99 (reference
  intent, src/RPBHKernels.cu:271-278) -- same sort order and forces as the
  oracle's sequential insertion;
* a pair that separates below level 32: sort order still equals the
  reference's in-order (deep digits), and the engine keeps computing
  repulsion (the reference adds none past depth 32);
* tiny graphs, clustered layouts, parameter changes, the speed state, invalid
  input, the Python mirror of the C++ interface and the graph_viewer CLI.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_rmse

pytestmark = pytest.mark.gpu


def _engine(g, xy, k_r=1.0, k_g=1.0, sg=True):
    from gpugraphlayout_b200 import Engine
    e = Engine(g.n, g.sources, g.targets, strong_gravity=sg, gravity=k_g, scale=k_r)
    e.set_positions(xy)
    return e


def test_coincident_bodies_replayed_like_oracle():
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(400, 2, seed=2)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 500, 500, 4)
    xy[7] = xy[3]
    xy[11] = xy[3]
    xy[20] = xy[19]
    e = _engine(g, xy)
    e.step(1)
    assert e.stats()["perturb_rounds"] >= 1
    fo = O.FA2(g, xy, 1.0, 1.0, True)
    fo.step(1)
    assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
    tot, ga = e.forces()
    assert rel_rmse(ga, fo.f_ga.reshape(-1, 2)) < 1e-5
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) < 1e-4
    # a second step from there needs no replay
    e.step(1)
    assert e.stats()["perturb_rounds"] == 0


def test_deep_pair_order_and_repulsion():
    from oracle import oracle as O
    g = O.Graph(np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32))
    xy = np.array([[-1024.0, -1024.0], [1024.0, 1024.0], [2.0 ** -25, 0.0],
                   [1.5 * 2.0 ** -24, 0.0]], np.float32)
    e = _engine(g, xy)
    e.step(1)
    t = O.Tree(xy, g.mass)
    assert t.maxdepth > 32
    assert np.array_equal(e.sort_order(), t.sort().astype(np.uint32))
    assert e.stats()["max_level"] == 32
    tot, ga = e.forces()
    rep = tot - ga
    assert np.abs(rep).sum() > 0  # the reference adds nothing here
    exact = O.exact_repulsion_f64(xy, g.mass, 1.0, np.arange(4, dtype=np.int32))
    # Below level ~21 the cell threshold (2w)^2 is under the softening eps,
    # so in float d^2+eps and dq+eps both round to eps and the reference's
    # rule takes the pair's own cell whole: a ~1e-3 effect, not exactness.
    assert rel_rmse(rep, exact) < 1e-2


@pytest.mark.parametrize("pairs", [[(0, 1)], [(0, 1), (1, 2)], [(5, 9), (9, 2), (2, 5), (7, 5)]])
def test_tiny_graphs(pairs):
    from oracle import oracle as O
    s = np.array([p[0] for p in pairs], np.uint32)
    t = np.array([p[1] for p in pairs], np.uint32)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 100, 100, 3)
    e = _engine(g, xy)
    fo = O.FA2(g, xy, 1.0, 1.0, True)
    for _ in range(3):
        e.step(1)
        fo.step(1)
        assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
        assert rel_rmse(e.get_positions(), fo.positions) < 1e-5


def test_clustered_layout_matches_oracle():
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.sbm_edges(6000, 12, 0.05, 0.002, 40, seed=3)
    g = O.Graph(s, t)
    rng = np.random.default_rng(5)
    centres = rng.uniform(-5000, 5000, size=(12, 2))
    xy = (centres[np.arange(g.n) % 12] + rng.normal(0, 2.0, size=(g.n, 2))).astype(np.float32)
    e = _engine(g, xy, k_r=2.0, sg=False)
    fo = O.FA2(g, xy, 2.0, 1.0, False)
    e.step(1)
    fo.step(1)
    assert np.array_equal(e.sort_order(), fo.sortd.astype(np.uint32))
    tot, _ = e.forces()
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) < 1e-4


def test_set_force_params_and_speed_state(ba3k):
    from oracle import oracle as O
    g = ba3k
    xy = O.random_positions(g.n, 2000, 2000, 11)
    e = _engine(g, xy, k_r=10.0)
    e.set_force_params(80.0, 2.0)
    e.step(1)
    fo = O.FA2(g, xy, 80.0, 2.0, True)
    fo.step(1)
    tot, _ = e.forces()
    assert rel_rmse(tot, fo.f_tot.reshape(-1, 2)) < 1e-4
    gs, se, fp = e.speed_state()
    assert gs == pytest.approx(fo.global_speed, rel=1e-5)
    # restore a checkpoint and continue: same as never having stopped
    pos = e.get_positions()
    e.step(2)
    after = e.get_positions()
    e.set_positions(pos)
    e.set_speed_state(gs, se, fp)
    e.step(2)
    assert np.array_equal(e.get_positions(), after)


def test_timed_steps_take_the_same_steps(ba3k):
    """fa2_step_timed, with per-kernel events or without, runs the iterations
    fa2_step runs: the same positions bit for bit, and a positive time."""
    from oracle import oracle as O
    xy = O.random_positions(ba3k.n, 2000, 2000, 8)
    ref = _engine(ba3k, xy, k_r=10.0)
    ref.step(6)
    for kernels in (False, True):
        e = _engine(ba3k, xy, k_r=10.0)
        ms, kms = e.step_timed(6, kernels=kernels)
        assert ms > 0.0
        assert bool(kms) == kernels
        if kernels:
            assert kms["traverse"] > 0.0 and kms["attract"] > 0.0
        assert np.array_equal(e.get_positions(), ref.get_positions())


@pytest.mark.parametrize("iters", [1, 5])
def test_step_host_equals_the_three_calls(ba3k, iters):
    """fa2_step_host (positions in, iterations, positions out, one host
    synchronisation) against fa2_set_positions + fa2_step + fa2_get_positions:
    the same positions and forces bit for bit, for several round trips in a
    row, with the input and output in one buffer, and with either side left
    out."""
    from oracle import oracle as O
    xy = O.random_positions(ba3k.n, 2000, 2000, 21)
    a = _engine(ba3k, xy, k_r=10.0)
    b = _engine(ba3k, xy, k_r=10.0)
    host = xy.copy()
    for _ in range(3):
        a.set_positions(host)
        a.step(iters)
        want = a.get_positions()
        b.step_host(host, iters, host)  # in and out in the same buffer
        assert np.array_equal(host, want)
        assert np.array_equal(b.forces()[0], a.forces()[0])
    # no input: from the device's positions; no output: positions stay there
    a.step(iters)
    b.step_host(None, iters, None)
    assert np.array_equal(b.get_positions(), a.get_positions())
    out = np.zeros_like(host)
    b.step_host(None, 0, out)
    assert np.array_equal(out, a.get_positions())
    with pytest.raises(ValueError):
        b.step_host(np.zeros((3, 2), np.float32), 1, None)


def test_step_host_replays_coincident_bodies():
    """A round trip whose first iteration must be replayed (coincident
    bodies) gives what the three calls give."""
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(400, 2, seed=2)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 500, 500, 4)
    xy[7] = xy[3]
    xy[11] = xy[3]
    xy[20] = xy[19]
    a = _engine(g, xy)
    a.step(3)
    assert a.stats()["perturb_rounds"] >= 1  # the first of the 3 was replayed
    want = a.get_positions()
    b = _engine(g, xy)
    out = np.zeros_like(xy)
    b.step_host(xy, 3, out)
    assert np.array_equal(out, want)
    assert np.array_equal(b.sort_order(), a.sort_order())


def test_deterministic_repeat(ba3k):
    from oracle import oracle as O
    xy = O.random_positions(ba3k.n, 2000, 2000, 5)
    runs = []
    for _ in range(2):
        e = _engine(ba3k, xy, k_r=10.0)
        e.step(10)
        runs.append(e.get_positions())
        e.close()
    assert np.array_equal(runs[0], runs[1])


def test_invalid_input_is_reported():
    from gpugraphlayout_b200 import Engine, Fa2Error
    with pytest.raises(Fa2Error) as ei:
        Engine(3, [0, 1], [1, 1])  # self-loop
    assert ei.value.status == 1
    with pytest.raises(Fa2Error) as ei:
        Engine(3, [0], [3])  # id out of range
    assert ei.value.status == 1
    with pytest.raises(Fa2Error) as ei:
        Engine(3, [0], [1], use_barneshut=False)
    assert ei.value.status == 7


def test_python_mirror_and_writers(tmp_path):
    """UGraph / GraphLayout / CUDAForceAtlas2 mirror; the bin writer writes the
    reference's record layout (uint32 edge-list id, float x, float y)."""
    import gpugraphlayout_b200 as G
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(1500, 3, seed=4)
    path = str(tmp_path / "ba.txt")
    synth.write_edgelist(path, s[::-1] + 7, t[::-1] + 7)
    g = G.UGraph(path)
    layout = G.GraphLayout(g)
    fa2 = G.CUDAForceAtlas2(layout, True, False, 1.0, 80.0)
    fa2.doSteps(20)
    fa2.sync_layout()
    out = str(tmp_path / "o.bin")
    layout.writeToBin(out)
    rec = np.fromfile(out, dtype=[("id", "<u4"), ("x", "<f4"), ("y", "<f4")])
    assert np.array_equal(rec["id"], g.node_map_r)
    assert np.array_equal(np.stack([rec["x"], rec["y"]], 1), layout.xy)
    assert np.isfinite(layout.xy).all()


def test_graph_viewer_cli_matches_api(tmp_path):
    """graph_viewer gpu ... bin: same file as the Python mirror with the CLI's
    defaults (srandom(1234), 10000 x 10000 box)."""
    import gpugraphlayout_b200 as G
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(2000, 3, seed=6)
    path = str(tmp_path / "g.txt")
    synth.write_edgelist(path, s, t)
    outdir = tmp_path / "out"
    outdir.mkdir()
    exe = os.path.join(ROOT, "gpugraphlayout_b200", "graph_viewer")
    r = subprocess.run([exe, "gpu", "30", "1", "sg", "10", "1", "approximate", path, str(outdir),
                        "bin"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "fetched" in r.stdout
    rec = np.fromfile(str(outdir / "g.txt_30.bin"), dtype=[("id", "<u4"), ("x", "<f4"), ("y", "<f4")])
    g = G.UGraph(path)
    layout = G.GraphLayout(g)
    fa2 = G.CUDAForceAtlas2(layout, True, True, 1.0, 10.0)
    for _ in range(30):
        fa2.doStep()
    fa2.sync_layout()
    assert np.array_equal(rec["id"], g.node_map_r)
    assert np.array_equal(np.stack([rec["x"], rec["y"]], 1), layout.xy)
    # an existing output file is refused, as in the reference
    r2 = subprocess.run([exe, "gpu", "30", "1", "sg", "10", "1", "approximate", path, str(outdir),
                         "bin"], capture_output=True, text=True, timeout=300)
    assert r2.returncode != 0 and "File exists" in r2.stdout
    # exact mode is refused on the GPU path
    r3 = subprocess.run([exe, "gpu", "3", "1", "sg", "10", "1", "exact", path, str(outdir), "bin"],
                        capture_output=True, text=True, timeout=60)
    assert r3.returncode != 0 and "requires Barnes-Hut" in r3.stderr


def test_graphs_of_no_and_one_node():
    """No nodes: every call works and does nothing.  One node: the tree is the
    root cell and the body, the body's own term is zero, so only gravity
    moves it, towards the origin."""
    from gpugraphlayout_b200 import Engine
    none = np.zeros(0, np.uint32)
    e0 = Engine(0, none, none)
    e0.set_positions(np.zeros((0, 2), np.float32))
    e0.step(3)
    assert e0.get_positions().shape == (0, 2)
    e1 = Engine(1, none, none, strong_gravity=True, gravity=1.0, scale=10.0)
    e1.set_positions(np.array([[30.0, 40.0]], np.float32))
    e1.step(1)
    tot, ga = e1.forces()
    assert np.array_equal(tot, ga)  # no repulsion on a lone body
    before = 50.0
    for _ in range(5):
        e1.step(1)
        r = float(np.hypot(*e1.get_positions()[0]))
        assert np.isfinite(r) and r < before
        before = r


def test_batch_with_empty_and_one_node_graphs():
    """Graphs of 0 and 1 nodes in a batch step like the rest, and the other
    graphs' layouts do not depend on them."""
    from gpugraphlayout_b200 import BatchEngine, synth
    from oracle import oracle as O
    s, t = synth.sbm_edges(60, 3, 0.1, 0.01, 40.0, seed=5)
    g = O.Graph(s, t)
    none = np.zeros(0, np.uint32)
    xy = O.random_positions(g.n, 500, 500, 6)
    b = BatchEngine([(0, none, none), (1, none, none), (g.n, g.sources, g.targets)], scale=2.0)
    b.set_positions(np.concatenate([np.zeros((0, 2), np.float32),
                                    np.array([[5.0, -5.0]], np.float32), xy]))
    b.step(4)
    pos = b.get_positions()
    assert pos.shape == (1 + g.n, 2) and np.isfinite(pos).all()
    alone = BatchEngine([(g.n, g.sources, g.targets)], scale=2.0)
    alone.set_positions(xy)
    alone.step(4)
    assert np.array_equal(pos[1:], alone.get_positions())
